// FP32 / FP64 FMA throughput probes: the denominators for kernels bound by the
// SIMT pipes (the FP32 Schur Gram, the FP64 Cholesky), which the measured HBM
// copy and bf16 GEMM peaks do not cover.  Each thread runs 8 independent FMA
// chains in registers; grid = 8 CTAs of 256 threads per SM.
#include "common.cuh"

namespace hs2 {

template <typename T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T* out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = x[k] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == (T)-1.2345) out[0] = s;  // keeps the chains alive
}

template <typename T>
static int probe(int iters, double* tflops) {
  int dev = 0, sms = 0;
  HS2_CUDA(cudaGetDevice(&dev));
  HS2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  T* out = nullptr;
  HS2_CUDA(cudaMalloc(&out, sizeof(T)));
  cudaEvent_t e0, e1;
  HS2_CUDA(cudaEventCreate(&e0));
  HS2_CUDA(cudaEventCreate(&e1));
  const int blocks = sms * 8;
  fma_probe_kernel<T><<<blocks, 256>>>(out, iters / 8, (T)0.999, (T)0.001);  // warm-up
  HS2_CUDA(cudaEventRecord(e0));
  fma_probe_kernel<T><<<blocks, 256>>>(out, iters, (T)0.999, (T)0.001);
  HS2_CUDA(cudaEventRecord(e1));
  HS2_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  HS2_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = 2.0 * 8.0 * iters * (double)blocks * 256.0 / (ms * 1e-3) / 1e12;
  return HS2_OK;
}

}  // namespace hs2

extern "C" int hs2_measure_simt_peaks(double* fp32_tflops, double* fp64_tflops) {
  using namespace hs2;
  int rc;
  if (fp32_tflops && (rc = probe<float>(1 << 16, fp32_tflops))) return rc;
  if (fp64_tflops && (rc = probe<double>(1 << 13, fp64_tflops))) return rc;
  return HS2_OK;
}
