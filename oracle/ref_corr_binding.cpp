// Python binding for the reference's correlation operators, compiled from the
// reference sources where they lie (TEST INFRASTRUCTURE ONLY; see build_ref.py).
//
// The reference's own binding file (src/droid.cpp) also declares the Eigen-based
// BA entry points, which cannot be built here, so this file binds only the four
// functions defined in src/correlation_kernels.cu and src/altcorr_kernel.cu,
// with the signatures those files define.
#include <torch/extension.h>
#include <vector>

std::vector<torch::Tensor> corr_index_cuda_forward(torch::Tensor volume, torch::Tensor coords, int radius);
std::vector<torch::Tensor> corr_index_cuda_backward(torch::Tensor volume, torch::Tensor coords,
                                                    torch::Tensor corr_grad, int radius);
std::vector<torch::Tensor> altcorr_cuda_forward(torch::Tensor fmap1, torch::Tensor fmap2, torch::Tensor coords,
                                                torch::Tensor ii, torch::Tensor jj, int radius);
// parameter order of the definition in src/altcorr_kernel.cu:175-182
std::vector<torch::Tensor> altcorr_cuda_backward(torch::Tensor fmap1, torch::Tensor fmap2, torch::Tensor coords,
                                                 torch::Tensor ii, torch::Tensor jj, torch::Tensor grad,
                                                 int radius);

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("corr_index_forward", &corr_index_cuda_forward);
  m.def("corr_index_backward", &corr_index_cuda_backward);
  m.def("altcorr_forward", &altcorr_cuda_forward);
  m.def("altcorr_backward", &altcorr_cuda_backward);
}
