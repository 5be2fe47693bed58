// Host harness for the FP64 Sim(3) code of hi-slam2_b200/hislam2_b200/csrc/sim3.cuh (TEST
// INFRASTRUCTURE).  The kernels of pgo.cu call the same __host__ __device__ functions per
// lane; this program calls them in the same order on the CPU, so tests/test_oracle_pgo.py
// can check the device arithmetic against the float64 oracle without a GPU.
//
//   sim3_host_harness factors IN OUT   IN: int64 N, Np; float poses[N*8]; int64 ii[Np], jj[Np];
//                                      float rel[Np*7]; float infos[Np*49]; double pw
//                                      OUT: double cols[Np*15*7]; float Hsp[4*Np*49];
//                                      float vsp[2*Np*7]; float chi[Np*2]
//   sim3_host_harness retr IN OUT      IN: int64 N, t0, t1; float poses[N*8]; float dx[(t1-t0)*7]
//                                      OUT: float poses[N*8]
//   sim3_host_harness explog IN OUT    IN: int64 n; double xi[n*7]
//                                      OUT: double g[n*8] (exp), double back[n*7] (log of it)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sim3.cuh"

using namespace hs2::sim3;

template <typename T>
static void rd(FILE* f, T* p, size_t n) {
  if (n && fread(p, sizeof(T), n, f) != n) {
    fprintf(stderr, "short read\n");
    std::exit(2);
  }
}

template <typename T>
static void wr(FILE* f, const T* p, size_t n) {
  if (n) fwrite(p, sizeof(T), n, f);
}

int main(int argc, char** argv) {
  if (argc != 4) return 1;
  FILE* in = fopen(argv[2], "rb");
  FILE* out = fopen(argv[3], "wb");
  if (!in || !out) return 1;
  if (!strcmp(argv[1], "factors")) {
    int64_t N, Np;
    rd(in, &N, 1);
    rd(in, &Np, 1);
    std::vector<float> poses(N * 8), rel(Np * 7), infos(Np * 49);
    std::vector<int64_t> ii(Np), jj(Np);
    double pw;
    rd(in, poses.data(), poses.size());
    rd(in, ii.data(), Np);
    rd(in, jj.data(), Np);
    rd(in, rel.data(), rel.size());
    rd(in, infos.data(), infos.size());
    rd(in, &pw, 1);
    std::vector<double> cols(Np * 15 * 7);
    std::vector<float> Hsp(4 * Np * 49), vsp(2 * Np * 7), chi(Np * 2);
    for (int64_t n = 0; n < Np; ++n) {
      float J[15][8];
      float W[2][7][8];
      const Sim3d Gi = from_floats(&poses[8 * ii[n]], true), Gj = from_floats(&poses[8 * jj[n]], true);
      const Sim3d Gij = from_floats(&rel[7 * n], false);
      for (int lane = 0; lane < 15; ++lane) {
        double col[7];
        factor_column(Gi, Gj, Gij, lane, col);
        for (int a = 0; a < 7; ++a) {
          cols[(n * 15 + lane) * 7 + a] = col[a];
          J[lane][a] = (float)col[a];
        }
      }
      const float* inf = &infos[49 * n];
      for (int e = 0; e < 98; ++e) W[e / 49][(e % 49) / 7][e % 7] = wjt_entry(J, inf, e / 49, (e % 49) / 7, e % 7, pw);
      for (int e = 0; e < 196; ++e)
        Hsp[((e / 49) * Np + n) * 49 + e % 49] = hsp_entry(W, J, e / 49, (e % 49) / 7, e % 7);
      for (int e = 0; e < 14; ++e) vsp[((e / 7) * Np + n) * 7 + e % 7] = vsp_entry(W, J, e / 7, e % 7);
      chi[2 * n] = chi_entry(J, inf, 0);
      chi[2 * n + 1] = chi_entry(J, inf, 1);
    }
    wr(out, cols.data(), cols.size());
    wr(out, Hsp.data(), Hsp.size());
    wr(out, vsp.data(), vsp.size());
    wr(out, chi.data(), chi.size());
  } else if (!strcmp(argv[1], "retr")) {
    int64_t N, t0, t1;
    rd(in, &N, 1);
    rd(in, &t0, 1);
    rd(in, &t1, 1);
    std::vector<float> poses(N * 8), dx((t1 - t0) * 7);
    rd(in, poses.data(), poses.size());
    rd(in, dx.data(), dx.size());
    for (int64_t k = 0; k < t1 - t0; ++k) {
      float* p = &poses[8 * (t0 + k)];
      double xi[7];
      for (int a = 0; a < 7; ++a) xi[a] = (double)dx[7 * k + a];
      const Sim3d G = mul(hs2::sim3::exp(xi), from_floats(p, true));
      for (int a = 0; a < 3; ++a) p[a] = (float)G.t[a];
      for (int a = 0; a < 4; ++a) p[3 + a] = (float)G.q[a];
      p[7] = (float)G.s;
    }
    wr(out, poses.data(), poses.size());
  } else if (!strcmp(argv[1], "explog")) {
    int64_t n;
    rd(in, &n, 1);
    std::vector<double> xi(n * 7), g(n * 8), back(n * 7);
    rd(in, xi.data(), xi.size());
    for (int64_t k = 0; k < n; ++k) {
      const Sim3d G = hs2::sim3::exp(&xi[7 * k]);
      for (int a = 0; a < 3; ++a) g[8 * k + a] = G.t[a];
      for (int a = 0; a < 4; ++a) g[8 * k + 3 + a] = G.q[a];
      g[8 * k + 7] = G.s;
      hs2::sim3::log(G, &back[7 * k]);
    }
    wr(out, g.data(), g.size());
    wr(out, back.data(), back.size());
  } else {
    return 1;
  }
  fclose(in);
  fclose(out);
  return 0;
}
