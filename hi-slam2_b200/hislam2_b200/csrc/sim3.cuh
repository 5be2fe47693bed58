// Sim(3) group in FP64 for the pose-graph terms: the conventions of lietorch's Sim3, which
// HI-SLAM2 uses for them (hislam2/pgo_buffer.py:39-63, hislam2/depth_video.py:244-270).
//   element  [t (3), q (4, x y z w), s]: X -> s R(q) X + t
//   tangent  [tau (3), phi (3), sigma]: the algebra element [[sigma I + [phi]x, tau], [0, 0]]
//   exp      R = Exp(phi), s = e^sigma, t = V tau with V = int_0^1 exp(u (sigma I + [phi]x)) du
//   log      its inverse (phi from the quaternion's principal angle, sigma = log s,
//            tau = V^-1 t)
// The rotation acts by p + w uv + v x uv, uv = 2 v x p, products are Hamilton products and
// the inverse conjugates, as lietorch does, so unnormalised float inputs behave alike.
// Everything is __host__ __device__: the same code runs in the kernels and in the host
// harness the tests compile.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define HS2_HD __host__ __device__ __forceinline__
#else
#define HS2_HD inline
#endif

namespace hs2 {
namespace sim3 {

struct Sim3d {
  double t[3];
  double q[4];
  double s;
};

HS2_HD void cross(const double a[3], const double b[3], double out[3]) {
  out[0] = a[1] * b[2] - a[2] * b[1];
  out[1] = a[2] * b[0] - a[0] * b[2];
  out[2] = a[0] * b[1] - a[1] * b[0];
}

HS2_HD void quat_mul(const double a[4], const double b[4], double out[4]) {
  double c[3];
  cross(a, b, c);
  out[0] = a[3] * b[0] + b[3] * a[0] + c[0];
  out[1] = a[3] * b[1] + b[3] * a[1] + c[1];
  out[2] = a[3] * b[2] + b[3] * a[2] + c[2];
  out[3] = a[3] * b[3] - (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]);
}

HS2_HD void quat_rotate(const double q[4], const double p[3], double out[3]) {
  double uv[3], c[3];
  cross(q, p, uv);
  uv[0] *= 2.0;
  uv[1] *= 2.0;
  uv[2] *= 2.0;
  cross(q, uv, c);
  out[0] = p[0] + q[3] * uv[0] + c[0];
  out[1] = p[1] + q[3] * uv[1] + c[1];
  out[2] = p[2] + q[3] * uv[2] + c[2];
}

HS2_HD Sim3d mul(const Sim3d& a, const Sim3d& b) {
  Sim3d r;
  double Rt[3];
  quat_rotate(a.q, b.t, Rt);
  r.t[0] = a.s * Rt[0] + a.t[0];
  r.t[1] = a.s * Rt[1] + a.t[1];
  r.t[2] = a.s * Rt[2] + a.t[2];
  quat_mul(a.q, b.q, r.q);
  r.s = a.s * b.s;
  return r;
}

HS2_HD Sim3d inv(const Sim3d& a) {
  Sim3d r;
  r.q[0] = -a.q[0];
  r.q[1] = -a.q[1];
  r.q[2] = -a.q[2];
  r.q[3] = a.q[3];
  r.s = 1.0 / a.s;
  double Rt[3];
  quat_rotate(r.q, a.t, Rt);
  r.t[0] = -r.s * Rt[0];
  r.t[1] = -r.s * Rt[1];
  r.t[2] = -r.s * Rt[2];
  return r;
}

// V = int_0^1 exp(u A) du, A = sigma I + [phi]x.  Below |A| = 0.5 the series
// sum_n A^n / (n+1)! (25 terms: truncation < 1e-33, no cancellation); above it the closed
// form a0 I + a1 [phi]x + a2 [phi]x^2 with a0 = (e^s - 1)/s, a1 theta = int e^(s u) sin(theta u),
// a2 theta^2 = a0 - int e^(s u) cos(theta u), whose terms carry only absolute rounding error.
HS2_HD void v_matrix(const double phi[3], double sigma, double V[3][3]) {
  const double th2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
  const double r2 = sigma * sigma + th2;
  if (r2 < 0.25) {
    const double A[3][3] = {{sigma, -phi[2], phi[1]}, {phi[2], sigma, -phi[0]}, {-phi[1], phi[0], sigma}};
    double T[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) V[i][j] = T[i][j];
    for (int n = 1; n <= 25; ++n) {
      double U[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) U[i][j] = (T[i][0] * A[0][j] + T[i][1] * A[1][j] + T[i][2] * A[2][j]) / (n + 1);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          T[i][j] = U[i][j];
          V[i][j] += U[i][j];
        }
    }
    return;
  }
  const double es = ::exp(sigma);
  const double a0 = fabs(sigma) < 1e-12 ? 1.0 + 0.5 * sigma : ::expm1(sigma) / sigma;
  double a1, a2;
  if (th2 < 1e-24) {   // pure scale (|sigma| >= 0.5 here)
    a1 = (es * (sigma - 1.0) + 1.0) / (sigma * sigma);
    a2 = (es * (sigma * sigma - 2.0 * sigma + 2.0) - 2.0) / (2.0 * sigma * sigma * sigma);
  } else {
    const double th = sqrt(th2), sn = sin(th), cs = cos(th);
    const double Is = (es * (sigma * sn - th * cs) + th) / r2;
    const double Ic = (es * (sigma * cs + th * sn) - sigma) / r2;
    a1 = Is / th;
    a2 = (a0 - Ic) / th2;
  }
  const double P[3][3] = {{0, -phi[2], phi[1]}, {phi[2], 0, -phi[0]}, {-phi[1], phi[0], 0}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double P2 = P[i][0] * P[0][j] + P[i][1] * P[1][j] + P[i][2] * P[2][j];
      V[i][j] = (i == j ? a0 : 0.0) + a1 * P[i][j] + a2 * P2;
    }
}

HS2_HD void so3_exp(const double phi[3], double q[4]) {
  const double th2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
  double im, re;
  if (th2 < 1e-8) {
    im = 0.5 - th2 / 48.0 + th2 * th2 / 3840.0;
    re = 1.0 - th2 / 8.0 + th2 * th2 / 384.0;
  } else {
    const double th = sqrt(th2);
    im = sin(0.5 * th) / th;
    re = cos(0.5 * th);
  }
  q[0] = im * phi[0];
  q[1] = im * phi[1];
  q[2] = im * phi[2];
  q[3] = re;
}

// principal rotation vector of q (q and -q are the same rotation)
HS2_HD void so3_log(const double qin[4], double phi[3]) {
  const double sg = qin[3] < 0.0 ? -1.0 : 1.0;
  const double v[3] = {sg * qin[0], sg * qin[1], sg * qin[2]};
  const double w = sg * qin[3];
  const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const double f = n < 1e-8 ? 2.0 / w - 2.0 * n * n / (3.0 * w * w * w) : 2.0 * atan2(n, w) / n;
  phi[0] = f * v[0];
  phi[1] = f * v[1];
  phi[2] = f * v[2];
}

HS2_HD Sim3d exp(const double xi[7]) {
  Sim3d g;
  double V[3][3];
  v_matrix(xi + 3, xi[6], V);
  for (int i = 0; i < 3; ++i) g.t[i] = V[i][0] * xi[0] + V[i][1] * xi[1] + V[i][2] * xi[2];
  so3_exp(xi + 3, g.q);
  g.s = ::exp(xi[6]);
  return g;
}

HS2_HD void log(const Sim3d& g, double xi[7]) {
  so3_log(g.q, xi + 3);
  xi[6] = ::log(g.s);
  double V[3][3];
  v_matrix(xi + 3, xi[6], V);
  // tau = V^-1 t by the adjugate
  const double c00 = V[1][1] * V[2][2] - V[1][2] * V[2][1];
  const double c01 = V[1][2] * V[2][0] - V[1][0] * V[2][2];
  const double c02 = V[1][0] * V[2][1] - V[1][1] * V[2][0];
  const double det = V[0][0] * c00 + V[0][1] * c01 + V[0][2] * c02;
  const double Ai[3][3] = {
      {c00, V[0][2] * V[2][1] - V[0][1] * V[2][2], V[0][1] * V[1][2] - V[0][2] * V[1][1]},
      {c01, V[0][0] * V[2][2] - V[0][2] * V[2][0], V[0][2] * V[1][0] - V[0][0] * V[1][2]},
      {c02, V[0][1] * V[2][0] - V[0][0] * V[2][1], V[0][0] * V[1][1] - V[0][1] * V[1][0]}};
  for (int i = 0; i < 3; ++i) xi[i] = (Ai[i][0] * g.t[0] + Ai[i][1] * g.t[1] + Ai[i][2] * g.t[2]) / det;
}

HS2_HD Sim3d from_floats(const float* p, bool has_scale) {
  Sim3d g;
  for (int i = 0; i < 3; ++i) g.t[i] = (double)p[i];
  for (int i = 0; i < 4; ++i) g.q[i] = (double)p[3 + i];
  g.s = has_scale ? (double)p[7] : 1.0;
  return g;
}

// The relative-pose factor's residual log(Gij Gi Gj^-1) and its central-difference
// Jacobians w.r.t. left perturbations exp(d) Gi and exp(d) Gj, step 1e-8, as
// hislam2/pgo_buffer.py:19-50 forms them.  col in 0..6: Ji column; 7..13: Jj column
// col-7; 14: the residual.  out receives 7 values.
HS2_HD void factor_column(const Sim3d& Gi, const Sim3d& Gj, const Sim3d& Gij, int col, double out[7]) {
  const double eps = 1e-8;
  if (col == 14) {
    log(mul(mul(Gij, Gi), inv(Gj)), out);
    return;
  }
  const int k = col % 7;
  double d[7] = {0, 0, 0, 0, 0, 0, 0};
  double plus[7], minus[7];
  d[k] = eps;
  const Sim3d Ep = exp(d);
  d[k] = -eps;
  const Sim3d Em = exp(d);
  if (col < 7) {
    const Sim3d Gji = inv(Gj);
    log(mul(mul(Gij, mul(Ep, Gi)), Gji), plus);
    log(mul(mul(Gij, mul(Em, Gi)), Gji), minus);
  } else {
    const Sim3d Gb = mul(Gij, Gi);
    log(mul(Gb, inv(mul(Ep, Gj))), plus);
    log(mul(Gb, inv(mul(Em, Gj))), minus);
  }
  for (int i = 0; i < 7; ++i) out[i] = (plus[i] - minus[i]) / 2.0 / eps;
}

// The factor's blocks from its float Jacobians and residual, at the reference's precision
// points (hislam2/pgo_buffer.py:51-62).  J is one factor's [15][8] table: J[k][a] = Ji[a][k]
// for k < 7, J[7 + k][a] = Jj[a][k], J[14][a] = r[a] (each rounded to float, as the
// reference's .type(torch.float32)); info is the factor's 7x7 information matrix.
//   wJT[x][a][b] = float(sum_c (pw * double(Jx[c][a])) * double(info[c][b]))   x = 0: Ji, 1: Jj
//   Hsp[blk][a][b] = sum_c wJT[blk >> 1][a][c] * J(blk & 1)[c][b]   (float)
//   vsp[x][a] = -sum_c wJT[x][a][c] * r[c]
//   chi = (r.r, r.(info r))
HS2_HD float wjt_entry(const float (*J)[8], const float* info, int x, int a, int b, double pw) {
  double acc = 0.0;
  for (int c = 0; c < 7; ++c) acc += (pw * (double)J[7 * x + a][c]) * (double)info[7 * c + b];
  return (float)acc;
}

HS2_HD float hsp_entry(const float (*W)[7][8], const float (*J)[8], int blk, int a, int b) {
  float acc = 0.f;
  for (int c = 0; c < 7; ++c) acc += W[blk >> 1][a][c] * J[7 * (blk & 1) + b][c];
  return acc;
}

HS2_HD float vsp_entry(const float (*W)[7][8], const float (*J)[8], int x, int a) {
  float acc = 0.f;
  for (int c = 0; c < 7; ++c) acc += W[x][a][c] * J[14][c];
  return -acc;
}

HS2_HD float chi_entry(const float (*J)[8], const float* info, int scaled) {
  float acc = 0.f;
  for (int b = 0; b < 7; ++b) {
    float rb = J[14][b];
    if (scaled) {
      float t = 0.f;
      for (int c = 0; c < 7; ++c) t += J[14][c] * info[7 * c + b];
      rb = t;
    }
    acc += rb * J[14][b];
  }
  return acc;
}

}  // namespace sim3
}  // namespace hs2
