// Small SU(N) matrix algebra (N = 2, 3) in registers, FP64.
#pragma once

#include "lym_internal.cuh"

namespace lym {

template <int N>
struct Mat {
  cx<double> m[N][N];
};

// reference gauge layout (nd, N, N, V): element (mu, i, j, s)
template <int N>
LYM_D Mat<N> load_link(const double2* __restrict__ U, int mu, int64_t s, int64_t V) {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) r.m[i][j] = ld(U + ((int64_t)(mu * N + i) * N + j) * V + s);
  return r;
}

template <int N>
LYM_D void store_link(double2* __restrict__ U, int mu, int64_t s, int64_t V, const Mat<N>& a) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) st(U + ((int64_t)(mu * N + i) * N + j) * V + s, a.m[i][j]);
}

template <int N>
LYM_D Mat<N> mzero() {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) r.m[i][j] = czero<double>();
  return r;
}

template <int N>
LYM_D Mat<N> mident() {
  Mat<N> r = mzero<N>();
#pragma unroll
  for (int i = 0; i < N; ++i) r.m[i][i] = {1.0, 0.0};
  return r;
}

// A B
template <int N>
LYM_D Mat<N> mul(const Mat<N>& a, const Mat<N>& b) {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<double> t = a.m[i][0] * b.m[0][j];
#pragma unroll
      for (int k = 1; k < N; ++k) cmac(t, a.m[i][k], b.m[k][j]);
      r.m[i][j] = t;
    }
  return r;
}

// A B^dag
template <int N>
LYM_D Mat<N> mul_nd(const Mat<N>& a, const Mat<N>& b) {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<double> t = czero<double>();
#pragma unroll
      for (int k = 0; k < N; ++k) t += a.m[i][k] * conj(b.m[j][k]);
      r.m[i][j] = t;
    }
  return r;
}

// A^dag B
template <int N>
LYM_D Mat<N> mul_dn(const Mat<N>& a, const Mat<N>& b) {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<double> t = czero<double>();
#pragma unroll
      for (int k = 0; k < N; ++k) t += cmul_cj(a.m[k][i], b.m[k][j]);
      r.m[i][j] = t;
    }
  return r;
}

template <int N>
LYM_D void madd(Mat<N>& a, const Mat<N>& b) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) a.m[i][j] += b.m[i][j];
}

template <int N>
LYM_D Mat<N> mscale(cx<double> s, const Mat<N>& a) {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) r.m[i][j] = s * a.m[i][j];
  return r;
}

template <int N>
LYM_D Mat<N> mdag(const Mat<N>& a) {
  Mat<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) r.m[i][j] = conj(a.m[j][i]);
  return r;
}

template <int N>
LYM_D cx<double> trace(const Mat<N>& a) {
  cx<double> t = czero<double>();
#pragma unroll
  for (int i = 0; i < N; ++i) t += a.m[i][i];
  return t;
}

template <int N>
LYM_D double fro2(const Mat<N>& a) {
  double t = 0;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) t += norm2(a.m[i][j]);
  return t;
}

LYM_D cx<double> det(const Mat<2>& a) { return a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0]; }
LYM_D cx<double> det(const Mat<3>& a) {
  return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
         a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
         a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
}

// inverse via the adjugate
LYM_D Mat<2> inverse(const Mat<2>& a) {
  cx<double> d = det(a);
  double n = norm2(d);
  cx<double> id = {d.re / n, -d.im / n};
  Mat<2> r;
  r.m[0][0] = id * a.m[1][1];
  r.m[0][1] = -(id * a.m[0][1]);
  r.m[1][0] = -(id * a.m[1][0]);
  r.m[1][1] = id * a.m[0][0];
  return r;
}
LYM_D Mat<3> inverse(const Mat<3>& a) {
  cx<double> d = det(a);
  double n = norm2(d);
  cx<double> id = {d.re / n, -d.im / n};
  Mat<3> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      // cofactor C_ji for r[i][j]
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3, i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      cx<double> c = a.m[j1][i1] * a.m[j2][i2] - a.m[j1][i2] * a.m[j2][i1];
      r.m[i][j] = id * c;
    }
  return r;
}

// principal N-th root of a non-zero complex number (matches numpy's z ** (1/N))
LYM_D cx<double> principal_root(cx<double> z, int n) {
  double r = sqrt(z.re * z.re + z.im * z.im);
  double ph = atan2(z.im, z.re);
  double rr = pow(r, 1.0 / n);
  double s, c;
  sincos(ph / n, &s, &c);
  return {rr * c, rr * s};
}

LYM_D cx<double> cdiv(cx<double> a, cx<double> b) {
  double n = norm2(b);
  return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}

}  // namespace lym
