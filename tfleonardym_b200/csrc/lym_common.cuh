// Common device/host helpers for the lym (TfLeonardYM hot path) CUDA library.
//
// Layout conventions at the library boundary are the reference's
// (emanueleusai/TfLeonardYM):
//   spinor  (ns, N, V)     complex128, site index fastest      (dirac.py:458-523)
//   gauge   (nd, N, N, V)  complex128, [mu][row][col][site]   (lattice.py:7)
//   site    lexicographic, LAST coordinate fastest             (lattice.py:107-114)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lym.h"

#define LYM_HD __host__ __device__ __forceinline__
#define LYM_D __device__ __forceinline__

namespace lym {

// ---------------------------------------------------------------------------
// complex arithmetic (T = float or double)
// ---------------------------------------------------------------------------
template <typename T>
struct cx {
  T re, im;
};

template <typename T> LYM_HD cx<T> mk(T r, T i) { return cx<T>{r, i}; }
template <typename T> LYM_HD cx<T> operator+(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> LYM_HD cx<T> operator-(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T> LYM_HD cx<T> operator-(cx<T> a) { return {-a.re, -a.im}; }
template <typename T> LYM_HD cx<T> operator*(cx<T> a, cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T> LYM_HD cx<T> operator*(T s, cx<T> a) { return {s * a.re, s * a.im}; }
template <typename T> LYM_HD cx<T> conj(cx<T> a) { return {a.re, -a.im}; }
// conj(a) * b
template <typename T> LYM_HD cx<T> cmul_cj(cx<T> a, cx<T> b) {
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
template <typename T> LYM_HD cx<T>& operator+=(cx<T>& a, cx<T> b) { a.re += b.re; a.im += b.im; return a; }
template <typename T> LYM_HD cx<T>& operator-=(cx<T>& a, cx<T> b) { a.re -= b.re; a.im -= b.im; return a; }
template <typename T> LYM_HD T norm2(cx<T> a) { return a.re * a.re + a.im * a.im; }
template <typename T> LYM_HD cx<T> czero() { return {T(0), T(0)}; }

// Fused complex multiply-accumulate: 4 FMAs instead of the 2 MUL + 2 FMA + 2 ADD
// that `t += a * b` becomes when the product is rounded on its own.
template <typename T> LYM_HD void cmac(cx<T>& t, cx<T> a, cx<T> b) {
  t.re = fma(a.re, b.re, t.re);
  t.re = fma(-a.im, b.im, t.re);
  t.im = fma(a.re, b.im, t.im);
  t.im = fma(a.im, b.re, t.im);
}
// t += conj(a) * b
template <typename T> LYM_HD void cmac_cj(cx<T>& t, cx<T> a, cx<T> b) {
  t.re = fma(a.re, b.re, t.re);
  t.re = fma(a.im, b.im, t.re);
  t.im = fma(a.re, b.im, t.im);
  t.im = fma(-a.im, b.re, t.im);
}

// Multiply by a unit phase encoded as 0:+1, 1:+i, 2:-1, 3:-i (compile-time when possible).
template <typename T> LYM_HD cx<T> mul_phase(int ph, cx<T> a) {
  switch (ph & 3) {
    case 0: return a;
    case 1: return {-a.im, a.re};
    case 2: return {-a.re, -a.im};
    default: return {a.im, -a.re};
  }
}
LYM_HD int phase_conj(int ph) { return (4 - ph) & 3; }
LYM_HD int phase_neg(int ph) { return (ph + 2) & 3; }

// ---------------------------------------------------------------------------
// Spin projection in the reference gamma basis (dirac.py:284-298).
//
// Every gamma_mu there has exactly one non-zero g_a in each upper row a
// (a < ns/2), at a lower column j_a.  For s = +1 (forward hop, 1 - gamma_mu)
// and s = -1 (backward hop, 1 + gamma_mu):
//   half spinor     h_a        = psi_a - s g_a psi_{j_a}
//   lower component out_{j_a} += -s conj(g_a) (U h)_a
// which follows from gamma_mu = gamma_mu^dag and gamma_mu^2 = 1.  The
// reference reaches the same rows through an LU factorisation of the
// projector (dirac.py:320-344, 483-496).
// ---------------------------------------------------------------------------
template <int ND> struct Gamma;

template <> struct Gamma<4> {
  static constexpr int NS = 4;
  // column j_a of upper row a for each mu
  LYM_HD static int col(int mu, int a) {
    // mu0: rows (0->3, 1->2); mu1: (0->3, 1->2); mu2: (0->2, 1->3); mu3: (0->2, 1->3)
    return (mu < 2) ? (3 - a) : (2 + a);
  }
  // phase of g_a: mu0: (-i, -i); mu1: (-1, +1); mu2: (-i, +i); mu3: (+1, +1)
  LYM_HD static int phase(int mu, int a) {
    switch (mu) {
      case 0: return 3;
      case 1: return a == 0 ? 2 : 0;
      case 2: return a == 0 ? 3 : 1;
      default: return 0;
    }
  }
};

template <> struct Gamma<2> {
  static constexpr int NS = 2;
  LYM_HD static int col(int, int) { return 1; }
  // sigma1: g = +1; sigma2: g = -i
  LYM_HD static int phase(int mu, int) { return mu == 0 ? 0 : 3; }
};

// Three dimensions (builder-defined: the reference has fermions in D = 2 and 4 only,
// dirac.py:283-300): two-component spinors with gamma_mu = sigma_{mu+1} (Pauli).
// There is no gamma_5 in odd dimensions, hence no hermitian form Q = gamma_d D; the
// solvers use D^dag = D with gamma_mu -> -gamma_mu.  (1 - s gamma_mu) has rank one:
//   mu = 0 (sigma1): h = psi0 - s psi1,    out0 += t, out1 += -s t
//   mu = 1 (sigma2): h = psi0 + i s psi1,  out0 += t, out1 += -i s t
//   mu = 2 (sigma3): s = +1: h = psi1, out1 += 2t;  s = -1: h = psi0, out0 += 2t
// with t = W h, W the hop's link (U or U^dag).  col / phase give the sigma1, sigma2
// rows in the form the D = 2 code uses; sigma3 goes through proj3 / recon3.
template <> struct Gamma<3> {
  static constexpr int NS = 2;
  LYM_HD static int col(int, int) { return 1; }
  LYM_HD static int phase(int mu, int) { return mu == 0 ? 0 : 3; }
};

template <typename R, int NC>
LYM_HD void proj3(int mu, int s, const cx<R> (&p0)[NC], const cx<R> (&p1)[NC], cx<R> (&h)[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (mu == 0) h[c] = s > 0 ? p0[c] - p1[c] : p0[c] + p1[c];
    else if (mu == 1) h[c] = p0[c] + mul_phase(s > 0 ? 1 : 3, p1[c]);
    else h[c] = s > 0 ? p1[c] : p0[c];
  }
}

template <typename R, int NC>
LYM_HD void recon3(int mu, int s, const cx<R> (&t)[NC], cx<R> (&o0)[NC], cx<R> (&o1)[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (mu == 0) {
      o0[c] += t[c];
      if (s > 0) o1[c] -= t[c];
      else o1[c] += t[c];
    } else if (mu == 1) {
      o0[c] += t[c];
      o1[c] += mul_phase(s > 0 ? 3 : 1, t[c]);
    } else if (s > 0) {
      o1[c] += R(2) * t[c];
    } else {
      o0[c] += R(2) * t[c];
    }
  }
}

// ---------------------------------------------------------------------------
// error handling
// ---------------------------------------------------------------------------
extern thread_local char g_last_error[512];
void set_error(const char* fmt, ...);

#define LYM_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      ::lym::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,           \
                       cudaGetErrorString(e_));                             \
      return LYM_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

#define LYM_CHECK_LAUNCH()                                                  \
  do {                                                                      \
    cudaError_t e_ = cudaGetLastError();                                    \
    if (e_ != cudaSuccess) {                                                \
      ::lym::set_error("%s:%d launch: %s", __FILE__, __LINE__,              \
                       cudaGetErrorString(e_));                             \
      return LYM_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

#define LYM_REQUIRE(cond, code, ...)                                        \
  do {                                                                      \
    if (!(cond)) {                                                          \
      ::lym::set_error(__VA_ARGS__);                                        \
      return code;                                                          \
    }                                                                       \
  } while (0)

inline unsigned grid_for(int64_t n, int block) {
  return (unsigned)((n + block - 1) / block);
}

}  // namespace lym
