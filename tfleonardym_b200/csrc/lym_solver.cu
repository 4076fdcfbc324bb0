// Solvers: the lym_gauge object (even-odd packing of the links), the even-odd
// preconditioned CG on M^dag M with FP64 reliable updates and sloppy inner
// iterations in FP64 / FP32 / norm-scaled FP16 / BF16, the full-lattice
// multishift CG, and the reference's MMMR (dirac_solver.py:19-53).
//
// Even-odd system (builder-defined; the reference has none): with
// D = 1 + kappa H (the reference sign, dirac.py:400,521),
//   b' = b_e - kappa H_eo b_o,  M = 1 - kappa^2 H_eo H_oe,  M x_e = b',
//   x_o = b_o - kappa H_oe x_e,  and M^dag = gamma_d M gamma_d.
// CG runs on M^dag M x_e = M^dag b'.  Iterations run in CUDA graphs (built
// from kernel nodes) of `chunk` iterations; all CG scalars (alpha, beta, |r|^2) stay on the
// device and are produced by the last block of each fused reduction.  A
// right-hand side pauses itself on the device when its sloppy residual drops
// below its pause target; the host then does the FP64 reliable update
// (x += x_sloppy, q = b' - M x, r = M^dag q) for the paused ones and checks
// the true residual |q| against tol |b|.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "lym_eo.cuh"
#include "lym_gauge_obj.cuh"
#include "lym_hop_tc.cuh"
#include "lym_internal.cuh"
#include "lym_kernels.cuh"

namespace lym {

struct CGState {
  double rr;      // |r|^2 of the recursive (sloppy) residual
  double alpha;
  double beta;
  double pause2;  // pause when rr < pause2
  int active;     // iterate while 1
  int iters;
  int max_iter;
  int pause_iter;  // pause at this iteration count at the latest (bounds the sloppy drift)
};

// ---------------------------------------------------------------------------
// geometry helpers
// ---------------------------------------------------------------------------
static EoGeom make_geom(const lym_lattice* lat) {
  EoGeom g{};
  g.nd = lat->nd;
  int st = 1;
  for (int d = lat->nd - 1; d >= 0; --d) {
    g.dims[d] = lat->dims[d];
    g.stride[d] = st;
    st *= lat->dims[d];
  }
  for (int d = lat->nd; d < 4; ++d) {
    g.dims[d] = 1;
    g.stride[d] = 0;
  }
  g.Lh = lat->dims[lat->nd - 1] / 2;
  g.Vh = lat->V / 2;
  return g;
}

// ---------------------------------------------------------------------------
// gauge packing
// ---------------------------------------------------------------------------
template <int GP, int NC>
LYM_D void store_link_eo(void* g, int nunits, int64_t Vh, int mu, int par, int64_t cb, bool comp,
                         const cx<double> (&u)[NC][NC]) {
  const int ncx = comp ? (NC - 1) * NC : NC * NC;
  cx<double> e[NC * NC];
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) e[i * NC + j] = u[i][j];
  if constexpr (GP == SP64) {
    double2* base = reinterpret_cast<double2*>(g) + ((int64_t)(mu * 2 + par) * nunits) * Vh + cb;
    for (int k = 0; k < ncx; ++k) base[k * Vh] = make_double2(e[k].re, e[k].im);
  } else if constexpr (GP == SP32) {
    float4* base = reinterpret_cast<float4*>(g) + ((int64_t)(mu * 2 + par) * nunits) * Vh + cb;
    for (int k = 0; k < nunits; ++k) {
      cx<double> a = 2 * k < ncx ? e[2 * k] : cx<double>{0, 0};
      cx<double> b = 2 * k + 1 < ncx ? e[2 * k + 1] : cx<double>{0, 0};
      base[k * Vh] = make_float4((float)a.re, (float)a.im, (float)b.re, (float)b.im);
    }
  } else {
    uint2* base = reinterpret_cast<uint2*>(g) + ((int64_t)(mu * 2 + par) * nunits) * Vh + cb;
    for (int k = 0; k < nunits; ++k) {
      cx<double> a = 2 * k < ncx ? e[2 * k] : cx<double>{0, 0};
      cx<double> b = 2 * k + 1 < ncx ? e[2 * k + 1] : cx<double>{0, 0};
      base[k * Vh] = make_uint2(pack2<SP16>((float)a.re, (float)a.im), pack2<SP16>((float)b.re, (float)b.im));
    }
  }
}

// Even-odd neighbour table (EoGeom::nbr): one thread per (cb, parity).
template <int ND>
__global__ void build_nbr_kernel(EoGeom g, int* __restrict__ nbr) {
  const int cb = blockIdx.x * blockDim.x + threadIdx.x;
  const int par = blockIdx.y;
  if (cb >= g.Vh) return;
  int x[ND];
  const int lex = eo_coords<ND>(g, cb, par, x);
  const int vh = (int)g.Vh;
#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
    const int up = nb_fwd<ND>(g, lex, x, mu) >> 1;
    const int dn = nb_bwd<ND>(g, lex, x, mu) >> 1;
    const bool tb = mu == ND - 1;
    // forward hop: the link on x crosses when x_t = L-1; backward: the link on x-t when x_t = 0
    nbr[(par * 2 * ND + 2 * mu) * vh + cb] = up | ((tb && x[ND - 1] == g.dims[ND - 1] - 1) ? kNbrBoundary : 0);
    nbr[(par * 2 * ND + 2 * mu + 1) * vh + cb] = dn | ((tb && x[ND - 1] == 0) ? kNbrBoundary : 0);
  }
}

template <int ND, int NC>
__global__ void pack_gauge_kernel(EoGeom g, int64_t V, const double2* __restrict__ ref, double bcr, double bci,
                                  double2* g64, float4* g32, int n32, int comp32, uint2* g16, int n16, int comp16,
                                  float4* g32f, int n32f, uint2* g16f, int n16f) {
  const int64_t lex = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (lex >= V) return;
  int x[ND];
  lex_coords<ND>(g, lex, x);
  int par = 0;
#pragma unroll
  for (int d = 0; d < ND; ++d) par += x[d];
  par &= 1;
  const int64_t cb = lex >> 1;
  cx<double> u[NC][NC], ub[NC][NC];
  const bool edge = (mu == ND - 1) && (x[ND - 1] == g.dims[ND - 1] - 1);
  const cx<double> bc{edge ? bcr : 1.0, edge ? bci : 0.0};
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      u[i][j] = ld(ref + ((int64_t)(mu * NC + i) * NC + j) * V + lex);
      ub[i][j] = bc * u[i][j];
    }
  store_link_eo<SP64, NC>(g64, NC * NC, g.Vh, mu, par, cb, false, ub);
  if (g32) store_link_eo<SP32, NC>(g32, n32, g.Vh, mu, par, cb, comp32, comp32 ? u : ub);
  if (g16) store_link_eo<SP16, NC>(g16, n16, g.Vh, mu, par, cb, comp16, comp16 ? u : ub);
  if (g32f) store_link_eo<SP32, NC>(g32f, n32f, g.Vh, mu, par, cb, false, ub);
  if (g16f) store_link_eo<SP16, NC>(g16f, n16f, g.Vh, mu, par, cb, false, ub);
}

// sum over links of |U U^dag - 1|^2 + |det U - 1|^2
template <int NC>
__global__ void unitarity_kernel(int64_t nl, const double2* __restrict__ ref, int64_t V, double* partials,
                                 unsigned* counter, double* result) {
  __shared__ double sh[32];
  double v[1] = {0.0};
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < nl; l += (int64_t)gridDim.x * blockDim.x) {
    const int mu = (int)(l / V);
    const int64_t s = l - mu * V;
    cx<double> u[NC][NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) u[i][j] = ld(ref + ((int64_t)(mu * NC + i) * NC + j) * V + s);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        cx<double> t = czero<double>();
#pragma unroll
        for (int k = 0; k < NC; ++k) t += u[i][k] * conj(u[j][k]);
        if (i == j) t.re -= 1.0;
        v[0] += norm2(t);
      }
    cx<double> d;
    if constexpr (NC == 2) d = u[0][0] * u[1][1] - u[0][1] * u[1][0];
    else
      d = u[0][0] * (u[1][1] * u[2][2] - u[1][2] * u[2][1]) - u[0][1] * (u[1][0] * u[2][2] - u[1][2] * u[2][0]) +
          u[0][2] * (u[1][0] * u[2][1] - u[1][1] * u[2][0]);
    d.re -= 1.0;
    v[0] += norm2(d);
  }
  if (grid_sum<1>(v, partials, counter, sh) && threadIdx.x == 0) result[0] = v[0];
}

// ---------------------------------------------------------------------------
// spinor conversions
// ---------------------------------------------------------------------------
// reference layout (nrhs, ns, N, V) -> FP64 even / odd fields; g5: multiply by gamma_d
template <int ND, int NC>
__global__ void ref_to_eo_kernel(EoGeom g, int64_t V, const double2* __restrict__ ref, EoField e, EoField o, int g5) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  const int64_t lex = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  if (lex >= V) return;
  int x[ND];
  lex_coords<ND>(g, lex, x);
  int par = 0;
#pragma unroll
  for (int d = 0; d < ND; ++d) par += x[d];
  par &= 1;
  cx<double> v[NCOMP];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) {
    v[c] = ld(ref + ((int64_t)rhs * NCOMP + c) * V + lex);
    if (g5 && c >= (NS / 2) * NC) v[c] = -v[c];
  }
  store_sp<SP64, NCOMP>(par ? o : e, rhs, lex >> 1, v);
}

template <int ND, int NC>
__global__ void eo_to_ref_kernel(EoGeom g, int64_t V, EoField e, EoField o, double2* __restrict__ ref) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  const int64_t lex = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  if (lex >= V) return;
  int x[ND];
  lex_coords<ND>(g, lex, x);
  int par = 0;
#pragma unroll
  for (int d = 0; d < ND; ++d) par += x[d];
  par &= 1;
  cx<double> v[NCOMP];
  load_sp<SP64, NCOMP>(par ? o : e, rhs, lex >> 1, v);
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) st(ref + ((int64_t)rhs * NCOMP + c) * V + lex, v[c]);
}

// dst (precision SP) = src (FP64); optionally also dst2 = src
template <int SP, int NCOMP>
LYM_D void convert_body(int64_t Vh, const EoField& src, const EoField& dst, const EoField& dst2, int only_update,
                        const int* upd, int bx, int rhs) {
  const int64_t cb = bx * (int64_t)blockDim.x + threadIdx.x;
  if (cb >= Vh) return;
  if (only_update && !upd[rhs]) return;
  cx<double> v[NCOMP];
  load_sp<SP64, NCOMP>(src, rhs, cb, v);
  cx<typename Prec<SP>::real> w[NCOMP];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) w[c] = {(typename Prec<SP>::real)v[c].re, (typename Prec<SP>::real)v[c].im};
  store_sp<SP, NCOMP>(dst, rhs, cb, w);
  if (dst2.data) store_sp<SP, NCOMP>(dst2, rhs, cb, w);
}

template <int SP, int NCOMP>
__global__ void convert_kernel(int64_t Vh, EoField src, EoField dst, EoField dst2, const CGState* st, int only_update,
                               const int* upd) {
  convert_body<SP, NCOMP>(Vh, src, dst, dst2, only_update, upd, blockIdx.x, blockIdx.y);
}

// x64 += xs; xs = 0  (for rhs with upd[rhs])
template <int XP, int NCOMP>
LYM_D void accumulate_body(int64_t Vh, const EoField& xs, const EoField& x64, const int* upd, int bx, int rhs) {
  const int64_t cb = bx * (int64_t)blockDim.x + threadIdx.x;
  if (cb >= Vh || !upd[rhs]) return;
  using R = typename Prec<XP>::real;
  cx<R> a[NCOMP];
  load_sp<XP, NCOMP>(xs, rhs, cb, a);
  cx<double> b[NCOMP];
  load_sp<SP64, NCOMP>(x64, rhs, cb, b);
  cx<R> z[NCOMP];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) {
    b[c] = b[c] + cx<double>{(double)a[c].re, (double)a[c].im};
    z[c] = czero<R>();
  }
  store_sp<SP64, NCOMP>(x64, rhs, cb, b);
  store_sp<XP, NCOMP>(xs, rhs, cb, z);
}

template <int XP, int NCOMP>
__global__ void accumulate_kernel(int64_t Vh, EoField xs, EoField x64, const int* upd) {
  accumulate_body<XP, NCOMP>(Vh, xs, x64, upd, blockIdx.x, blockIdx.y);
}

template <int NCOMP>
__global__ void zero64_kernel(int64_t Vh, EoField f) {
  const int64_t cb = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cb >= Vh) return;
  cx<double> z[NCOMP];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) z[c] = czero<double>();
  store_sp<SP64, NCOMP>(f, blockIdx.y, cb, z);
}

// ---------------------------------------------------------------------------
// FP64 hop with a linear-combination epilogue (reliable updates, setup):
//   out = z0 + a1 z1 + c * G5OUT(hop(G5IN(in)))  ; optional |out|^2 -> res[rhs]
// ---------------------------------------------------------------------------
template <int ND, int NC, bool G5IN, bool G5OUT>
LYM_D void hop64_lincomb_body(const EoGeom& g, const HopGauge& hg, const EoField& in, int par, const EoField& out,
                              const EoField& z0, const EoField& z1, double a1, double c, const int* upd,
                              double* partials, unsigned* counters, double* res, int nblk, int bx, int rhs) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  __shared__ double sh[32];
  const int64_t cb = bx * (int64_t)blockDim.x + threadIdx.x;
  if (upd && !upd[rhs]) return;  // uniform per block
  double nrm[1] = {0.0};
  if (cb < g.Vh) {
    cx<double> acc[NS][NC];
    hop_site<ND, NC, SP64, SP64, false, G5IN>(g, hg, in, rhs, cb, par, acc);
    cx<double> v[NCOMP], a[NCOMP];
    if (z0.data) load_sp<SP64, NCOMP>(z0, rhs, cb, v);
    else
#pragma unroll
      for (int k = 0; k < NCOMP; ++k) v[k] = czero<double>();
    if (z1.data) {
      load_sp<SP64, NCOMP>(z1, rhs, cb, a);
#pragma unroll
      for (int k = 0; k < NCOMP; ++k) v[k] += a1 * a[k];
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) {
        cx<double> h = (G5OUT && s >= NS / 2) ? -acc[s][cc] : acc[s][cc];
        v[s * NC + cc] += c * h;
        nrm[0] += norm2(v[s * NC + cc]);
      }
    store_sp<SP64, NCOMP>(out, rhs, cb, v);
  }
  if (res) {
    if (grid_sum_n<1>(nrm, partials + (int64_t)rhs * nblk, counters + rhs, sh, bx, nblk) && threadIdx.x == 0)
      res[rhs] = nrm[0];
  }
}

template <int ND, int NC, bool G5IN, bool G5OUT>
__global__ void __launch_bounds__(128, 1) hop64_lincomb_kernel(EoGeom g, HopGauge hg, EoField in, int par, EoField out,
                                                            EoField z0, EoField z1, double a1, double c,
                                                            const int* upd, double* partials, unsigned* counters,
                                                            double* res, int nblk) {
  hop64_lincomb_body<ND, NC, G5IN, G5OUT>(g, hg, in, par, out, z0, z1, a1, c, upd, partials, counters, res, nblk,
                                          blockIdx.x, blockIdx.y);
}

// |f|^2 per rhs (FP64 field)
template <int NCOMP>
__global__ void __launch_bounds__(128) norm64_kernel(int64_t Vh, EoField f, double* partials, unsigned* counters,
                                                     double* res, int nblk, int accumulate) {
  __shared__ double sh[32];
  const int64_t cb = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  double n[1] = {0.0};
  if (cb < Vh) {
    cx<double> v[NCOMP];
    load_sp<SP64, NCOMP>(f, rhs, cb, v);
#pragma unroll
    for (int k = 0; k < NCOMP; ++k) n[0] += norm2(v[k]);
  }
  if (grid_sum<1>(n, partials + (int64_t)rhs * nblk, counters + rhs, sh) && threadIdx.x == 0)
    res[rhs] = accumulate ? res[rhs] + n[0] : n[0];
}

// ---------------------------------------------------------------------------
// sloppy CG iteration kernels (precision SP, links GP/COMP)
// ---------------------------------------------------------------------------

// Launch bounds of the hop kernels: FP64 ones declare one resident block per
// SM as enough, which lets ptxas keep every neighbour's loads in flight at once
// (about 250 registers); the memory-bound FP64 hop runs ~20% faster at 32^4
// that way.  Sloppy ones keep ptxas's default register target.
//
// The kernel bodies below take the block's site block `bx` and rhs tile `by`
// (and, for the reductions, the site-block count nblk) so that the
// multi-lattice kernels can run them for any lattice of one launch.

// s = H_oe G5IN(p) for the rhs tile by*R .. +R-1 (odd output);
// st == nullptr: every rhs (profiling hook)
template <int ND, int NC, int SP, int GP, bool COMP, bool G5IN, int R, int MX>
LYM_D void cg_hop_body(const EoGeom& g, const HopGauge& hg, const EoField& in, const EoField& out, int par,
                       const CGState* st, int bx, int by) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  const int i = bx * blockDim.x + threadIdx.x;
  const int rhs0 = by * R;
  int act[R];
  int any = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    act[r] = st ? st[rhs0 + r].active : 1;
    any |= act[r];
  }
  if (!any || i >= g.Vh) return;
  using RT = typename Prec<SP>::real;
  cx<RT> acc[R][NS][NC];
  hop_any<ND, NC, SP, GP, COMP, G5IN, R, MX>(g, hg, in, rhs0, i, par, act, acc);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (!act[r]) continue;
    cx<RT> v[NCOMP];
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int c = 0; c < NC; ++c) v[s * NC + c] = acc[r][s][c];
    store_sp<SP, NCOMP>(out, rhs0 + r, i, v);
  }
}

template <int ND, int NC, int SP, int GP, bool COMP, bool G5IN, int R, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cg_hop_kernel(EoGeom g, HopGauge hg, EoField in, EoField out, int par,
                                                     const CGState* st) {
  cg_hop_body<ND, NC, SP, GP, COMP, G5IN, R, MX>(g, hg, in, out, par, st, blockIdx.x, blockIdx.y);
}

// t = p - kappa^2 H_eo s ; alpha = rr / |t|^2   (rhs tile of R)
template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
LYM_D void cg_t_body(const EoGeom& g, const HopGauge& hg, const EoField& s, const EoField& p, const EoField& t,
                     double k2, CGState* st, double* partials, unsigned* counters, int nblk, int bx, int by) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  __shared__ double sh[R * 32];
  const int i = bx * blockDim.x + threadIdx.x;
  const int rhs0 = by * R;
  int act[R];
  int any = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    act[r] = st[rhs0 + r].active;
    any |= act[r];
  }
  if (!any) return;  // uniform per block
  using RT = typename Prec<SP>::real;
  double n[R];
#pragma unroll
  for (int r = 0; r < R; ++r) n[r] = 0.0;
  if (i < g.Vh) {
    cx<RT> acc[R][NS][NC];
    hop_any<ND, NC, SP, GP, COMP, false, R, MX>(g, hg, s, rhs0, i, 0, act, acc);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = r, cb = i;
      if (!act[r]) continue;
      cx<RT> v[NCOMP];
      load_sp<SP, NCOMP>(p, rhs0 + r, cb, v);
#pragma unroll
      for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          cx<RT>& w = v[a * NC + c];
          w -= (RT)k2 * acc[q][a][c];
          n[r] += (double)w.re * w.re + (double)w.im * w.im;
        }
      store_sp<SP, NCOMP>(t, rhs0 + r, cb, v);
    }
  }
  if (grid_sum_n<R>(n, partials + (int64_t)by * nblk * R, counters + by, sh, bx, nblk) && threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!act[r]) continue;
      CGState& S = st[rhs0 + r];
      if (n[r] > 0.0 && S.rr > 0.0) {
        S.alpha = S.rr / n[r];
      } else {
        S.alpha = 0.0;
        S.active = 0;  // p = 0: nothing left to do
      }
    }
  }
}

template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cg_t_kernel(EoGeom g, HopGauge hg, EoField s, EoField p, EoField t, double k2,
                                                   CGState* st, double* partials, unsigned* counters, int nblk) {
  cg_t_body<ND, NC, SP, GP, COMP, R, MX>(g, hg, s, p, t, k2, st, partials, counters, nblk, blockIdx.x, blockIdx.y);
}

// Ap = t - kappa^2 gamma_d H_eo s ; r -= alpha Ap ; beta = |r|^2 / rr   (rhs tile of R).
// x += alpha p runs in cg_p, which reads p anyway.
template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
LYM_D void cg_update_body(const EoGeom& g, const HopGauge& hg, const EoField& s, const EoField& t, const EoField& r,
                          double k2, CGState* st, double* partials, unsigned* counters, int nblk, int bx, int by) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  __shared__ double sh[R * 32];
  const int i = bx * blockDim.x + threadIdx.x;
  const int rhs0 = by * R;
  int act[R];
  int any = 0;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    act[q] = st[rhs0 + q].active;
    any |= act[q];
  }
  if (!any) return;  // uniform per block
  using RT = typename Prec<SP>::real;
  double n[R];
#pragma unroll
  for (int q = 0; q < R; ++q) n[q] = 0.0;
  if (i < g.Vh) {
    cx<RT> acc[R][NS][NC];
    // M^dag = gamma_d M gamma_d in 2 and 4 dimensions (gamma_d on the output below);
    // in 3 the adjoint hop itself
    hop_any<ND, NC, SP, GP, COMP, ND == 3, R, MX>(g, hg, s, rhs0, i, 0, act, acc);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int m = q, cb = i;
      if (!act[q]) continue;
      cx<RT> tv[NCOMP], rv[NCOMP];
      load_sp<SP, NCOMP>(t, rhs0 + q, cb, tv);
      load_sp<SP, NCOMP>(r, rhs0 + q, cb, rv);
      const RT a = (RT)st[rhs0 + q].alpha;
#pragma unroll
      for (int sp = 0; sp < NS; ++sp)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const int k = sp * NC + c;
          cx<RT> h = acc[m][sp][c];
          if (ND != 3 && sp >= NS / 2) h = -h;
          cx<RT> ap = tv[k] - (RT)k2 * h;
          rv[k] -= a * ap;
          n[q] += (double)rv[k].re * rv[k].re + (double)rv[k].im * rv[k].im;
        }
      store_sp<SP, NCOMP>(r, rhs0 + q, cb, rv);
    }
  }
  if (grid_sum_n<R>(n, partials + (int64_t)by * nblk * R, counters + by, sh, bx, nblk) && threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      if (!act[q]) continue;
      CGState& S = st[rhs0 + q];
      S.beta = n[q] / S.rr;
      S.rr = n[q];
      S.iters += 1;
      if (S.rr < S.pause2 || S.iters >= S.max_iter || S.iters >= S.pause_iter)
        S.active = 2;  // finish the p update, then stop
    }
  }
}

template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cg_update_kernel(EoGeom g, HopGauge hg, EoField s, EoField t,
                                                                           EoField r, double k2, CGState* st,
                                                                           double* partials, unsigned* counters,
                                                                           int nblk) {
  cg_update_body<ND, NC, SP, GP, COMP, R, MX>(g, hg, s, t, r, k2, st, partials, counters, nblk, blockIdx.x,
                                              blockIdx.y);
}

// Reliable-update residual in the sloppy precision: r = t - kappa^2 gamma_d H_eo s
// (t = q converted, s = H_oe gamma_d t), i.e. r = M^dag q, for rhs with upd[rhs];
// res[rhs] = |r|^2.
template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
LYM_D void cg_rnew_body(const EoGeom& g, const HopGauge& hg, const EoField& s, const EoField& t, const EoField& r,
                        double k2, const int* upd, double* partials, unsigned* counters, double* res, int nblk,
                        int bx, int by) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  __shared__ double sh[R * 32];
  const int i = bx * blockDim.x + threadIdx.x;
  const int rhs0 = by * R;
  int act[R];
  int any = 0;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    act[q] = upd[rhs0 + q];
    any |= act[q];
  }
  if (!any) return;  // uniform per block
  using RT = typename Prec<SP>::real;
  double n[R];
#pragma unroll
  for (int q = 0; q < R; ++q) n[q] = 0.0;
  if (i < g.Vh) {
    cx<RT> acc[R][NS][NC];
    hop_any<ND, NC, SP, GP, COMP, ND == 3, R, MX>(g, hg, s, rhs0, i, 0, act, acc);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int m = q, cb = i;
      if (!act[q]) continue;
      cx<RT> v[NCOMP];
      load_sp<SP, NCOMP>(t, rhs0 + q, cb, v);
#pragma unroll
      for (int sp = 0; sp < NS; ++sp)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          cx<RT> h = acc[m][sp][c];
          if (ND != 3 && sp >= NS / 2) h = -h;
          cx<RT>& w = v[sp * NC + c];
          w -= (RT)k2 * h;
          n[q] += (double)w.re * w.re + (double)w.im * w.im;
        }
      store_sp<SP, NCOMP>(r, rhs0 + q, cb, v);
    }
  }
  if (grid_sum_n<R>(n, partials + (int64_t)by * nblk * R, counters + by, sh, bx, nblk) && threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < R; ++q)
      if (act[q]) res[rhs0 + q] = n[q];
  }
}

template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cg_rnew_kernel(EoGeom g, HopGauge hg, EoField s, EoField t, EoField r,
                                                      double k2, const int* upd, double* partials,
                                                      unsigned* counters, double* res, int nblk) {
  cg_rnew_body<ND, NC, SP, GP, COMP, R, MX>(g, hg, s, t, r, k2, upd, partials, counters, res, nblk, blockIdx.x,
                                            blockIdx.y);
}

// dst = src (same precision) for rhs with upd[rhs]
template <int SP, int NCOMP>
__global__ void __launch_bounds__(128) copy_sp_kernel(int64_t Vh, EoField src, EoField dst, const int* upd) {
  const int64_t cb = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  if (cb >= Vh || !upd[rhs]) return;
  cx<typename Prec<SP>::real> v[NCOMP];
  load_sp<SP, NCOMP>(src, rhs, cb, v);
  store_sp<SP, NCOMP>(dst, rhs, cb, v);
}

// x += alpha p (x in the accumulator precision XP), then p = r + beta p; the
// last block of each rhs to finish then turns the "stop after the p update"
// marker (active == 2) into a pause.  Every block of the rhs read `active`
// before it counted itself, so the last one may change it.
template <int SP, int XP, int NCOMP>
LYM_D void cg_p_body(int64_t Vh, const EoField& r, const EoField& p, const EoField& x, CGState* st,
                     unsigned* counters, int bx, int rhs, int nblk) {
  const int64_t cb = bx * (int64_t)blockDim.x + threadIdx.x;
  const int act = st[rhs].active;
  if (!act) return;  // uniform per rhs
  if (cb < Vh) {
    using R = typename Prec<SP>::real;
    using XR = typename Prec<XP>::real;
    const R b = (R)st[rhs].beta;
    const XR alpha = (XR)st[rhs].alpha;
    cx<R> rv[NCOMP], pv[NCOMP];
    cx<XR> xv[NCOMP];
    load_sp<SP, NCOMP>(r, rhs, cb, rv);
    load_sp<SP, NCOMP>(p, rhs, cb, pv);
    load_sp<XP, NCOMP>(x, rhs, cb, xv);
#pragma unroll
    for (int k = 0; k < NCOMP; ++k) {
      xv[k] += alpha * cx<XR>{(XR)pv[k].re, (XR)pv[k].im};
      pv[k] = rv[k] + b * pv[k];
    }
    store_sp<XP, NCOMP>(x, rhs, cb, xv);
    store_sp<SP, NCOMP>(p, rhs, cb, pv);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counters + rhs, 1u) == (unsigned)nblk - 1) {
      if (act == 2) st[rhs].active = 0;
      counters[rhs] = 0u;  // ready for the next use of this slot
    }
  }
}

template <int SP, int XP, int NCOMP>
__global__ void __launch_bounds__(128) cg_p_kernel(int64_t Vh, EoField r, EoField p, EoField x, CGState* st,
                                                   unsigned* counters) {
  cg_p_body<SP, XP, NCOMP>(Vh, r, p, x, st, counters, blockIdx.x, blockIdx.y, gridDim.x);
}

// ---------------------------------------------------------------------------
// tensor-core FP16 hop kernels (4D SU(3), FP16 spinors, full FP16 links; the hop
// core and its layout are in lym_hop_tc.cuh).  One thread per (site, rhs), a
// CTA per (8 sites, 16 rhs); the epilogues are the one-rhs forms of the bodies
// above.
// ---------------------------------------------------------------------------
LYM_D double* tc_red(char* smem) {
  using P = tc::Plan;
  return reinterpret_cast<double*>(smem + 2 * P::kTile + P::kLinks);
}


// s = H G5IN(p) (output parity par); st == nullptr: every rhs
template <bool G5IN>
__global__ void __launch_bounds__(tc::kThreads) cg_hop_tc_kernel(EoGeom g, HopGauge hg, EoField in, EoField out, int par,
                                                        const CGState* st) {
  extern __shared__ __align__(16) char smem[];
  constexpr int S = tc::kS, RG = tc::kRG, NCOMP = 12;
  const int i = threadIdx.x % S, r = threadIdx.x / S, rhs = blockIdx.y * RG + r;
  const bool act = st ? st[rhs].active != 0 : true;
  if (!__syncthreads_or(act)) return;  // no rhs of this group active (uniform per block)
  const int cb = blockIdx.x * S + i;
  cx<float> acc[4][3];
  tc::hop_tc<G5IN>(g, hg, in, par, blockIdx.x * S, blockIdx.y * RG, i, r, act, smem, acc);
  if (!act || cb >= g.Vh) return;
  cx<float> v[NCOMP];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) v[s * 3 + c] = acc[s][c];
  store_sp<SP16, NCOMP>(out, rhs, cb, v);
}

// t = p - kappa^2 H_eo s ; alpha = rr / |t|^2
__global__ void __launch_bounds__(tc::kThreads) cg_t_tc_kernel(EoGeom g, HopGauge hg, EoField s, EoField p, EoField t,
                                                      double k2, CGState* st, double* partials,
                                                      unsigned* counters, int nblk) {
  extern __shared__ __align__(16) char smem[];
  constexpr int S = tc::kS, RG = tc::kRG, NCOMP = 12;
  const int i = threadIdx.x % S, r = threadIdx.x / S, rhs = blockIdx.y * RG + r;
  const bool act = st[rhs].active != 0;
  if (!__syncthreads_or(act)) return;  // uniform per block
  const int cb = blockIdx.x * S + i;
  cx<float> acc[4][3];
  tc::hop_tc<false>(g, hg, s, 0, blockIdx.x * S, blockIdx.y * RG, i, r, act, smem, acc);
  double n = 0.0;
  if (act && cb < g.Vh) {
    cx<float> v[NCOMP];
    load_sp<SP16, NCOMP>(p, rhs, cb, v);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cx<float>& w = v[a * 3 + c];
        w -= (float)k2 * acc[a][c];
        n += (double)w.re * w.re + (double)w.im * w.im;
      }
    store_sp<SP16, NCOMP>(t, rhs, cb, v);
  }
  double tot = 0.0;
  if (tc::grid_rhs_sum(n, tc_red(smem), partials, counters, nblk, tot) && threadIdx.x < RG) {
    CGState& Sx = st[blockIdx.y * RG + threadIdx.x];
    if (Sx.active) {
      if (tot > 0.0 && Sx.rr > 0.0) {
        Sx.alpha = Sx.rr / tot;
      } else {
        Sx.alpha = 0.0;
        Sx.active = 0;  // p = 0: nothing left to do
      }
    }
  }
}

// Ap = t - kappa^2 gamma_d H_eo s ; r -= alpha Ap ; beta = |r|^2 / rr (x += alpha p in cg_p)
__global__ void __launch_bounds__(tc::kThreads) cg_update_tc_kernel(EoGeom g, HopGauge hg, EoField s, EoField t,
                                                                   EoField r, double k2, CGState* st,
                                                                   double* partials, unsigned* counters, int nblk) {
  extern __shared__ __align__(16) char smem[];
  constexpr int S = tc::kS, RG = tc::kRG, NCOMP = 12;
  const int i = threadIdx.x % S, q = threadIdx.x / S, rhs = blockIdx.y * RG + q;
  const bool act = st[rhs].active != 0;
  if (!__syncthreads_or(act)) return;  // uniform per block
  const int cb = blockIdx.x * S + i;
  cx<float> acc[4][3];
  tc::hop_tc<false>(g, hg, s, 0, blockIdx.x * S, blockIdx.y * RG, i, q, act, smem, acc);
  double n = 0.0;
  if (act && cb < g.Vh) {
    cx<float> tv[NCOMP], rv[NCOMP];
    load_sp<SP16, NCOMP>(t, rhs, cb, tv);
    load_sp<SP16, NCOMP>(r, rhs, cb, rv);
    const float a = (float)st[rhs].alpha;
#pragma unroll
    for (int sp = 0; sp < 4; ++sp)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int k = sp * 3 + c;
        cx<float> h = acc[sp][c];
        if (sp >= 2) h = -h;
        const cx<float> ap = tv[k] - (float)k2 * h;
        rv[k] -= a * ap;
        n += (double)rv[k].re * rv[k].re + (double)rv[k].im * rv[k].im;
      }
    store_sp<SP16, NCOMP>(r, rhs, cb, rv);
  }
  double tot = 0.0;
  if (tc::grid_rhs_sum(n, tc_red(smem), partials, counters, nblk, tot) && threadIdx.x < RG) {
    CGState& Sx = st[blockIdx.y * RG + threadIdx.x];
    if (Sx.active) {
      Sx.beta = tot / Sx.rr;
      Sx.rr = tot;
      Sx.iters += 1;
      if (Sx.rr < Sx.pause2 || Sx.iters >= Sx.max_iter || Sx.iters >= Sx.pause_iter)
        Sx.active = 2;  // finish the p update, then stop
    }
  }
}

// r = t - kappa^2 gamma_d H_eo s for rhs with upd[rhs]; res[rhs] = |r|^2
__global__ void __launch_bounds__(tc::kThreads) cg_rnew_tc_kernel(EoGeom g, HopGauge hg, EoField s, EoField t, EoField r,
                                                         double k2, const int* upd, double* partials,
                                                         unsigned* counters, double* res, int nblk) {
  extern __shared__ __align__(16) char smem[];
  constexpr int S = tc::kS, RG = tc::kRG, NCOMP = 12;
  const int i = threadIdx.x % S, q = threadIdx.x / S, rhs = blockIdx.y * RG + q;
  const bool act = upd[rhs] != 0;
  if (!__syncthreads_or(act)) return;  // uniform per block
  const int cb = blockIdx.x * S + i;
  cx<float> acc[4][3];
  tc::hop_tc<false>(g, hg, s, 0, blockIdx.x * S, blockIdx.y * RG, i, q, act, smem, acc);
  double n = 0.0;
  if (act && cb < g.Vh) {
    cx<float> v[NCOMP];
    load_sp<SP16, NCOMP>(t, rhs, cb, v);
#pragma unroll
    for (int sp = 0; sp < 4; ++sp)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cx<float> h = acc[sp][c];
        if (sp >= 2) h = -h;
        cx<float>& w = v[sp * 3 + c];
        w -= (float)k2 * h;
        n += (double)w.re * w.re + (double)w.im * w.im;
      }
    store_sp<SP16, NCOMP>(r, rhs, cb, v);
  }
  double tot = 0.0;
  if (tc::grid_rhs_sum(n, tc_red(smem), partials, counters, nblk, tot) && threadIdx.x < RG) {
    const int q2 = blockIdx.y * RG + threadIdx.x;
    if (upd[q2]) res[q2] = tot;
  }
}

// ---------------------------------------------------------------------------
// per-(ND, NC, SP, COMP) operation table
// ---------------------------------------------------------------------------
struct Work;
struct CgOps {
  void (*iterate)(Work&, cudaStream_t);                 // one sloppy CG iteration (5 launches)
  void (*hop64)(Work&, int par, const EoField& in, const EoField& out, const EoField& z0, const EoField& z1,
                double a1, double c, bool g5in, bool g5out, bool with_norm, cudaStream_t);
  void (*to_eo)(Work&, const void* ref, int g5, cudaStream_t);
  void (*from_eo)(Work&, void* ref, cudaStream_t);
  void (*norm64)(Work&, const EoField& f, int accumulate, cudaStream_t);
  void (*convert)(Work&, const EoField& src, const EoField& dst, const EoField& dst2, bool only_update, cudaStream_t);
  void (*accumulate)(Work&, cudaStream_t);
  void (*zero64)(Work&, const EoField& f, cudaStream_t);
  void (*dslash)(Work&, cudaStream_t);                  // s_o = H_oe p_e, every rhs
  void (*rnew)(Work&, cudaStream_t);                    // r = M^dag t (sloppy), masked, |r|^2 -> res
  void (*copy_rp)(Work&, cudaStream_t);                 // p = r, masked (restart)
  void (*preload)();                                    // load the iteration kernels before a graph is built
};
// kernels one iterate() call launches
constexpr int kLaunchesPerIteration = 5;
// solver workspaces a gauge object keeps, keyed by (precision, capacity)
constexpr size_t kMaxWorkspaces = 6;

struct Work {
  lym_gauge* g = nullptr;
  int nrhs = 0, sp = 0, xp = 0;  // nrhs: padded count every field holds
  int nreal = 0;                 // right-hand sides the caller passes (this call)
  int dirty = 0;                 // leading source slots that may hold an earlier call's sources
  int R = 1;                     // right-hand sides per thread in the hop kernels (autotuned)
  int mx = 0;                    // FP16 hop arithmetic: 0 FP32 (hop_tile), 1 mixed (hop_tile_mx)
  bool tuned = false;
  int tuned_i = 0;
  // hop-kernel candidates: right-hand sides per thread x compressed / full links
  // (x FP32 / mixed-precision arithmetic for FP16)
  static constexpr int kMaxCand = 16;
  int ncand = 0, cur = 0;
  int rcand[kMaxCand] = {1};
  bool ccand[kMaxCand] = {};
  int mcand[kMaxCand] = {};
  CgOps ops_r[kMaxCand]{};
  int64_t Vh = 0;
  int nblk = 0;
  double kappa = 0;
  // FP64 fields
  EoField be, bo, bp, x64, xo, q, s64;
  // sloppy fields
  EoField r, p, t, s, xs;
  CGState* st = nullptr;
  CGState* st_host = nullptr;
  CGState* st_ahead = nullptr;    // pinned: the state after the chunk launched ahead (cg_solve_on)
  int* upd = nullptr;
  int* upd_host = nullptr;
  double* partials = nullptr;
  double* partials_tc = nullptr;  // per rhs and 8-site block: the tensor-core hop's reductions
  unsigned* counters = nullptr;
  double* res = nullptr;       // per rhs, several result slots
  double* res_host = nullptr;
  void* pool = nullptr;
  size_t pool_bytes = 0;
  HopGauge hg64, hgs, hgs_c, hgs_f;  // hgs: the links of the selected candidate
  CgOps ops{};
  cudaGraphExec_t graph = nullptr;
  GraphRec rec;                   // graph being recorded by build_graph (explicit kernel nodes)
  int graph_chunk = 0;
  double graph_kappa = 0;
  int graph_cand = -1;
  cudaStream_t graph_stream = nullptr;
  cudaStream_t stream = nullptr;  // solves run here (non-blocking, fenced to the caller's stream by events)
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaEvent_t ev_state[2] = {nullptr, nullptr};  // the two state copies in flight
  int64_t launches = 0;           // kernels launched by the current call (graph nodes included)
};

// Launch a kernel, or, while build_graph records, append it to the graph as a
// kernel node after the previous one (launch_rec).
template <typename... KArgs, typename... Args>
static void launch(Work& w, cudaStream_t st, void (*kernel)(KArgs...), dim3 grid, dim3 block, Args&&... args) {
  launch_rec(w.rec, st, kernel, grid, block, std::forward<Args>(args)...);
}

template <typename... KArgs, typename... Args>
static void launch_smem(Work& w, cudaStream_t st, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                        Args&&... args) {
  launch_rec_smem(w.rec, st, kernel, grid, block, smem, std::forward<Args>(args)...);
}

template <int ND, int NC, int SP, bool COMP, int R, int MX>
struct Impl {
  static constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  static constexpr int GP = SP == SP64 ? SP64 : (SP == SP32 ? SP32 : SP16);
  // the sloppy solution accumulates in FP32 for the half-precision modes (a
  // norm-scaled half accumulator loses the small late corrections and forces
  // frequent reliable updates) and in the sloppy precision otherwise
  static constexpr int XP = (SP == SP16 || SP == SPB16) ? SP32 : SP;

  static void iterate(Work& w, cudaStream_t st) {
    const double k2 = w.kappa * w.kappa;
    dim3 grid(w.nblk, w.nrhs), tile(w.nblk, w.nrhs / R);
    const CGState* cst = w.st;
    launch(w, st, cg_hop_kernel<ND, NC, SP, GP, COMP, false, R, MX>, tile, dim3(128), w.g->geom, w.hgs, w.p, w.s, 1,
           cst);
    launch(w, st, cg_t_kernel<ND, NC, SP, GP, COMP, R, MX>, tile, dim3(128), w.g->geom, w.hgs, w.s, w.p, w.t, k2,
           w.st, w.partials, w.counters, w.nblk);
    launch(w, st, cg_hop_kernel<ND, NC, SP, GP, COMP, true, R, MX>, tile, dim3(128), w.g->geom, w.hgs, w.t, w.s, 1,
           cst);
    launch(w, st, cg_update_kernel<ND, NC, SP, GP, COMP, R, MX>, tile, dim3(128), w.g->geom, w.hgs, w.s, w.t, w.r,
           k2, w.st, w.partials, w.counters, w.nblk);
    launch(w, st, cg_p_kernel<SP, XP, NCOMP>, grid, dim3(128), w.Vh, w.r, w.p, w.xs, w.st, w.counters);
  }

  static void hop64(Work& w, int par, const EoField& in, const EoField& out, const EoField& z0, const EoField& z1,
                    double a1, double c, bool g5in, bool g5out, bool with_norm, cudaStream_t st) {
    dim3 grid(w.nblk, w.nrhs);
    double* res = with_norm ? w.res : nullptr;
    w.launches += 1;
#define LYM_H64(A, B)                                                                                   \
  hop64_lincomb_kernel<ND, NC, A, B><<<grid, 128, 0, st>>>(w.g->geom, w.hg64, in, par, out, z0, z1, a1, c, \
                                                           w.upd, w.partials, w.counters, res, w.nblk)
    if (g5in && g5out) LYM_H64(true, true);
    else if (g5in) LYM_H64(true, false);
    else if (g5out) LYM_H64(false, true);
    else LYM_H64(false, false);
#undef LYM_H64
  }

  static void to_eo(Work& w, const void* ref, int g5, cudaStream_t st) {
    dim3 grid(grid_for(w.g->V, 128), w.nreal);
    w.launches += 1;
    ref_to_eo_kernel<ND, NC><<<grid, 128, 0, st>>>(w.g->geom, w.g->V, (const double2*)ref, w.be, w.bo, g5);
  }
  static void from_eo(Work& w, void* ref, cudaStream_t st) {
    dim3 grid(grid_for(w.g->V, 128), w.nreal);
    w.launches += 1;
    eo_to_ref_kernel<ND, NC><<<grid, 128, 0, st>>>(w.g->geom, w.g->V, w.x64, w.xo, (double2*)ref);
  }
  static void norm64(Work& w, const EoField& f, int accumulate, cudaStream_t st) {
    dim3 grid(w.nblk, w.nrhs);
    w.launches += 1;
    norm64_kernel<NCOMP><<<grid, 128, 0, st>>>(w.Vh, f, w.partials, w.counters, w.res, w.nblk, accumulate);
  }
  static void convert(Work& w, const EoField& src, const EoField& dst, const EoField& dst2, bool only_update,
                      cudaStream_t st) {
    dim3 grid(w.nblk, w.nrhs);
    w.launches += 1;
    convert_kernel<SP, NCOMP><<<grid, 128, 0, st>>>(w.Vh, src, dst, dst2, w.st, only_update, w.upd);
  }
  static void accumulate(Work& w, cudaStream_t st) {
    if constexpr (SP != SP64) {
      dim3 grid(w.nblk, w.nrhs);
      w.launches += 1;
      accumulate_kernel<XP, NCOMP><<<grid, 128, 0, st>>>(w.Vh, w.xs, w.x64, w.upd);
    }
  }
  static void zero64(Work& w, const EoField& f, cudaStream_t st) {
    dim3 grid(w.nblk, w.nrhs);
    w.launches += 1;
    zero64_kernel<NCOMP><<<grid, 128, 0, st>>>(w.Vh, f);
  }
  static void dslash(Work& w, cudaStream_t st) {
    dim3 tile(w.nblk, w.nrhs / R);
    w.launches += 1;
    cg_hop_kernel<ND, NC, SP, GP, COMP, false, R, MX><<<tile, 128, 0, st>>>(w.g->geom, w.hgs, w.p, w.s, 1, nullptr);
  }
  static void rnew(Work& w, cudaStream_t st) {
    const double k2 = w.kappa * w.kappa;
    dim3 tile(w.nblk, w.nrhs / R);
    w.launches += 2;
    cg_hop_kernel<ND, NC, SP, GP, COMP, true, R, MX><<<tile, 128, 0, st>>>(w.g->geom, w.hgs, w.t, w.s, 1, nullptr);
    cg_rnew_kernel<ND, NC, SP, GP, COMP, R, MX><<<tile, 128, 0, st>>>(w.g->geom, w.hgs, w.s, w.t, w.r, k2, w.upd,
                                                                      w.partials, w.counters, w.res, w.nblk);
  }
  static void copy_rp(Work& w, cudaStream_t st) {
    dim3 grid(w.nblk, w.nrhs);
    w.launches += 1;
    copy_sp_kernel<SP, NCOMP><<<grid, 128, 0, st>>>(w.Vh, w.r, w.p, w.upd);
  }
  // Loads every kernel iterate() launches (with lazily loaded modules a kernel's
  // code is loaded at its first use) before build_graph records them.
  static void preload() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, cg_hop_kernel<ND, NC, SP, GP, COMP, false, R, MX>);
    cudaFuncGetAttributes(&a, cg_hop_kernel<ND, NC, SP, GP, COMP, true, R, MX>);
    cudaFuncGetAttributes(&a, cg_t_kernel<ND, NC, SP, GP, COMP, R, MX>);
    cudaFuncGetAttributes(&a, cg_update_kernel<ND, NC, SP, GP, COMP, R, MX>);
    cudaFuncGetAttributes(&a, cg_p_kernel<SP, XP, NCOMP>);
  }

  static CgOps table() {
    return CgOps{&iterate, &hop64, &to_eo, &from_eo, &norm64, &convert, &accumulate, &zero64, &dslash, &rnew,
                 &copy_rp, &preload};
  }
};

// The tensor-core FP16 hop (4D SU(3), full FP16 links): iterate / dslash / rnew
// run the cg_*_tc kernels with 16 right-hand sides per CTA; everything else is
// the FP16 mixed-precision table's.
struct ImplTC {
  using Base = Impl<4, 3, SP16, false, 1, 1>;
  using P = tc::Plan;
  static constexpr int S = tc::kS, RG = tc::kRG;
  static unsigned nblk(const Work& w) { return (unsigned)((w.Vh + S - 1) / S); }
  // the kernels take more than 48 KB of dynamic shared memory
  static void prepare() {
    cudaFuncSetAttribute(cg_hop_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, P::kBytes);
    cudaFuncSetAttribute(cg_hop_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, P::kBytes);
    cudaFuncSetAttribute(cg_t_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P::kBytes);
    cudaFuncSetAttribute(cg_update_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P::kBytes);
    cudaFuncSetAttribute(cg_rnew_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P::kBytes);
  }
  static void iterate(Work& w, cudaStream_t st) {
    const double k2 = w.kappa * w.kappa;
    const dim3 grid(w.nblk, w.nrhs), tile(nblk(w), w.nrhs / RG);
    const int nb = (int)nblk(w);
    const CGState* cst = w.st;
    launch_smem(w, st, cg_hop_tc_kernel<false>, tile, dim3(tc::kThreads), P::kBytes, w.g->geom, w.hgs, w.p, w.s, 1, cst);
    launch_smem(w, st, cg_t_tc_kernel, tile, dim3(tc::kThreads), P::kBytes, w.g->geom, w.hgs, w.s, w.p, w.t, k2, w.st,
                w.partials_tc, w.counters, nb);
    launch_smem(w, st, cg_hop_tc_kernel<true>, tile, dim3(tc::kThreads), P::kBytes, w.g->geom, w.hgs, w.t, w.s, 1, cst);
    launch_smem(w, st, cg_update_tc_kernel, tile, dim3(tc::kThreads), P::kBytes, w.g->geom, w.hgs, w.s, w.t, w.r, k2,
                w.st, w.partials_tc, w.counters, nb);
    launch(w, st, cg_p_kernel<SP16, SP32, 12>, grid, dim3(128), w.Vh, w.r, w.p, w.xs, w.st, w.counters);
  }
  static void dslash(Work& w, cudaStream_t st) {
    prepare();
    w.launches += 1;
    cg_hop_tc_kernel<false><<<dim3(nblk(w), w.nrhs / RG), tc::kThreads, P::kBytes, st>>>(w.g->geom, w.hgs, w.p, w.s, 1,
                                                                                   nullptr);
  }
  static void rnew(Work& w, cudaStream_t st) {
    prepare();
    const double k2 = w.kappa * w.kappa;
    const dim3 tile(nblk(w), w.nrhs / RG);
    w.launches += 2;
    cg_hop_tc_kernel<true><<<tile, tc::kThreads, P::kBytes, st>>>(w.g->geom, w.hgs, w.t, w.s, 1, nullptr);
    cg_rnew_tc_kernel<<<tile, tc::kThreads, P::kBytes, st>>>(w.g->geom, w.hgs, w.s, w.t, w.r, k2, w.upd, w.partials_tc,
                                                        w.counters, w.res, (int)nblk(w));
  }
  static void preload() {
    Base::preload();
    prepare();
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, cg_hop_tc_kernel<false>);
    cudaFuncGetAttributes(&a, cg_hop_tc_kernel<true>);
    cudaFuncGetAttributes(&a, cg_t_tc_kernel);
    cudaFuncGetAttributes(&a, cg_update_tc_kernel);
  }
  static CgOps table() {
    CgOps t = Base::table();
    t.iterate = &iterate;
    t.dslash = &dslash;
    t.rnew = &rnew;
    t.preload = &preload;
    return t;
  }
};

template <int ND, int NC, int R>
static CgOps pick_sp(int sp, bool comp, int mx) {
  switch (sp) {
    case SP64: return Impl<ND, NC, SP64, false, 1, 0>::table();  // FP64 keeps one rhs per thread (registers)
    case SP32: return comp ? Impl<ND, NC, SP32, true, R, 0>::table() : Impl<ND, NC, SP32, false, R, 0>::table();
    case SP16:
      if constexpr (ND != 3) {
        if constexpr (R == 1) {
          if (mx == 3) return Impl<ND, NC, SP16, false, 1, 3>::table();
        }
        if (mx == 4) return Impl<ND, NC, SP16, false, R, 4>::table();
        if constexpr (R <= 2) {
          if (mx == 5) return Impl<ND, NC, SP16, false, R, 5>::table();
        }
        if (mx) return Impl<ND, NC, SP16, false, R, 1>::table();
      }
      return comp ? Impl<ND, NC, SP16, true, R, 0>::table() : Impl<ND, NC, SP16, false, R, 0>::table();
    default: return comp ? Impl<ND, NC, SPB16, true, R, 0>::table() : Impl<ND, NC, SPB16, false, R, 0>::table();
  }
}

template <int R>
static bool pick_ops_r(int nd, int nc, int sp, bool comp, int mx, CgOps* out) {
  if (nd == 2 && nc == 2) *out = pick_sp<2, 2, R>(sp, comp, mx);
  else if (nd == 2 && nc == 3) *out = pick_sp<2, 3, R>(sp, comp, mx);
  else if (nd == 3 && nc == 2) *out = pick_sp<3, 2, R>(sp, comp, mx);
  else if (nd == 3 && nc == 3) *out = pick_sp<3, 3, R>(sp, comp, mx);
  else if (nd == 4 && nc == 2) *out = pick_sp<4, 2, R>(sp, comp, mx);
  else if (nd == 4 && nc == 3) *out = pick_sp<4, 3, R>(sp, comp, mx);
  else return false;
  return true;
}

// mx: the mixed-precision hops (FP16 spinors, full links): 1 = f16 x f16 + f32 FMAs,
// 4 = the same with neighbour indices from coordinate arithmetic, 5 = that with the t
// neighbours by warp shuffle (1 or 2 rhs per thread), 3 = packed half FMAs within a
// direction (one rhs per thread)
static bool pick_ops(int nd, int nc, int sp, bool comp, int R, int mx, CgOps* out) {
  if (R == 4) return pick_ops_r<4>(nd, nc, sp, comp, mx, out);
  if (R == 2) return pick_ops_r<2>(nd, nc, sp, comp, mx, out);
  return pick_ops_r<1>(nd, nc, sp, comp, mx, out);
}

static size_t field_bytes(int sp, int ncomp, int64_t Vh, int nrhs) {
  const int cpu = sp == SP64 ? 1 : (sp == SP32 ? 2 : 4);
  size_t b = (size_t)units_for(ncomp, cpu) * 16 * Vh * nrhs;
  if (sp == SP16 || sp == SPB16) b += sizeof(float) * Vh * nrhs;
  return (b + 255) & ~(size_t)255;
}

static EoField carve(char*& cur, int sp, int ncomp, int64_t Vh, int nrhs) {
  EoField f;
  const int cpu = sp == SP64 ? 1 : (sp == SP32 ? 2 : 4);
  f.nunits = units_for(ncomp, cpu);
  f.Vh = Vh;
  f.data = cur;
  size_t b = (size_t)f.nunits * 16 * Vh * nrhs;
  if (sp == SP16 || sp == SPB16) {
    f.norm = reinterpret_cast<float*>(cur + b);
    b += sizeof(float) * Vh * nrhs;
  }
  cur += (b + 255) & ~(size_t)255;
  return f;
}

static void free_work(Work* w) {
  if (!w) return;
  if (w->graph) cudaGraphExecDestroy(w->graph);
  if (w->stream) cudaStreamSynchronize(w->stream);
  if (w->pool) cudaFree(w->pool);
  if (w->ev_in) cudaEventDestroy(w->ev_in);
  if (w->ev_out) cudaEventDestroy(w->ev_out);
  for (cudaEvent_t e : w->ev_state)
    if (e) cudaEventDestroy(e);
  if (w->st_ahead) cudaFreeHost(w->st_ahead);
  if (w->stream) cudaStreamDestroy(w->stream);
  if (w->st_host) cudaFreeHost(w->st_host);
  if (w->upd_host) cudaFreeHost(w->upd_host);
  if (w->res_host) cudaFreeHost(w->res_host);
  delete w;
}

// Workspace capacity for nrhs right-hand sides: FP64 exactly nrhs; the sloppy
// precisions 1, 2, or nrhs rounded up to a multiple of 4 (so the hop kernels can take
// 1, 2 or 4 rhs per thread).  Batches of 3 and 4 rhs share one workspace, and so on:
// the padding never exceeds 3 slots (they get zero sources and finish before the first
// iteration), while a server's varying batch sizes need at most six workspaces per
// precision up to 16 rhs.
static int work_capacity(int nrhs, int sp) {
  if (sp == SP64 || nrhs <= 2) return nrhs;
  return (nrhs + 3) / 4 * 4;
}

// Zero the source slots an earlier call with more right-hand sides left behind
// (slots nreal .. dirty of the even and odd source fields), on the solve's stream.
static int clear_stale_sources(Work& w, cudaStream_t st) {
  if (w.dirty > w.nreal) {
    const size_t per = (size_t)w.g->ncomp * sizeof(double2) * (size_t)w.Vh;  // one rhs of an FP64 field
    const size_t off = per * (size_t)w.nreal, len = per * (size_t)(w.dirty - w.nreal);
    LYM_CUDA(cudaMemsetAsync((char*)w.be.data + off, 0, len, st));
    LYM_CUDA(cudaMemsetAsync((char*)w.bo.data + off, 0, len, st));
  }
  w.dirty = w.nreal;
  return LYM_OK;
}

static Work* find_work(lym_gauge* g, int nrhs, int sp) {
  for (size_t i = 0; i < g->works.size(); ++i) {
    Work* w = g->works[i];
    if (w->nrhs == nrhs && w->sp == sp) {
      g->works.erase(g->works.begin() + i);  // most recently used first
      g->works.insert(g->works.begin(), w);
      return w;
    }
  }
  return nullptr;
}

static void free_all_work(lym_gauge* g) {
  for (Work* w : g->works) free_work(w);
  g->works.clear();
}

static int get_work(lym_gauge* g, int nrhs, int sp, Work** out) {
  const int cap = work_capacity(nrhs, sp);
  Work* w = find_work(g, cap, sp);
  if (w) {
    w->nreal = nrhs;
    *out = w;
    return LYM_OK;
  }
  while (g->works.size() >= kMaxWorkspaces) {
    free_work(g->works.back());
    g->works.pop_back();
  }
  w = new Work();
  w->g = g;
  w->nreal = nrhs;
  // the capacity is 1, 2 or a multiple of 4, so the hop kernels can take 1, 2 or 4
  // rhs per thread; padding rhs have zero sources and finish before the first iteration
  nrhs = cap;
  w->nrhs = nrhs;
  w->sp = sp;
  w->xp = (sp == SP16 || sp == SPB16) ? SP32 : sp;
  w->Vh = g->Vh;
  w->nblk = (int)grid_for(g->Vh, 128);
  int nc_ = 0;
  for (int comp = 0; comp < 2; ++comp) {
    if (comp && !(g->comp && sp != SP64)) continue;  // compressed links need SU(N) links and a sloppy precision
    // the t-shuffle form needs full warps and t rows aligned to them
    const int lh = g->geom.Lh;
    const bool tsh_ok = lh >= 1 && lh <= 32 && (lh & (lh - 1)) == 0 && g->Vh % 32 == 0;
    for (int mx : {0, 1, 3, 4, 5}) {
      if (mx && (sp != SP16 || comp || g->nd == 3)) continue;  // the mixed-precision hops: FP16 spinors, full links, 2 or 4 dimensions
      if (mx == 5 && !tsh_ok) continue;
      for (int R : {1, 2, 4}) {
        if (nrhs % R != 0 || (sp == SP64 && R > 1)) continue;
        if (mx == 3 && R != 1) continue;  // the packed-half hop: one rhs per thread
        if (mx == 5 && R > 2) continue;
        if (!pick_ops(g->nd, g->nc, sp, comp != 0, R, mx, &w->ops_r[nc_])) {
          delete w;
          set_error("unsupported (nd=%d, N=%d) for the even-odd solver", g->nd, g->nc);
          return LYM_ERR_UNSUPPORTED;
        }
        w->rcand[nc_] = R;
        w->ccand[nc_] = comp != 0;
        w->mcand[nc_] = mx;
        ++nc_;
      }
    }
  }
  // the tensor-core hop: 4D SU(3), FP16 spinors, full links, 16 rhs per CTA
  if (sp == SP16 && g->nd == 4 && g->nc == 3 && nrhs % tc::kRG == 0) {
    w->ops_r[nc_] = ImplTC::table();
    w->rcand[nc_] = tc::kRG;
    w->ccand[nc_] = false;
    w->mcand[nc_] = 2;
    ++nc_;
  }
  const bool has_tc = nc_ > 0 && w->mcand[nc_ - 1] == 2;
  const size_t ntc = has_tc ? (size_t)nrhs * (size_t)((g->Vh + tc::kS - 1) / tc::kS) : 0;
  w->ncand = nc_;
  w->ops = w->ops_r[0];
  w->R = w->rcand[0];
  w->mx = w->mcand[0];
  const int nc = g->ncomp;
  size_t bytes = 7 * field_bytes(SP64, nc, g->Vh, nrhs);
  bytes += 4 * field_bytes(sp, nc, g->Vh, nrhs);
  if (sp != SP64) bytes += field_bytes(w->xp, nc, g->Vh, nrhs);
  const size_t nres = 8;
  bytes += ((sizeof(CGState) * nrhs + 255) & ~(size_t)255);
  bytes += ((sizeof(int) * nrhs + 255) & ~(size_t)255);
  bytes += ((sizeof(double) * (size_t)nrhs * w->nblk + 255) & ~(size_t)255);
  bytes += ((sizeof(unsigned) * nrhs + 255) & ~(size_t)255);
  bytes += ((sizeof(double) * nrhs * nres + 255) & ~(size_t)255);
  bytes += ((sizeof(double) * ntc + 255) & ~(size_t)255);
  if (cudaMalloc(&w->pool, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete w;
    set_error("solver workspace of %zu bytes does not fit", bytes);
    return LYM_ERR_OOM;
  }
  w->pool_bytes = bytes;
  char* cur = (char*)w->pool;
  w->be = carve(cur, SP64, nc, g->Vh, nrhs);
  w->bo = carve(cur, SP64, nc, g->Vh, nrhs);
  w->bp = carve(cur, SP64, nc, g->Vh, nrhs);
  w->x64 = carve(cur, SP64, nc, g->Vh, nrhs);
  w->xo = carve(cur, SP64, nc, g->Vh, nrhs);
  w->q = carve(cur, SP64, nc, g->Vh, nrhs);
  w->s64 = carve(cur, SP64, nc, g->Vh, nrhs);
  w->r = carve(cur, sp, nc, g->Vh, nrhs);
  w->p = carve(cur, sp, nc, g->Vh, nrhs);
  w->t = carve(cur, sp, nc, g->Vh, nrhs);
  w->s = carve(cur, sp, nc, g->Vh, nrhs);
  w->xs = sp == SP64 ? w->x64 : carve(cur, w->xp, nc, g->Vh, nrhs);
  w->st = reinterpret_cast<CGState*>(cur);
  cur += (sizeof(CGState) * nrhs + 255) & ~(size_t)255;
  w->upd = reinterpret_cast<int*>(cur);
  cur += (sizeof(int) * nrhs + 255) & ~(size_t)255;
  w->partials = reinterpret_cast<double*>(cur);
  cur += (sizeof(double) * (size_t)nrhs * w->nblk + 255) & ~(size_t)255;
  w->counters = reinterpret_cast<unsigned*>(cur);
  cur += (sizeof(unsigned) * nrhs + 255) & ~(size_t)255;
  w->res = reinterpret_cast<double*>(cur);
  cur += (sizeof(double) * nrhs * nres + 255) & ~(size_t)255;
  w->partials_tc = ntc ? reinterpret_cast<double*>(cur) : nullptr;
  // zero everything: reduction counters, and the padding rhs' sources stay zero for good
  if (cudaMemset(w->pool, 0, bytes) != cudaSuccess ||
      cudaMallocHost(&w->st_host, sizeof(CGState) * nrhs) != cudaSuccess ||
      cudaMallocHost(&w->st_ahead, sizeof(CGState) * nrhs) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_state[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_state[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost(&w->upd_host, sizeof(int) * nrhs) != cudaSuccess ||
      cudaMallocHost(&w->res_host, sizeof(double) * nrhs * nres) != cudaSuccess ||
      cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    free_work(w);
    set_error("solver workspace host buffers");
    return LYM_ERR_OOM;
  }
  w->hg64 = HopGauge{g->u64, g->nc * g->nc, 1.0, 0.0};
  if (sp == SP64) {
    w->hgs_f = w->hgs_c = w->hg64;
  } else if (sp == SP32) {
    w->hgs_c = HopGauge{g->u32, g->n32, g->bcr, g->bci};
    w->hgs_f = HopGauge{g->u32f, g->n32f, 1.0, 0.0};
  } else {
    w->hgs_c = HopGauge{g->u16, g->n16, g->bcr, g->bci};
    w->hgs_f = HopGauge{g->u16f, g->n16f, 1.0, 0.0};
  }
  w->hgs = w->ccand[0] ? w->hgs_c : w->hgs_f;
  g->works.insert(g->works.begin(), w);
  *out = w;
  return LYM_OK;
}

static int fetch_res(Work& w, int n, cudaStream_t st) {
  LYM_CUDA(cudaMemcpyAsync(w.res_host, w.res, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  return LYM_OK;
}

// Reliable update for the rhs flagged in upd_host (already copied to upd):
// x += x_sloppy and the true residual q = b' - M x in FP64 (the convergence
// test); then the new recursion residual r = M^dag q in the sloppy precision
// (it only has to be accurate relative to |q|).  Leaves |q|^2 in
// res_host[0..nrhs) and |r|^2 in res_host[nrhs..2 nrhs).  t and s serve as
// temporaries: the next iteration recomputes both before reading them.
// sync = false: everything is only enqueued on st (the multi-lattice driver
// enqueues every lattice's update and synchronises once).
static int reliable_update(Work& w, cudaStream_t st, bool sync = true) {
  const double k = w.kappa, k2 = k * k;
  EoField none;
  w.ops.accumulate(w, st);
  w.ops.hop64(w, 1, w.x64, w.s64, none, none, 0.0, 1.0, false, false, false, st);
  w.ops.hop64(w, 0, w.s64, w.q, w.bp, w.x64, -1.0, k2, false, false, true, st);
  LYM_CUDA(cudaMemcpyAsync(w.res_host, w.res, sizeof(double) * w.nrhs, cudaMemcpyDeviceToHost, st));
  w.ops.convert(w, w.q, w.t, none, true, st);
  w.ops.rnew(w, st);
  LYM_CUDA(cudaMemcpyAsync(w.res_host + w.nrhs, w.res, sizeof(double) * w.nrhs, cudaMemcpyDeviceToHost, st));
  LYM_CHECK_LAUNCH();
  if (sync) LYM_CUDA(cudaStreamSynchronize(st));
  return LYM_OK;
}

static int build_graph(Work& w, int chunk, cudaStream_t st) {
  if (w.graph && w.graph_chunk == chunk && w.graph_kappa == w.kappa && w.graph_stream == st && w.graph_cand == w.cur)
    return LYM_OK;
  if (w.graph) {
    cudaGraphExecDestroy(w.graph);
    w.graph = nullptr;
  }
  w.ops.preload();
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaGraphCreate(&graph, 0);
  if (e == cudaSuccess) {
    w.rec = GraphRec{graph, nullptr, cudaSuccess};
    for (int i = 0; i < chunk; ++i) w.ops.iterate(w, st);
    e = w.rec.err;
    w.rec = GraphRec{};
  }
  if (e == cudaSuccess) {
    e = cudaGraphInstantiate(&w.graph, graph, 0);
    if (e != cudaSuccess) w.graph = nullptr;
  }
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    // a graph that could not be built leaves nothing launched; the solve runs
    // the same kernels as plain launches instead (w.graph stays null)
    cudaGetLastError();
    w.graph_chunk = chunk;
    w.graph_cand = w.cur;
    w.graph_kappa = w.kappa;
    w.graph_stream = st;
    return LYM_OK;
  }
  w.graph_chunk = chunk;
  w.graph_cand = w.cur;
  w.graph_kappa = w.kappa;
  w.graph_stream = st;
  return LYM_OK;
}

// Autotuner: time the hop kernel for every (right-hand sides per thread,
// compressed or full links, FP32 or mixed-precision FP16 arithmetic)
// candidate the workspace supports and keep the fastest (once per workspace).
// forced_rhs > 0: the largest rhs tile not above it, with compressed links
// when forced_comp and the links allow it (else full links), and the mixed-
// precision hop when forced_mx and the precision is FP16.
static void select_cand(Work& w, int i) {
  w.cur = i;
  w.ops = w.ops_r[i];
  w.R = w.rcand[i];
  w.mx = w.mcand[i];
  w.hgs = w.ccand[i] ? w.hgs_c : w.hgs_f;
}

// Process-wide tuning results keyed by lattice shape, colours, sloppy
// precision, right-hand sides and link compressibility: a workspace created
// later for the same key (another gauge object of the same shape, such as a
// solve-server worker's copy) takes the pick without timing again, and the
// mutex keeps two tuning runs from timing each other's launches.
struct TuneKey {
  int v[9];
  bool operator<(const TuneKey& o) const { return std::lexicographical_compare(v, v + 9, o.v, o.v + 9); }
};
struct TunePick {
  int R;
  bool comp;
  int mx;
};
static std::mutex g_tune_mutex;
static std::map<TuneKey, TunePick> g_tune_cache;

static TuneKey tune_key(const Work& w) {
  const EoGeom& g = w.g->geom;
  return TuneKey{{g.nd, w.g->nc, g.dims[0], g.dims[1], g.dims[2], g.dims[3], w.sp, w.nrhs, w.g->comp ? 1 : 0}};
}

static int autotune(Work& w, cudaStream_t st, int forced_rhs, int forced_comp, int forced_mx) {
  if (forced_rhs > 0) {
    bool comp = false;
    int mx = 0;
    for (int i = 0; i < w.ncand; ++i) {
      comp = comp || (forced_comp && w.ccand[i]);
      if (forced_mx && w.mcand[i] == forced_mx) mx = forced_mx;
    }
    int pick = 0;
    for (int i = 0; i < w.ncand; ++i)
      if (w.ccand[i] == comp && w.mcand[i] == mx && w.rcand[i] <= forced_rhs) pick = i;
    select_cand(w, pick);
    return LYM_OK;
  }
  if (w.tuned) {
    select_cand(w, w.tuned_i);
    return LYM_OK;
  }
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  const TuneKey key = tune_key(w);
  auto hit = g_tune_cache.find(key);
  if (hit != g_tune_cache.end()) {
    for (int i = 0; i < w.ncand; ++i) {
      if (w.rcand[i] == hit->second.R && w.ccand[i] == hit->second.comp && w.mcand[i] == hit->second.mx) {
        select_cand(w, i);
        w.tuned = true;
        w.tuned_i = i;
        return LYM_OK;
      }
    }
  }
  cudaEvent_t e0, e1;
  LYM_CUDA(cudaEventCreate(&e0));
  LYM_CUDA(cudaEventCreate(&e1));
  // five interleaved rounds, median time per candidate: robust against a
  // concurrent solve on another stream slowing a measurement down, and against
  // one lucky round deciding between candidates a few per cent apart
  constexpr int kRounds = 5;
  float times[Work::kMaxCand][kRounds];
  float tbest[Work::kMaxCand];
  // Candidates timed: the packed-half hop (mixed_fma 3) and the tensor-core hop (2) run
  // only when asked for (the first's FP16 colour sums cost iterations at tight
  // tolerances that a dslash timing does not see; the second never won a measured
  // workspace).  With FP16 spinors and a mixed-precision form available, the forms that
  // never won in the tile sweeps at 16^4 and 32^4 (FP32 arithmetic, compressed links,
  // 4 rhs per thread) are not timed either: every timed candidate costs each new
  // (geometry, precision, capacity) of a solve server a few dozen dslash launches.
  bool has_mx = false;
  for (int i = 0; i < w.ncand; ++i) has_mx = has_mx || w.mcand[i] == 1;
  auto tunable = [&](int i) {
    if (w.mcand[i] == 2 || w.mcand[i] == 3) return false;
    if (w.sp == SP16 && has_mx && (w.mcand[i] == 0 || w.rcand[i] == 4)) return false;
    return true;
  };
  for (int round = 0; round < kRounds; ++round) {
    for (int i = 0; i < w.ncand; ++i) {
      if (!tunable(i)) continue;
      select_cand(w, i);
      w.ops.dslash(w, st);
      cudaEventRecord(e0, st);
      for (int k = 0; k < 4; ++k) w.ops.dslash(w, st);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      times[i][round] = ms;
    }
  }
  for (int i = 0; i < w.ncand; ++i) {
    if (!tunable(i)) continue;
    std::sort(times[i], times[i] + kRounds);
    tbest[i] = times[i][kRounds / 2];
  }
  int bi = -1;
  for (int i = 0; i < w.ncand; ++i)
    if (tunable(i) && (bi < 0 || tbest[i] < tbest[bi])) bi = i;
  if (bi < 0) bi = 0;  // nothing timed (cannot happen: the one-rhs form of each precision is timed)
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  LYM_CHECK_LAUNCH();
  select_cand(w, bi);
  w.tuned = true;
  w.tuned_i = bi;
  g_tune_cache[key] = TunePick{w.rcand[bi], w.ccand[bi], w.mcand[bi]};
  return LYM_OK;
}

static int cg_solve_on(Work& w, lym_gauge* g, double kappa, int nrhs, const void* b, void* x,
                       const lym_solver_params* prm, lym_solver_report* rep, cudaStream_t st);

static int cg_solve(lym_gauge* g, double kappa, int nrhs, const void* b, void* x, const lym_solver_params* prm,
                    lym_solver_report* rep, cudaStream_t caller) {
  LYM_REQUIRE(g && b && x && prm && rep, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nrhs >= 1 && nrhs <= 4096, LYM_ERR_BAD_ARG, "nrhs out of range");
  LYM_REQUIRE(prm->tol > 0 && prm->max_iter > 0, LYM_ERR_BAD_ARG, "tol and max_iter must be positive");
  LYM_REQUIRE(prm->precision >= 0 && prm->precision <= 3, LYM_ERR_BAD_ARG, "bad precision");
  const int sp = prm->precision;
  LYM_REQUIRE(sp == SP64 || (g->prec_mask >> sp) & 1u, LYM_ERR_BAD_ARG,
              "precision %d was not enabled in lym_gauge_create", sp);
  LYM_REQUIRE(g->nd != 3 || !prm->hermitian, LYM_ERR_UNSUPPORTED,
              "three dimensions have no hermitian form gamma_d D (two-component spinors, no gamma_5)");
  std::lock_guard<std::recursive_mutex> own(g->mu);
  Work* wp;
  int rc = get_work(g, nrhs, sp, &wp);
  if (rc) return rc;
  Work& w = *wp;
  // order the solve after the caller's prior work, and the caller's later work after the solve
  LYM_CUDA(cudaEventRecord(w.ev_in, caller));
  LYM_CUDA(cudaStreamWaitEvent(w.stream, w.ev_in, 0));
  rc = cg_solve_on(w, g, kappa, nrhs, b, x, prm, rep, w.stream);
  cudaEventRecord(w.ev_out, w.stream);
  cudaStreamWaitEvent(caller, w.ev_out, 0);
  return rc;
}

static int cg_solve_on(Work& w, lym_gauge* g, double kappa, int nrhs, const void* b, void* x,
                       const lym_solver_params* prm, lym_solver_report* rep, cudaStream_t st) {
  int rc = LYM_OK;
  const int sp = prm->precision;
  const int nreal = nrhs;
  nrhs = w.nrhs;  // padded count from here on
  w.kappa = kappa;
  w.launches = 0;
  const double k = kappa;
  const double delta = prm->delta > 0 && prm->delta < 1 ? prm->delta : 0.1;
  const int chunk = prm->chunk > 0 ? std::min(prm->chunk, 256) : 8;
  EoField none;

  // source: b (or gamma_d b for Q x = b) in even-odd form, |b|^2, b' = b_e - kappa H_eo b_o
  rc = clear_stale_sources(w, st);
  if (rc) return rc;
  w.ops.to_eo(w, b, prm->hermitian ? 1 : 0, st);
  w.ops.norm64(w, w.be, 0, st);
  w.ops.norm64(w, w.bo, 1, st);
  LYM_CHECK_LAUNCH();
  rc = fetch_res(w, nrhs, st);
  if (rc) return rc;
  std::vector<double> bnorm2(w.res_host, w.res_host + nrhs);
  for (int i = 0; i < nrhs; ++i) w.upd_host[i] = 1;
  LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
  w.ops.hop64(w, 0, w.bo, w.bp, w.be, none, 0.0, -k, false, false, false, st);
  w.ops.zero64(w, w.x64, st);
  if (sp != SP64) LYM_CUDA(cudaMemsetAsync(w.xs.data, 0, field_bytes(w.xp, g->ncomp, w.Vh, nrhs), st));
  LYM_CHECK_LAUNCH();

  std::vector<int> done(nrhs, 0), updates(nrhs, 0), restart(nrhs, 0);
  std::vector<double> target(nrhs, 0.0), tres(nrhs, 0.0), prev_q2(nrhs, 0.0);
  // sloppy runs get a reliable update at least this often, whatever the residual does
  const int max_interval = sp == SP64 ? (1 << 30) : 50;
  auto plan_rhs = [&](int i, double q2, double r2) -> void {
    CGState& S = w.st_host[i];
    const double want = prm->tol * prm->tol * bnorm2[i];
    tres[i] = bnorm2[i] > 0 ? std::sqrt(q2 / bnorm2[i]) : 0.0;
    // the true residual stalled since the last update: the sloppy recursion
    // drifted, so restart the search direction from the true residual
    restart[i] = (prev_q2[i] > 0.0 && q2 > 0.25 * prev_q2[i]) ? 1 : 0;
    prev_q2[i] = q2;
    if (q2 <= want || r2 == 0.0) {
      done[i] = 1;
      S.active = 0;
      return;
    }
    // pause target for the recursive residual of the normal equations:
    // scale the present one by how far the true residual still has to fall
    const double est = r2 * (want / q2) * 0.25;
    target[i] = est;
    S.rr = r2;
    S.pause2 = sp == SP64 ? est : std::max(est, delta * delta * r2);
    S.pause_iter = S.iters + max_interval;
    S.active = S.iters >= S.max_iter ? 0 : 1;
  };
  for (int i = 0; i < nrhs; ++i) {
    CGState& S = w.st_host[i];
    std::memset(&S, 0, sizeof(S));
    S.max_iter = prm->max_iter;
  }
  // initial residual (x = 0): q = b', r = M^dag b'
  rc = reliable_update(w, st);
  if (rc) return rc;
  for (int i = 0; i < nrhs; ++i) plan_rhs(i, w.res_host[i], w.res_host[nrhs + i]);
  LYM_CUDA(cudaMemcpyAsync(w.st, w.st_host, sizeof(CGState) * nrhs, cudaMemcpyHostToDevice, st));
  w.ops.copy_rp(w, st);  // p = r (upd is all ones here)
  LYM_CHECK_LAUNCH();
  rc = autotune(w, st, prm->rhs_per_thread, prm->compressed_links, prm->mixed_fma);
  if (rc) return rc;
  rc = build_graph(w, chunk, st);
  if (rc) return rc;

  while (true) {
    bool any_active = false;
    for (int i = 0; i < nrhs; ++i) any_active = any_active || (!done[i] && w.st_host[i].active);
    if (!any_active) break;
    // run chunks until every rhs paused, finished or hit max_iter.  One chunk
    // is always in flight ahead of the state the host looks at, so the device
    // keeps iterating while the host thread wakes up; a chunk launched after
    // every rhs paused does nothing (its blocks find no active rhs and return,
    // the state stays as it was).
    auto launch_chunk = [&](CGState* to, cudaEvent_t ev) -> int {
      if (w.graph) {
        LYM_CUDA(cudaGraphLaunch(w.graph, st));
      } else {
        for (int i = 0; i < chunk; ++i) w.ops.iterate(w, st);
        LYM_CHECK_LAUNCH();
      }
      w.launches += (int64_t)chunk * kLaunchesPerIteration;
      LYM_CUDA(cudaMemcpyAsync(to, w.st, sizeof(CGState) * nrhs, cudaMemcpyDeviceToHost, st));
      LYM_CUDA(cudaEventRecord(ev, st));
      return LYM_OK;
    };
    CGState* bufs[2] = {w.st_host, w.st_ahead};
    int cur = 0;
    rc = launch_chunk(bufs[0], w.ev_state[0]);
    if (rc) return rc;
    while (true) {
      rc = launch_chunk(bufs[1 - cur], w.ev_state[1 - cur]);  // ahead
      if (rc) return rc;
      LYM_CUDA(cudaEventSynchronize(w.ev_state[cur]));
      bool running = false;
      for (int i = 0; i < nrhs; ++i) running = running || bufs[cur][i].active;
      if (!running) {
        LYM_CUDA(cudaEventSynchronize(w.ev_state[1 - cur]));  // the chunk ahead: no change
        break;
      }
      cur = 1 - cur;
    }
    if (bufs[cur] != w.st_host) std::memcpy(w.st_host, bufs[cur], sizeof(CGState) * nrhs);
    // reliable update for every rhs that paused and is not done
    bool any = false;
    for (int i = 0; i < nrhs; ++i) {
      w.upd_host[i] = (!done[i]) ? 1 : 0;
      any = any || w.upd_host[i];
    }
    if (!any) break;
    LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
    rc = reliable_update(w, st);
    if (rc) return rc;
    std::vector<double> q2(w.res_host, w.res_host + nrhs), r2(w.res_host + nrhs, w.res_host + 2 * nrhs);
    for (int i = 0; i < nrhs; ++i) {
      if (!w.upd_host[i]) continue;
      updates[i] += 1;
      plan_rhs(i, q2[i], r2[i]);
    }
    LYM_CUDA(cudaMemcpyAsync(w.st, w.st_host, sizeof(CGState) * nrhs, cudaMemcpyHostToDevice, st));
    // p is kept across an update, except where the true residual stalled
    bool any_restart = false;
    for (int i = 0; i < nrhs; ++i) {
      w.upd_host[i] = (!done[i] && restart[i]) ? 1 : 0;
      any_restart = any_restart || w.upd_host[i];
    }
    if (any_restart) {
      LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
      w.ops.copy_rp(w, st);
    }
    LYM_CHECK_LAUNCH();
    bool left = false;
    for (int i = 0; i < nrhs; ++i) left = left || (!done[i] && w.st_host[i].iters < prm->max_iter);
    if (!left) break;
  }
  // x_o = b_o - kappa H_oe x_e, back to the reference layout
  for (int i = 0; i < nrhs; ++i) w.upd_host[i] = 1;
  LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
  w.ops.hop64(w, 1, w.x64, w.xo, w.bo, none, 0.0, -k, false, false, false, st);
  w.ops.from_eo(w, x, st);
  LYM_CHECK_LAUNCH();
  LYM_CUDA(cudaStreamSynchronize(st));
  int status = LYM_OK;
  for (int i = 0; i < nreal; ++i) {
    rep[i].status = done[i] ? LYM_OK : LYM_ERR_NOT_CONVERGED;
    rep[i].iterations = w.st_host[i].iters;
    rep[i].reliable_updates = updates[i];
    rep[i].true_residual = tres[i];
    rep[i].kernel_launches = w.launches;
    rep[i].rhs_per_thread = w.R;
    rep[i].compressed_links = w.ccand[w.cur] ? 1 : 0;
    rep[i].mixed_fma = w.mx;
    if (!done[i]) status = LYM_ERR_NOT_CONVERGED;
  }
  return status;
}

// ---------------------------------------------------------------------------
// Several lattices in the same launches (lym_wilson_solve_multi)
//
// Independent lattices of the same (nd, N) -- each with its own geometry,
// kappa, links and right-hand sides -- run their sloppy CG iterations in the
// same five launches per iteration: every lattice owns a contiguous range of
// blocks (its site blocks x its right-hand sides) of one grid, a block finds
// its lattice by binary search over the range starts and runs the same kernel
// body as the single-lattice launch.  Setup, FP64 reliable updates and the
// odd-site reconstruction stay per lattice (they are rare).  One rhs per
// thread; FP32 takes the 12-real links when every lattice's links are SU(N),
// FP16 the mixed-precision hop with full links.
// ---------------------------------------------------------------------------
struct CgLat {
  EoGeom g;
  HopGauge hg, hg64;
  EoField p, s, t, r, xs;
  EoField x64, s64, q, bp;  // FP64 fields of the reliable update
  CGState* st;
  const int* upd;
  double* res;
  double* partials;
  unsigned* counters;
  int64_t Vh;
  int nblk, nrhs;
  double k2;
  int b0;  // first block of this lattice: its blocks are b0 + rhs * nblk + site block
};

LYM_D int cg_lat_of(const CgLat* __restrict__ lats, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (lats[mid].b0 <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int ND, int NC, int SP, int GP, bool COMP, bool G5IN, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cgm_hop_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, by = local / D.nblk, bx = local - by * D.nblk;
  cg_hop_body<ND, NC, SP, GP, COMP, G5IN, 1, MX>(D.g, D.hg, G5IN ? D.t : D.p, D.s, 1, D.st, bx, by);
}

template <int ND, int NC, int SP, int GP, bool COMP, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cgm_t_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, by = local / D.nblk, bx = local - by * D.nblk;
  cg_t_body<ND, NC, SP, GP, COMP, 1, MX>(D.g, D.hg, D.s, D.p, D.t, D.k2, D.st, D.partials, D.counters, D.nblk, bx,
                                         by);
}

template <int ND, int NC, int SP, int GP, bool COMP, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cgm_update_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, by = local / D.nblk, bx = local - by * D.nblk;
  cg_update_body<ND, NC, SP, GP, COMP, 1, MX>(D.g, D.hg, D.s, D.t, D.r, D.k2, D.st, D.partials, D.counters, D.nblk,
                                              bx, by);
}

template <int SP, int XP, int NCOMP>
__global__ void __launch_bounds__(128) cgm_p_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, rhs = local / D.nblk, bx = local - rhs * D.nblk;
  cg_p_body<SP, XP, NCOMP>(D.Vh, D.r, D.p, D.xs, D.st, D.counters, bx, rhs, D.nblk);
}

// The FP64 reliable update of every lattice (the rhs with upd set), as
// reliable_update does for one: x64 += x_sloppy; s64 = H_oe x64;
// q = b' - M x64 with |q|^2 -> res; t = q (sloppy); s = H_oe gamma_d t;
// r = M^dag q with |r|^2 -> res.
template <int XP, int NCOMP>
__global__ void __launch_bounds__(128) cgm_accumulate_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, rhs = local / D.nblk, bx = local - rhs * D.nblk;
  accumulate_body<XP, NCOMP>(D.Vh, D.xs, D.x64, D.upd, bx, rhs);
}

template <int ND, int NC>
__global__ void __launch_bounds__(128, 1) cgm_hx64_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, rhs = local / D.nblk, bx = local - rhs * D.nblk;
  const EoField none;
  hop64_lincomb_body<ND, NC, false, false>(D.g, D.hg64, D.x64, 1, D.s64, none, none, 0.0, 1.0, D.upd, nullptr,
                                           nullptr, nullptr, D.nblk, bx, rhs);
}

template <int ND, int NC>
__global__ void __launch_bounds__(128, 1) cgm_q64_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, rhs = local / D.nblk, bx = local - rhs * D.nblk;
  hop64_lincomb_body<ND, NC, false, false>(D.g, D.hg64, D.s64, 0, D.q, D.bp, D.x64, -1.0, D.k2, D.upd, D.partials,
                                           D.counters, D.res, D.nblk, bx, rhs);
}

template <int SP, int NCOMP>
__global__ void __launch_bounds__(128) cgm_convert_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, rhs = local / D.nblk, bx = local - rhs * D.nblk;
  const EoField none;
  convert_body<SP, NCOMP>(D.Vh, D.q, D.t, none, 1, D.upd, bx, rhs);
}

template <int ND, int NC, int SP, int GP, bool COMP, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cgm_hopt_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, by = local / D.nblk, bx = local - by * D.nblk;
  cg_hop_body<ND, NC, SP, GP, COMP, true, 1, MX>(D.g, D.hg, D.t, D.s, 1, nullptr, bx, by);
}

template <int ND, int NC, int SP, int GP, bool COMP, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0) cgm_rnew_kernel(const CgLat* __restrict__ lats, int n) {
  const CgLat& D = lats[cg_lat_of(lats, n, blockIdx.x)];
  const int local = blockIdx.x - D.b0, by = local / D.nblk, bx = local - by * D.nblk;
  cg_rnew_body<ND, NC, SP, GP, COMP, 1, MX>(D.g, D.hg, D.s, D.t, D.r, D.k2, D.upd, D.partials, D.counters, D.res,
                                            D.nblk, bx, by);
}

struct MultiOps {
  void (*iterate)(GraphRec&, cudaStream_t, const CgLat*, int n, int blocks);  // one iteration, 5 launches
  void (*q_part)(cudaStream_t, const CgLat*, int n, int blocks);  // reliable update up to |q|^2
  void (*r_part)(cudaStream_t, const CgLat*, int n, int blocks);  // the rest: r = M^dag q, |r|^2
  void (*preload)();
};
constexpr int kMultiUpdateLaunches = 6;

template <int ND, int NC, int SP, bool COMP, int MX>
struct MultiImpl {
  static constexpr int NCOMP = Gamma<ND>::NS * NC;
  static constexpr int GP = SP == SP64 ? SP64 : (SP == SP32 ? SP32 : SP16);
  static constexpr int XP = (SP == SP16 || SP == SPB16) ? SP32 : SP;
  static void iterate(GraphRec& rec, cudaStream_t st, const CgLat* lats, int n, int blocks) {
    const dim3 grid(blocks), blk(128);
    launch_rec(rec, st, cgm_hop_kernel<ND, NC, SP, GP, COMP, false, MX>, grid, blk, lats, n);
    launch_rec(rec, st, cgm_t_kernel<ND, NC, SP, GP, COMP, MX>, grid, blk, lats, n);
    launch_rec(rec, st, cgm_hop_kernel<ND, NC, SP, GP, COMP, true, MX>, grid, blk, lats, n);
    launch_rec(rec, st, cgm_update_kernel<ND, NC, SP, GP, COMP, MX>, grid, blk, lats, n);
    launch_rec(rec, st, cgm_p_kernel<SP, XP, NCOMP>, grid, blk, lats, n);
  }
  static void q_part(cudaStream_t st, const CgLat* lats, int n, int blocks) {
    if constexpr (SP != SP64) cgm_accumulate_kernel<XP, NCOMP><<<blocks, 128, 0, st>>>(lats, n);
    cgm_hx64_kernel<ND, NC><<<blocks, 128, 0, st>>>(lats, n);
    cgm_q64_kernel<ND, NC><<<blocks, 128, 0, st>>>(lats, n);
  }
  static void r_part(cudaStream_t st, const CgLat* lats, int n, int blocks) {
    cgm_convert_kernel<SP, NCOMP><<<blocks, 128, 0, st>>>(lats, n);
    cgm_hopt_kernel<ND, NC, SP, GP, COMP, MX><<<blocks, 128, 0, st>>>(lats, n);
    cgm_rnew_kernel<ND, NC, SP, GP, COMP, MX><<<blocks, 128, 0, st>>>(lats, n);
  }
  static void preload() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, cgm_hop_kernel<ND, NC, SP, GP, COMP, false, MX>);
    cudaFuncGetAttributes(&a, cgm_t_kernel<ND, NC, SP, GP, COMP, MX>);
    cudaFuncGetAttributes(&a, cgm_hop_kernel<ND, NC, SP, GP, COMP, true, MX>);
    cudaFuncGetAttributes(&a, cgm_update_kernel<ND, NC, SP, GP, COMP, MX>);
    cudaFuncGetAttributes(&a, cgm_p_kernel<SP, XP, NCOMP>);
  }
  static MultiOps table() { return MultiOps{&iterate, &q_part, &r_part, &preload}; }
};

template <int ND, int NC>
static MultiOps multi_pick_sp(int sp, bool comp) {
  switch (sp) {
    case SP64: return MultiImpl<ND, NC, SP64, false, 0>::table();
    case SP32: return comp ? MultiImpl<ND, NC, SP32, true, 0>::table() : MultiImpl<ND, NC, SP32, false, 0>::table();
    case SP16:
      if constexpr (ND == 3) return MultiImpl<ND, NC, SP16, false, 0>::table();
      else return MultiImpl<ND, NC, SP16, false, 1>::table();
    default: return MultiImpl<ND, NC, SPB16, false, 0>::table();
  }
}

static bool multi_pick(int nd, int nc, int sp, bool comp, MultiOps* out) {
  if (nd == 2 && nc == 2) *out = multi_pick_sp<2, 2>(sp, comp);
  else if (nd == 2 && nc == 3) *out = multi_pick_sp<2, 3>(sp, comp);
  else if (nd == 3 && nc == 2) *out = multi_pick_sp<3, 2>(sp, comp);
  else if (nd == 3 && nc == 3) *out = multi_pick_sp<3, 3>(sp, comp);
  else if (nd == 4 && nc == 2) *out = multi_pick_sp<4, 2>(sp, comp);
  else if (nd == 4 && nc == 3) *out = multi_pick_sp<4, 3>(sp, comp);
  else return false;
  return true;
}

// Per-lattice CG bookkeeping of the multi-lattice driver (the same decisions
// as cg_solve_on's, for one workspace).
struct MultiLat {
  Work* w = nullptr;
  int nreal = 0;
  double tol = 0;  // target true relative residual of this lattice
  std::vector<double> bnorm2, tres, prev_q2;
  std::vector<int> done, updates, restart;
};

static void multi_plan(MultiLat& L, const lym_solver_params* prm, double delta, int i, double q2, double r2) {
  Work& w = *L.w;
  CGState& S = w.st_host[i];
  const int sp = w.sp;
  const double want = L.tol * L.tol * L.bnorm2[i];
  L.tres[i] = L.bnorm2[i] > 0 ? std::sqrt(q2 / L.bnorm2[i]) : 0.0;
  L.restart[i] = (L.prev_q2[i] > 0.0 && q2 > 0.25 * L.prev_q2[i]) ? 1 : 0;
  L.prev_q2[i] = q2;
  if (q2 <= want || r2 == 0.0) {
    L.done[i] = 1;
    S.active = 0;
    return;
  }
  const double est = r2 * (want / q2) * 0.25;
  S.rr = r2;
  S.pause2 = sp == SP64 ? est : std::max(est, delta * delta * r2);
  S.pause_iter = S.iters + (sp == SP64 ? (1 << 30) : 50);
  S.active = S.iters >= S.max_iter ? 0 : 1;
}

static int cg_solve_multi(int nlat, lym_gauge* const* gs, const double* kappas, const double* tols,
                          const int* nrhs, const void* const* bs, void* const* xs, const lym_solver_params* prm,
                          lym_solver_report* rep, cudaStream_t caller) {
  const int sp = prm->precision;
  LYM_REQUIRE(gs[0], LYM_ERR_BAD_ARG, "null argument (lattice 0)");
  const int nd = gs[0]->nd, nc = gs[0]->nc;
  LYM_REQUIRE(nd != 3 || !prm->hermitian, LYM_ERR_UNSUPPORTED,
              "three dimensions have no hermitian form gamma_d D (two-component spinors, no gamma_5)");
  bool comp_all = sp == SP32;
  for (int l = 0; l < nlat; ++l) {
    LYM_REQUIRE(gs[l] && bs[l] && xs[l], LYM_ERR_BAD_ARG, "null argument (lattice %d)", l);
    LYM_REQUIRE(gs[l]->nd == nd && gs[l]->nc == nc, LYM_ERR_BAD_ARG, "every lattice needs the same nd and N");
    LYM_REQUIRE(nrhs[l] >= 1 && nrhs[l] <= 4096, LYM_ERR_BAD_ARG, "nrhs out of range (lattice %d)", l);
    LYM_REQUIRE(sp == SP64 || (gs[l]->prec_mask >> sp) & 1u, LYM_ERR_BAD_ARG,
                "precision %d was not enabled in lym_gauge_create (lattice %d)", sp, l);
    for (int k = 0; k < l; ++k)
      LYM_REQUIRE(gs[k] != gs[l], LYM_ERR_BAD_ARG, "a gauge object appears twice (lattices %d and %d)", k, l);
    LYM_REQUIRE(!tols || tols[l] > 0, LYM_ERR_BAD_ARG, "tolerance must be positive (lattice %d)", l);
    comp_all = comp_all && gs[l]->comp;
  }
  // take every gauge object's lock in address order (no two callers can wait on each other)
  std::vector<lym_gauge*> order(gs, gs + nlat);
  std::sort(order.begin(), order.end());
  std::vector<std::unique_lock<std::recursive_mutex>> own;
  own.reserve(nlat);
  for (lym_gauge* g : order) own.emplace_back(g->mu);
  const int mx = (sp == SP16 && nd != 3) ? 1 : 0;
  MultiOps ops;
  LYM_REQUIRE(multi_pick(nd, nc, sp, comp_all, &ops), LYM_ERR_UNSUPPORTED, "unsupported (nd=%d, N=%d)", nd, nc);
  std::vector<MultiLat> lats(nlat);
  for (int l = 0; l < nlat; ++l) {
    int rc = get_work(gs[l], nrhs[l], sp, &lats[l].w);
    if (rc) return rc;
    Work& w = *lats[l].w;
    int pick = -1;
    for (int i = 0; i < w.ncand; ++i)
      if (w.rcand[i] == 1 && w.ccand[i] == comp_all && w.mcand[i] == mx) pick = i;
    LYM_REQUIRE(pick >= 0, LYM_ERR_UNSUPPORTED, "no one-rhs hop tile for lattice %d", l);
    select_cand(w, pick);
  }
  cudaStream_t st = lats[0].w->stream;
  LYM_CUDA(cudaEventRecord(lats[0].w->ev_in, caller));
  LYM_CUDA(cudaStreamWaitEvent(st, lats[0].w->ev_in, 0));
  struct Fence {
    cudaEvent_t ev;
    cudaStream_t from, to;
    ~Fence() {
      cudaEventRecord(ev, from);
      cudaStreamWaitEvent(to, ev, 0);
    }
  } fence{lats[0].w->ev_out, st, caller};
  const double delta = prm->delta > 0 && prm->delta < 1 ? prm->delta : 0.1;
  const int chunk = prm->chunk > 0 ? std::min(prm->chunk, 256) : 8;
  EoField none;
  // lattice descriptors (device copy for the multi-lattice kernels)
  std::vector<CgLat> desc(nlat);
  int blocks = 0;
  for (int l = 0; l < nlat; ++l) {
    Work& w = *lats[l].w;
    CgLat& D = desc[l];
    D.g = gs[l]->geom;
    D.hg = w.hgs;
    D.hg64 = w.hg64;
    D.p = w.p;
    D.s = w.s;
    D.t = w.t;
    D.r = w.r;
    D.xs = w.xs;
    D.x64 = w.x64;
    D.s64 = w.s64;
    D.q = w.q;
    D.bp = w.bp;
    D.st = w.st;
    D.upd = w.upd;
    D.res = w.res;
    D.partials = w.partials;
    D.counters = w.counters;
    D.Vh = w.Vh;
    D.nblk = w.nblk;
    D.nrhs = w.nrhs;
    D.k2 = kappas[l] * kappas[l];
    D.b0 = blocks;
    LYM_REQUIRE((int64_t)blocks + (int64_t)w.nblk * w.nrhs < (int64_t(1) << 31), LYM_ERR_UNSUPPORTED,
                "too many blocks for one launch");
    blocks += w.nblk * w.nrhs;
  }
  CgLat* d_desc = nullptr;
  LYM_CUDA(cudaMallocAsync(&d_desc, sizeof(CgLat) * nlat, st));
  struct Release {
    CgLat* p;
    cudaStream_t st;
    cudaGraphExec_t exec = nullptr;
    ~Release() {
      if (exec) cudaGraphExecDestroy(exec);
      cudaFreeAsync(p, st);
    }
  } release{d_desc, st};
  LYM_CUDA(cudaMemcpyAsync(d_desc, desc.data(), sizeof(CgLat) * nlat, cudaMemcpyHostToDevice, st));
  int64_t launches = 0;
  // FP64 reliable update of every lattice's rhs with upd set, in launches over all
  // lattices; |q|^2 lands in res_host[0..n), |r|^2 in res_host[n..2n)
  auto fused_update = [&]() -> int {
    ops.q_part(st, d_desc, nlat, blocks);
    LYM_CHECK_LAUNCH();
    for (auto& L : lats)
      LYM_CUDA(cudaMemcpyAsync(L.w->res_host, L.w->res, sizeof(double) * L.w->nrhs, cudaMemcpyDeviceToHost, st));
    ops.r_part(st, d_desc, nlat, blocks);
    LYM_CHECK_LAUNCH();
    for (auto& L : lats)
      LYM_CUDA(cudaMemcpyAsync(L.w->res_host + L.w->nrhs, L.w->res, sizeof(double) * L.w->nrhs,
                               cudaMemcpyDeviceToHost, st));
    LYM_CUDA(cudaStreamSynchronize(st));
    launches += kMultiUpdateLaunches;
    return LYM_OK;
  };
  // per-lattice setup, as cg_solve_on: source, |b|^2, b', x = 0; then the first
  // residual of every lattice at once, and p = r
  for (int l = 0; l < nlat; ++l) {
    MultiLat& L = lats[l];
    Work& w = *L.w;
    const int n = w.nrhs;
    L.nreal = nrhs[l];
    L.tol = tols ? tols[l] : prm->tol;
    w.kappa = kappas[l];
    w.launches = 0;
    const double k = kappas[l];
    int rz = clear_stale_sources(w, st);
    if (rz) return rz;
    w.ops.to_eo(w, bs[l], prm->hermitian ? 1 : 0, st);
    w.ops.norm64(w, w.be, 0, st);
    w.ops.norm64(w, w.bo, 1, st);
    LYM_CHECK_LAUNCH();
    // |b|^2 to res_host[4n..5n) (the reliable update fills [0..2n))
    LYM_CUDA(cudaMemcpyAsync(w.res_host + 4 * n, w.res, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    for (int i = 0; i < n; ++i) w.upd_host[i] = 1;
    LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    w.ops.hop64(w, 0, w.bo, w.bp, w.be, none, 0.0, -k, false, false, false, st);
    w.ops.zero64(w, w.x64, st);
    if (sp != SP64) LYM_CUDA(cudaMemsetAsync(w.xs.data, 0, field_bytes(w.xp, gs[l]->ncomp, w.Vh, n), st));
    LYM_CHECK_LAUNCH();
  }
  int rc = fused_update();
  if (rc) return rc;
  for (int l = 0; l < nlat; ++l) {
    MultiLat& L = lats[l];
    Work& w = *L.w;
    const int n = w.nrhs;
    L.bnorm2.assign(w.res_host + 4 * n, w.res_host + 5 * n);
    L.tres.assign(n, 0.0);
    L.prev_q2.assign(n, 0.0);
    L.done.assign(n, 0);
    L.updates.assign(n, 0);
    L.restart.assign(n, 0);
    for (int i = 0; i < n; ++i) {
      std::memset(&w.st_host[i], 0, sizeof(CGState));
      w.st_host[i].max_iter = prm->max_iter;
      multi_plan(L, prm, delta, i, w.res_host[i], w.res_host[n + i]);
    }
    LYM_CUDA(cudaMemcpyAsync(w.st, w.st_host, sizeof(CGState) * n, cudaMemcpyHostToDevice, st));
    w.ops.copy_rp(w, st);
    LYM_CHECK_LAUNCH();
  }
  // the graph of `chunk` iterations over all lattices
  ops.preload();
  {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess) {
      GraphRec rec{graph, nullptr, cudaSuccess};
      for (int i = 0; i < chunk; ++i) ops.iterate(rec, st, d_desc, nlat, blocks);
      e = rec.err;
    }
    if (e == cudaSuccess && cudaGraphInstantiate(&release.exec, graph, 0) != cudaSuccess) release.exec = nullptr;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();  // without a graph the iterations run as plain launches
  }
  auto active_any = [&]() {
    for (auto& L : lats)
      for (int i = 0; i < L.w->nrhs; ++i)
        if (!L.done[i] && L.w->st_host[i].active) return true;
    return false;
  };
  // chunks until every rhs of every lattice paused, finished or hit max_iter; the host
  // reads the state after each chunk.  (A chunk launched ahead of that read, as the
  // single-lattice solve does, measured 11-20 % slower here: the chunk launched after
  // the last pause runs as empty launches over every lattice of the class, which costs
  // more than the wait it hides.)
  while (active_any()) {
    while (true) {
      if (release.exec) {
        LYM_CUDA(cudaGraphLaunch(release.exec, st));
      } else {
        GraphRec direct;
        for (int i = 0; i < chunk; ++i) ops.iterate(direct, st, d_desc, nlat, blocks);
        LYM_CHECK_LAUNCH();
      }
      launches += (int64_t)chunk * kLaunchesPerIteration;
      for (auto& L : lats)
        LYM_CUDA(cudaMemcpyAsync(L.w->st_host, L.w->st, sizeof(CGState) * L.w->nrhs, cudaMemcpyDeviceToHost, st));
      LYM_CUDA(cudaStreamSynchronize(st));
      bool running = false;
      for (auto& L : lats)
        for (int i = 0; i < L.w->nrhs; ++i) running = running || L.w->st_host[i].active;
      if (!running) break;
    }
    // reliable updates of every rhs that paused and is not done, all lattices in
    // the same launches, one host wait
    std::vector<int> updated(nlat, 0);
    bool any_update = false;
    for (int l = 0; l < nlat; ++l) {
      MultiLat& L = lats[l];
      Work& w = *L.w;
      const int n = w.nrhs;
      for (int i = 0; i < n; ++i) {
        w.upd_host[i] = !L.done[i] ? 1 : 0;  // as cg_solve_on: capped rhs get their last update too
        updated[l] = updated[l] || w.upd_host[i];
      }
      any_update = any_update || updated[l];
      LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    }
    if (!any_update) break;
    rc = fused_update();
    if (rc) return rc;
    for (int l = 0; l < nlat; ++l) {
      if (!updated[l]) continue;
      MultiLat& L = lats[l];
      Work& w = *L.w;
      const int n = w.nrhs;
      for (int i = 0; i < n; ++i) {
        if (!w.upd_host[i]) continue;
        L.updates[i] += 1;
        multi_plan(L, prm, delta, i, w.res_host[i], w.res_host[n + i]);
      }
      LYM_CUDA(cudaMemcpyAsync(w.st, w.st_host, sizeof(CGState) * n, cudaMemcpyHostToDevice, st));
      bool any_restart = false;
      for (int i = 0; i < n; ++i) {
        w.upd_host[i] = (!L.done[i] && L.restart[i]) ? 1 : 0;
        any_restart = any_restart || w.upd_host[i];
      }
      if (any_restart) {
        LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * n, cudaMemcpyHostToDevice, st));
        w.ops.copy_rp(w, st);
      }
      LYM_CHECK_LAUNCH();
    }
  }
  // x_o = b_o - kappa H_oe x_e and the reference layout, lattice by lattice
  int status = LYM_OK;
  int64_t total_launches = launches;
  for (int l = 0; l < nlat; ++l) {
    Work& w = *lats[l].w;
    for (int i = 0; i < w.nrhs; ++i) w.upd_host[i] = 1;
    LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_host, sizeof(int) * w.nrhs, cudaMemcpyHostToDevice, st));
    w.ops.hop64(w, 1, w.x64, w.xo, w.bo, none, 0.0, -kappas[l], false, false, false, st);
    w.ops.from_eo(w, xs[l], st);
    LYM_CHECK_LAUNCH();
    total_launches += w.launches;
  }
  LYM_CUDA(cudaStreamSynchronize(st));
  int k = 0;
  for (int l = 0; l < nlat; ++l) {
    MultiLat& L = lats[l];
    Work& w = *L.w;
    for (int i = 0; i < L.nreal; ++i, ++k) {
      rep[k].status = L.done[i] ? LYM_OK : LYM_ERR_NOT_CONVERGED;
      rep[k].iterations = w.st_host[i].iters;
      rep[k].reliable_updates = L.updates[i];
      rep[k].true_residual = L.tres[i];
      rep[k].kernel_launches = total_launches;
      rep[k].rhs_per_thread = 1;
      rep[k].compressed_links = comp_all ? 1 : 0;
      rep[k].mixed_fma = mx;
      if (!L.done[i]) status = LYM_ERR_NOT_CONVERGED;
    }
  }
  return status;
}

static int dslash_eo(lym_gauge* g, int precision, int nrhs, int repeats, cudaStream_t st) {
  LYM_REQUIRE(g && repeats >= 0, LYM_ERR_BAD_ARG, "bad argument");
  std::lock_guard<std::recursive_mutex> own(g->mu);
  Work* w = find_work(g, nrhs, precision);
  LYM_REQUIRE(w, LYM_ERR_BAD_ARG,
              "no solver workspace for precision %d and %d right-hand sides", precision, nrhs);
  for (int i = 0; i < repeats; ++i) w->ops.dslash(*w, st);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int gauge_view(const lym_gauge* g, GaugeView* v) {
  LYM_REQUIRE(g && v, LYM_ERR_BAD_ARG, "null argument");
  v->lat = g->lat;
  v->nc = g->nc;
  v->ncomp = g->ncomp;
  v->V = g->V;
  v->bcr = g->bcr;
  v->bci = g->bci;
  v->uref = g->uref;
  return LYM_OK;
}

}  // namespace lym

using namespace lym;

// ---------------------------------------------------------------------------
// gauge object
// ---------------------------------------------------------------------------
static int pack_gauge(lym_gauge* g, const void* gauge, cudaStream_t st) {
  const int64_t V = g->V;
  // what the solver workspaces (and their CUDA graphs) point at
  const void* held[5] = {g->u32, g->u16, g->u32f, g->u16f, g->nbr};
  const bool held_comp = g->comp;
  LYM_CUDA(cudaMemcpyAsync(g->uref, gauge, sizeof(double2) * g->nd * g->nc * g->nc * V, cudaMemcpyDeviceToDevice, st));
  // decide on link compression for the sloppy copies: links must be SU(N)
  Scratch* s;
  int rc = scratch_get(&s);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(host_reduce_mutex());
    const int slot = 1;
    const int64_t nl = (int64_t)g->nd * V;
    unsigned nb = reduction_blocks(nl, 256);
    double* part = s->partials + (size_t)slot * Scratch::kMaxBlocks * Scratch::kMaxVals;
    double* res = s->results + slot * Scratch::kMaxVals;
    if (g->nc == 2)
      unitarity_kernel<2><<<nb, 256, 0, st>>>(nl, (const double2*)gauge, V, part, s->counters + slot, res);
    else
      unitarity_kernel<3><<<nb, 256, 0, st>>>(nl, (const double2*)gauge, V, part, s->counters + slot, res);
    LYM_CHECK_LAUNCH();
    LYM_CUDA(cudaMemcpyAsync(s->host + slot * Scratch::kMaxVals, res, sizeof(double), cudaMemcpyDeviceToHost, st));
    LYM_CUDA(cudaStreamSynchronize(st));
    const double dev = s->host[slot * Scratch::kMaxVals] / (double)nl;
    g->comp = dev < 1e-16;  // every link SU(N) to about 1e-8
  }
  const int nc = g->nc;
  const bool want32 = (g->prec_mask >> LYM_PREC_F32) & 1u;
  const bool want16 = ((g->prec_mask >> LYM_PREC_F16) & 1u) || ((g->prec_mask >> LYM_PREC_BF16) & 1u);
  const int nxc = (nc - 1) * nc, nxf = nc * nc;
  auto ensure = [&](void** p, size_t bytes, bool want) -> int {
    if (!want) {
      if (*p) cudaFree(*p);
      *p = nullptr;
      return LYM_OK;
    }
    if (*p) return LYM_OK;  // sizes depend only on the lattice and N, fixed for this object
    if (cudaMalloc(p, bytes) != cudaSuccess) {
      cudaGetLastError();
      set_error("sloppy links do not fit");
      return LYM_ERR_OOM;
    }
    return LYM_OK;
  };
  g->n32 = units_for(nxc, 2);
  g->n16 = units_for(nxc, 2);
  g->n32f = units_for(nxf, 2);
  g->n16f = units_for(nxf, 2);
  const size_t per = (size_t)2 * g->nd * g->Vh;
  if ((rc = ensure((void**)&g->u32, sizeof(float4) * g->n32 * per, want32 && g->comp)) ||
      (rc = ensure((void**)&g->u16, sizeof(uint2) * g->n16 * per, want16 && g->comp)) ||
      (rc = ensure((void**)&g->u32f, sizeof(float4) * g->n32f * per, want32)) ||
      (rc = ensure((void**)&g->u16f, sizeof(uint2) * g->n16f * per, want16)))
    return rc;
  if (!g->nbr) {
    if (cudaMalloc(&g->nbr, sizeof(int) * 2 * g->nd * 2 * g->Vh) != cudaSuccess) {
      cudaGetLastError();
      set_error("neighbour table does not fit");
      return LYM_ERR_OOM;
    }
    g->geom.nbr = g->nbr;
    dim3 tg(grid_for(g->Vh, 128), 2);
    if (g->nd == 2) build_nbr_kernel<2><<<tg, 128, 0, st>>>(g->geom, g->nbr);
    else if (g->nd == 3) build_nbr_kernel<3><<<tg, 128, 0, st>>>(g->geom, g->nbr);
    else build_nbr_kernel<4><<<tg, 128, 0, st>>>(g->geom, g->nbr);
    LYM_CHECK_LAUNCH();
  }
  dim3 grid(grid_for(V, 128), g->nd);
#define LYM_PACK(ND_, NC_)                                                                                        \
  pack_gauge_kernel<ND_, NC_><<<grid, 128, 0, st>>>(g->geom, V, (const double2*)gauge, g->bcr, g->bci, g->u64, \
                                                    g->u32, g->n32, 1, g->u16, g->n16, 1, g->u32f, g->n32f,     \
                                                    g->u16f, g->n16f)
  if (g->nd == 2 && nc == 2) LYM_PACK(2, 2);
  else if (g->nd == 2 && nc == 3) LYM_PACK(2, 3);
  else if (g->nd == 3 && nc == 2) LYM_PACK(3, 2);
  else if (g->nd == 3 && nc == 3) LYM_PACK(3, 3);
  else if (g->nd == 4 && nc == 2) LYM_PACK(4, 2);
  else LYM_PACK(4, 3);
#undef LYM_PACK
  LYM_CHECK_LAUNCH();
  // The links were rewritten in place.  Workspaces stay valid unless a sloppy
  // copy moved or the compression changed (their hop-kernel choices and graphs
  // hold those pointers); keeping them spares an HMC step the workspace setup.
  const void* now[5] = {g->u32, g->u16, g->u32f, g->u16f, g->nbr};
  if (g->comp != held_comp || std::memcmp(held, now, sizeof(held)) != 0) {
    free_all_work(g);
    free_ms_works(g);
  }
  return LYM_OK;
}

extern "C" {

int lym_gauge_create(const lym_lattice* lat, int nc, const void* gauge, double bc_re, double bc_im,
                     unsigned prec_mask, void* stream, lym_gauge** out) {
  LYM_REQUIRE(lat && gauge && out, LYM_ERR_BAD_ARG, "null argument");
  if (lat->nd < 2 || lat->nd > 4) {
    set_error("Number of dimensions %d not supported for fermions!", lat->nd);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N=%d not supported (2 or 3)", nc);
  LYM_REQUIRE(lat->even, LYM_ERR_UNSUPPORTED, "even-odd ordering needs every extent even");
  const int ns = lat->nd == 4 ? 4 : 2;  // two-component spinors in 2 and 3 dimensions
  // the hop kernels index one rhs of a field with 32-bit offsets
  LYM_REQUIRE((int64_t)ns * nc * (lat->V / 2) < (int64_t(1) << 31), LYM_ERR_UNSUPPORTED,
              "lattice too large for 32-bit field offsets");
  lym_gauge* g = new lym_gauge();
  g->lat = lat;
  g->nc = nc;
  g->nd = lat->nd;
  g->ns = ns;
  g->ncomp = g->ns * nc;
  g->V = lat->V;
  g->Vh = lat->V / 2;
  g->bcr = bc_re;
  g->bci = bc_im;
  g->prec_mask = prec_mask;
  g->geom = make_geom(lat);
  const size_t nlink = (size_t)g->nd * nc * nc * g->V;
  if (cudaMalloc(&g->uref, sizeof(double2) * nlink) != cudaSuccess ||
      cudaMalloc(&g->u64, sizeof(double2) * nlink) != cudaSuccess) {
    cudaGetLastError();
    if (g->uref) cudaFree(g->uref);
    delete g;
    set_error("gauge copies do not fit");
    return LYM_ERR_OOM;
  }
  int rc = pack_gauge(g, gauge, (cudaStream_t)stream);
  if (rc) {
    lym_gauge_destroy(g);
    return rc;
  }
  *out = g;
  return LYM_OK;
}

int lym_gauge_update(lym_gauge* g, const void* gauge, void* stream) {
  LYM_REQUIRE(g && gauge, LYM_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::recursive_mutex> own(g->mu);
  return pack_gauge(g, gauge, (cudaStream_t)stream);
}

int lym_gauge_destroy(lym_gauge* g) {
  if (!g) return LYM_OK;
  cudaDeviceSynchronize();
  free_all_work(g);
  free_ms_works(g);
  if (g->uref) cudaFree(g->uref);
  if (g->u64) cudaFree(g->u64);
  if (g->u32) cudaFree(g->u32);
  if (g->u16) cudaFree(g->u16);
  if (g->u32f) cudaFree(g->u32f);
  if (g->u16f) cudaFree(g->u16f);
  if (g->nbr) cudaFree(g->nbr);
  delete g;
  return LYM_OK;
}

int lym_wilson_solve(lym_gauge* g, double kappa, int nrhs, const void* b, void* x, const lym_solver_params* params,
                     lym_solver_report* reports, void* stream) {
  return cg_solve(g, kappa, nrhs, b, x, params, reports, (cudaStream_t)stream);
}

int lym_wilson_solve_multi(int nlat, lym_gauge* const* gauges, const double* kappas, const double* tols,
                           const int* nrhs, const void* const* b, void* const* x, const lym_solver_params* params,
                           lym_solver_report* reports, void* stream) {
  LYM_REQUIRE(nlat >= 1 && nlat <= 1024, LYM_ERR_BAD_ARG, "nlat out of range");
  LYM_REQUIRE(gauges && kappas && nrhs && b && x && params && reports, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(params->tol > 0 && params->max_iter > 0, LYM_ERR_BAD_ARG, "tol and max_iter must be positive");
  LYM_REQUIRE(params->precision >= 0 && params->precision <= 3, LYM_ERR_BAD_ARG, "bad precision");
  return cg_solve_multi(nlat, gauges, kappas, tols, nrhs, b, x, params, reports, (cudaStream_t)stream);
}

int lym_dslash_eo(lym_gauge* g, int precision, int nrhs, int repeats, void* stream) {
  return dslash_eo(g, precision, nrhs, repeats, (cudaStream_t)stream);
}

}  // extern "C"
