// Even-odd multishift CG with reduced-precision inner iterations.
//
// Solves the full-lattice shifted systems
//   (Q^2 + sigma_k) x_{i,k} = b_i,   Q = gamma_d D,  D = 1 + kappa H,
// for nrhs right-hand sides b_i and nshift shifts sigma_k >= 0 -- the systems
// the reference's multishift_solver (dirac_solver.py:19-53) solves by MMMR in
// complex128 for RationalApproximation (dirac.py:40-73) -- with the vectors in
// the solvers' even-odd layout and the inner iterations in FP64, FP32 or
// norm-scaled FP16 / BF16 (builder-defined; the reference has one precision).
//
// A full-lattice field is a stack of even halves followed by the odd halves
// (slot k of a field with n slots per parity: k even, n + k odd).  One Q^2
// application is four even-odd hops: w = D p (w_par = p_par + kappa H p_other)
// and Q^2 p = gamma_d D gamma_d w = w + kappa gamma_d H gamma_d w.
//
// Phase 1 -- one multishift CG per right-hand side ("group"), all groups in
// the same launches (Jegerlehner's recurrences, hep-lat/9612014).  The base
// system is the smallest shift sigma_0 (the slowest to converge); only its
// direction p_0 goes through the operator.  Per iteration three kernels:
//   ms_dp : w = D p_0 ; |w|^2, |p_0|^2 -> alpha = rr / (|w|^2 + sigma_0 |p_0|^2)
//   ms_ap : r' = r - alpha (Q^2 + sigma_0) p_0 ; |r'|^2 -> beta; the last
//           block runs the FP64 zeta / alpha_k / beta_k recurrences of every shift
//   ms_p0 : x_0 += alpha p_0 ; p_0 = r' + beta p_0 (x_0 must use the p_0 the
//           operator saw, rounded to the inner precision)
// and every kMsBlock iterations
//   ms_xpm: for each shifted system k > 0, the kMsBlock pending steps
//           x_k += alpha_k p_k ; p_k = zeta_k r' + beta_k p_k
//           with x_k and p_k in registers: each shift's two vectors are read
//           and written once per kMsBlock iterations instead of every
//           iteration (the residuals r' of those iterations sit in a ring of
//           kMsBlock fields, the coefficients in per-shift rings), the same
//           arithmetic in the same order.
// All scalars stay on the device; iterations run in CUDA graphs of `chunk`
// iterations (a multiple of kMsBlock, ending with ms_xpm).  A group pauses
// itself when its sloppy residual fell by delta; the host then does an FP64
// reliable update: x64_k += x_k for every shift,
// r = b - (Q^2 + sigma_0) x64_0 in FP64 (the true base residual), which
// replaces the sloppy r; the directions and zetas carry on.  A group ends
// when its true base residual is below tol |b|.
//
// FP64 head: with a reduced inner precision the shifted systems cannot see
// the reliable updates (their residuals are only known as zeta_k r), so the
// rounding of the early iterations, while |r| is still of order |b|, stays in
// their solutions.  The iterations therefore run in FP64 until the base true
// residual is below a switch point (params->switch_residual, by default 1e-4
// for FP32, 1e-6 for FP16, 1e-7 for BF16), then the state (directions, zetas,
// recurrences) moves to the inner precision and the solve carries on.
//
// Verification: the FP64 true residual of every (i, k).  Phase 2 -- every
// (i, k) still above tol |b_i| (the shifted solutions drift with the inner
// precision) runs a CG of its own on (Q^2 + sigma_k) from x_ik, again with
// FP64 reliable updates, all such pairs in the same launches (groups of one
// shift, the same kernels).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "lym_eo.cuh"
#include "lym_gauge_obj.cuh"
#include "lym_internal.cuh"

namespace lym {

constexpr int kMsMaxShifts = 32;
constexpr int kMsBlock = 8;  // iterations per blocked shift update (ms_xpm)

// LYM_MS_TRACE=1 in the environment prints every reliable-update decision and
// the per-shift verification to stderr.
static bool ms_trace() {
  static const bool on = [] {
    const char* v = std::getenv("LYM_MS_TRACE");
    return v && *v && *v != '0';
  }();
  return on;
}

struct MsGroup {
  double rr;          // |r|^2 of the sloppy base residual
  double alpha;       // this iteration's base alpha
  double alpha_prev;  // the previous iteration's alpha and beta (zeta recurrence)
  double beta_prev;
  double pause2;      // pause when rr < pause2
  double sigma;       // base shift
  int active;         // 1 iterate; 2 stop after this iteration's x / p update; 0 paused or done
  int iters;
  int max_iter;
  int pause_iter;     // pause at this iteration count at the latest (bounds the sloppy drift)
  int nstep;          // iterations whose shift updates ms_xpm has not applied yet
};

struct MsShift {
  double sigma;
  double z, zprev;    // zeta of this and the previous iteration
  double stop2;       // the shift stops once zeta^2 rr < stop2
  // step k (ring index k mod kMsBlock): x += a p ; p = zn r_{k+1} + b p, if run
  double a[kMsBlock], b[kMsBlock], zn[kMsBlock];
  int run[kMsBlock];
  int active;         // still iterating
};

// View of a field from slot `slot` on (every precision uses 16-byte units).
LYM_HD EoField sub(const EoField& f, int64_t slot) {
  EoField v = f;
  v.data = static_cast<char*>(f.data) + slot * f.nunits * f.Vh * 16;
  v.norm = f.norm ? f.norm + slot * f.Vh : nullptr;
  return v;
}

LYM_D int eo_block_parity(int nblk) { return blockIdx.x >= (unsigned)nblk ? 1 : 0; }

// ---------------------------------------------------------------------------
// sloppy iteration kernels; grids (2 nblk, G / R): blocks [0, nblk) even sites,
// [nblk, 2 nblk) odd sites, R groups per thread sharing each link
// ---------------------------------------------------------------------------

// w = p + kappa H p (p = the base direction); |w|^2 and |p|^2 -> alpha
template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0)
    ms_dp_kernel(EoGeom g, HopGauge hg, EoField pb, EoField w, int G, double kappa, MsGroup* grp,
                 double* partials, unsigned* counters, int nblk) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  using RT = typename Prec<SP>::real;
  __shared__ double sh[2 * R * 32];
  const int par = eo_block_parity(nblk);
  const int i = (blockIdx.x - par * nblk) * blockDim.x + threadIdx.x;
  const int g0 = blockIdx.y * R;
  int act[R];
  int any = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    act[r] = grp[g0 + r].active;
    any |= act[r];
  }
  if (!any) return;  // uniform per block
  double n[2 * R];
#pragma unroll
  for (int k = 0; k < 2 * R; ++k) n[k] = 0.0;
  if (i < g.Vh) {
    cx<RT> acc[R][NS][NC];
    hop_any<ND, NC, SP, GP, COMP, false, R, MX>(g, hg, sub(pb, (1 - par) * G), g0, i, par, act, acc);
    const EoField pin = sub(pb, par * G), wout = sub(w, par * G);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!act[r]) continue;
      cx<RT> v[NCOMP];
      load_sp<SP, NCOMP>(pin, g0 + r, i, v);
#pragma unroll
      for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          cx<RT>& u = v[a * NC + c];
          n[2 * r + 1] += (double)u.re * u.re + (double)u.im * u.im;
          u += (RT)kappa * acc[r][a][c];
          n[2 * r] += (double)u.re * u.re + (double)u.im * u.im;
        }
      store_sp<SP, NCOMP>(wout, g0 + r, i, v);
    }
  }
  if (grid_sum<2 * R>(n, partials + (int64_t)blockIdx.y * gridDim.x * 2 * R, counters + blockIdx.y, sh) &&
      threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!act[r]) continue;
      MsGroup& M = grp[g0 + r];
      // <p, (Q^2 + sigma) p> = |D p|^2 + sigma |p|^2
      const double den = n[2 * r] + M.sigma * n[2 * r + 1];
      if (den > 0.0 && M.rr > 0.0) {
        M.alpha = M.rr / den;
      } else {
        M.alpha = 0.0;
        M.active = 0;  // p = 0: nothing left to do
      }
    }
  }
}

// r -= alpha (w + kappa gamma_d H gamma_d w + sigma_0 p); |r|^2 -> beta; the
// last block then advances every shift's recurrences (one thread per shift)
template <int ND, int NC, int SP, int GP, bool COMP, int R, int MX>
__global__ void __launch_bounds__(128, SP == SP64 ? 1 : 0)
    ms_ap_kernel(EoGeom g, HopGauge hg, EoField w, EoField pb, EoField ring, int G, int S, double kappa,
                 MsGroup* grp, MsShift* shf, double* partials, unsigned* counters, int nblk) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  using RT = typename Prec<SP>::real;
  __shared__ double sh[R * 32];
  __shared__ double s_al[R], s_ap[R], s_bp[R], s_sg[R], s_rr[R], s_be[R];
  __shared__ int s_ix[R];
  const int par = eo_block_parity(nblk);
  const int i = (blockIdx.x - par * nblk) * blockDim.x + threadIdx.x;
  const int g0 = blockIdx.y * R;
  int act[R];
  int any = 0;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    act[q] = grp[g0 + q].active;
    any |= act[q];
  }
  if (!any) return;  // uniform per block
  double n[R];
#pragma unroll
  for (int q = 0; q < R; ++q) n[q] = 0.0;
  if (i < g.Vh) {
    cx<RT> acc[R][NS][NC];
    hop_any<ND, NC, SP, GP, COMP, true, R, MX>(g, hg, sub(w, (1 - par) * G), g0, i, par, act, acc);
    const EoField wv = sub(w, par * G), pv = sub(pb, par * G);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      if (!act[q]) continue;
      const RT al = (RT)grp[g0 + q].alpha, sg = (RT)grp[g0 + q].sigma, k = (RT)kappa;
      // r_it lives in ring slot it mod kMsBlock; r_{it+1} goes to the next one
      const int it = grp[g0 + q].iters;
      const EoField rin = sub(ring, (int64_t)(it % kMsBlock) * 2 * G + par * G);
      const EoField rout = sub(ring, (int64_t)((it + 1) % kMsBlock) * 2 * G + par * G);
      cx<RT> x[NCOMP], p[NCOMP], y[NCOMP];
      load_sp<SP, NCOMP>(wv, g0 + q, i, x);
      load_sp<SP, NCOMP>(pv, g0 + q, i, p);
      load_sp<SP, NCOMP>(rin, g0 + q, i, y);
#pragma unroll
      for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const int m = a * NC + c;
          cx<RT> h = acc[q][a][c];
          if (a >= NS / 2) h = -h;
          const cx<RT> ap = x[m] + k * h + sg * p[m];
          y[m] -= al * ap;
          n[q] += (double)y[m].re * y[m].re + (double)y[m].im * y[m].im;
        }
      store_sp<SP, NCOMP>(rout, g0 + q, i, y);
    }
  }
  if (!grid_sum<R>(n, partials + (int64_t)blockIdx.y * gridDim.x * R, counters + blockIdx.y, sh)) return;
  // the last block of this group tile (uniform): recurrences
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      if (!act[q]) continue;
      const MsGroup& M = grp[g0 + q];
      s_rr[q] = n[q];
      s_be[q] = M.rr > 0.0 ? n[q] / M.rr : 0.0;
      s_al[q] = M.alpha;
      s_ap[q] = M.alpha_prev;
      s_bp[q] = M.beta_prev;
      s_sg[q] = M.sigma;
      s_ix[q] = M.iters % kMsBlock;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < R * S; t += blockDim.x) {
    const int q = t / S, s = t - q * S;
    if (!act[q]) continue;
    MsShift& T = shf[(int64_t)(g0 + q) * S + s];
    const int ix = s_ix[q];
    T.run[ix] = T.active;
    if (!T.active) continue;
    const double al = s_al[q], be = s_be[q];
    double zn = 1.0;
    if (s == 0) {  // the base system
      T.a[ix] = al;
      T.b[ix] = be;
    } else {
      const double den = al * s_bp[q] * (T.zprev - T.z) + T.zprev * s_ap[q] * (1.0 + (T.sigma - s_sg[q]) * al);
      zn = den != 0.0 ? T.z * T.zprev * s_ap[q] / den : 0.0;
      const double ratio = T.z != 0.0 ? zn / T.z : 0.0;
      T.a[ix] = al * ratio;
      T.b[ix] = be * ratio * ratio;
      if (zn * zn * s_rr[q] < T.stop2 || zn == 0.0) T.active = 0;  // after this update
    }
    T.zn[ix] = zn;
    T.zprev = T.z;
    T.z = zn;
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      if (!act[q]) continue;
      MsGroup& M = grp[g0 + q];
      M.alpha_prev = M.alpha;
      M.beta_prev = s_be[q];
      M.rr = s_rr[q];
      M.iters += 1;
      M.nstep += 1;
      if (M.rr < M.pause2 || M.iters >= M.max_iter || M.iters >= M.pause_iter) M.active = 2;
    }
  }
}

// The base system: x_0 += alpha p_0 ; p_0 = r_{it} + beta p_0 (r_{it}: the
// residual ms_ap just wrote; x_0 is shift slot 0 of xs); grid (2 nblk, G).
// The last block of a group turns "stop after this iteration" (active == 2)
// into a pause.
template <int SP, int XP, int NCOMP>
__global__ void __launch_bounds__(128) ms_p0_kernel(int64_t Vh, int nblk, int G, int S, EoField ring, EoField pb,
                                                    EoField xs, MsGroup* grp, unsigned* counters) {
  using RT = typename Prec<SP>::real;
  using XR = typename Prec<XP>::real;
  const int par = eo_block_parity(nblk);
  const int64_t cb = (blockIdx.x - par * nblk) * (int64_t)blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  const int act = grp[gi].active;
  if (!act) return;  // uniform per group
  if (cb < Vh) {
    const RT be = (RT)grp[gi].beta_prev;
    const XR al = (XR)grp[gi].alpha;
    const EoField rv = sub(ring, (int64_t)(grp[gi].iters % kMsBlock) * 2 * G + par * G);
    const int xslot = par * G * S + gi * S;
    cx<RT> r[NCOMP], p[NCOMP];
    cx<XR> x[NCOMP];
    load_sp<SP, NCOMP>(rv, gi, cb, r);
    load_sp<SP, NCOMP>(pb, par * G + gi, cb, p);
    load_sp<XP, NCOMP>(xs, xslot, cb, x);
#pragma unroll
    for (int k = 0; k < NCOMP; ++k) {
      x[k] += al * cx<XR>{(XR)p[k].re, (XR)p[k].im};
      p[k] = r[k] + be * p[k];
    }
    store_sp<SP, NCOMP>(pb, par * G + gi, cb, p);
    store_sp<XP, NCOMP>(xs, xslot, cb, x);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counters + gi, 1u) == gridDim.x - 1) {
      if (act == 2) grp[gi].active = 0;
      counters[gi] = 0u;  // ready for the next use of this slot
    }
  }
}

// The pending updates of each group's shifted systems k > 0 (steps
// it - nstep .. it - 1):
// x_k += a p_k ; p_k = zn r + b p_k per step, p_k and x_k held in registers
// (ps / xs: every shift's direction and sloppy solution at the last block
// boundary, slot gi * S + k per parity); grid (2 nblk, G).  The last block of
// a group clears its pending count.
template <int SP, int XP, int NCOMP>
__global__ void __launch_bounds__(128) ms_xpm_kernel(int64_t Vh, int nblk, int G, int S, EoField ring, EoField ps,
                                                     EoField xs, MsGroup* grp, const MsShift* shf,
                                                     unsigned* counters) {
  using RT = typename Prec<SP>::real;
  using XR = typename Prec<XP>::real;
  const int par = eo_block_parity(nblk);
  const int64_t cb = (blockIdx.x - par * nblk) * (int64_t)blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  const int n = grp[gi].nstep;
  if (n == 0) return;  // uniform per group
  const int k0 = grp[gi].iters - n;
  if (cb < Vh) {
    for (int s = 1; s < S; ++s) {
      const MsShift& T = shf[(int64_t)gi * S + s];
      if (!T.run[k0 % kMsBlock]) continue;
      const int slot = par * G * S + gi * S + s;
      cx<RT> pv[NCOMP];
      cx<XR> xv[NCOMP];
      load_sp<SP, NCOMP>(ps, slot, cb, pv);
      load_sp<XP, NCOMP>(xs, slot, cb, xv);
      for (int j = 0; j < n; ++j) {
        const int ix = (k0 + j) % kMsBlock;
        if (!T.run[ix]) break;  // the shift stopped after its previous step
        const XR a = (XR)T.a[ix];
        const RT zn = (RT)T.zn[ix], b = (RT)T.b[ix];
        cx<RT> rv[NCOMP];
        load_sp<SP, NCOMP>(sub(ring, (int64_t)((k0 + j + 1) % kMsBlock) * 2 * G + par * G), gi, cb, rv);
#pragma unroll
        for (int k = 0; k < NCOMP; ++k) {
          xv[k] += a * cx<XR>{(XR)pv[k].re, (XR)pv[k].im};
          pv[k] = zn * rv[k] + b * pv[k];
        }
      }
      store_sp<SP, NCOMP>(ps, slot, cb, pv);
      store_sp<XP, NCOMP>(xs, slot, cb, xv);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counters + gi, 1u) == gridDim.x - 1) {
      grp[gi].nstep = 0;
      counters[gi] = 0u;  // ready for the next use of this slot
    }
  }
}

// ms_xpm for the precisions without a per-site norm (FP64, FP32; x in the
// same precision): each thread takes one site and UPT of its NU 16-byte units
// (NG = NU / UPT threads per site, consecutive sites in a block, so every load
// stays coalesced), which leaves room to hold the pending ring residuals in
// registers for all shifts.  The coefficients are real, so the update is
// component-wise.  Grid (2 nblk NG, G).
LYM_D void ms_axpy(double2& x, double a, const double2& p) {
  x.x += a * p.x;
  x.y += a * p.y;
}
LYM_D void ms_axpy(float4& x, float a, const float4& p) {
  x.x += a * p.x;
  x.y += a * p.y;
  x.z += a * p.z;
  x.w += a * p.w;
}
LYM_D void ms_lincomb(double2& p, double zn, const double2& r, double b) {
  p.x = zn * r.x + b * p.x;
  p.y = zn * r.y + b * p.y;
}
LYM_D void ms_lincomb(float4& p, float zn, const float4& r, float b) {
  p.x = zn * r.x + b * p.x;
  p.y = zn * r.y + b * p.y;
  p.z = zn * r.z + b * p.z;
  p.w = zn * r.w + b * p.w;
}

template <int SP, int NU, int NG>
__global__ void __launch_bounds__(128) ms_xpm_split_kernel(int64_t Vh, int nblk, int G, int S, EoField ring,
                                                           EoField ps, EoField xs, MsGroup* grp, const MsShift* shf,
                                                           unsigned* counters) {
  static_assert(SP == SP64 || SP == SP32, "no per-site norm");
  static_assert(NU % NG == 0, "units split evenly");
  using U = typename Prec<SP>::unit;
  using RT = typename Prec<SP>::real;
  constexpr int UPT = NU / NG;
  const int part = blockIdx.x % NG;
  const int rest = blockIdx.x / NG;
  const int par = rest >= nblk ? 1 : 0;
  const int64_t cb = (rest - par * nblk) * (int64_t)blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  const int n = grp[gi].nstep;
  if (n == 0) return;  // uniform per group
  const int k0 = grp[gi].iters - n;
  if (cb < Vh) {
    const int64_t vh = Vh, unit0 = (int64_t)part * UPT;
    auto field_at = [&](const EoField& f, int64_t slot) {
      return reinterpret_cast<U*>(f.data) + (slot * f.nunits + unit0) * vh + cb;
    };
    U rr[kMsBlock][UPT];
#pragma unroll
    for (int j = 0; j < kMsBlock; ++j) {
      if (j >= n) break;
      const U* rp = field_at(ring, (int64_t)((k0 + j + 1) % kMsBlock) * 2 * G + par * G + gi);
#pragma unroll
      for (int u = 0; u < UPT; ++u) rr[j][u] = __ldg(rp + u * vh);
    }
    for (int s = 1; s < S; ++s) {
      const MsShift& T = shf[(int64_t)gi * S + s];
      if (!T.run[k0 % kMsBlock]) continue;
      const int64_t slot = (int64_t)par * G * S + gi * S + s;
      U* pp = field_at(ps, slot);
      U* xp = field_at(xs, slot);
      U pv[UPT], xv[UPT];
#pragma unroll
      for (int u = 0; u < UPT; ++u) {
        pv[u] = pp[u * vh];
        xv[u] = xp[u * vh];
      }
#pragma unroll
      for (int j = 0; j < kMsBlock; ++j) {
        if (j >= n) break;
        const int ix = (k0 + j) % kMsBlock;
        if (!T.run[ix]) break;  // the shift stopped after its previous step
        const RT a = (RT)T.a[ix], zn = (RT)T.zn[ix], b = (RT)T.b[ix];
#pragma unroll
        for (int u = 0; u < UPT; ++u) {
          ms_axpy(xv[u], a, pv[u]);
          ms_lincomb(pv[u], zn, rr[j][u], b);
        }
      }
#pragma unroll
      for (int u = 0; u < UPT; ++u) {
        pp[u * vh] = pv[u];
        xp[u * vh] = xv[u];
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counters + gi, 1u) == gridDim.x - 1) {
      grp[gi].nstep = 0;
      counters[gi] = 0u;  // ready for the next use of this slot
    }
  }
}

// threads per site of ms_xpm_split: at most three 16-byte units each
template <int NU> constexpr int ms_xpm_parts() { return NU % 4 == 0 && NU >= 8 ? 4 : (NU % 2 == 0 && NU > 3 ? 2 : 1); }

// ---------------------------------------------------------------------------
// FP64 kernels (reliable updates, verification); grids (2 nblk, G).
// The solutions x64 (nxs slots per parity, group gi's shift s at xmap[gi] + s)
// and sources b64 (nbs per parity, group gi's at bmap[gi]) may belong to
// another workspace.
// ---------------------------------------------------------------------------

// w64 = x + kappa H x, x = shift s of each group with upd
template <int ND, int NC>
__global__ void __launch_bounds__(128, 1) ms_dx64_kernel(EoGeom g, HopGauge hg, EoField x64, int nxs, const int* xmap,
                                                         int s, EoField w64, int G, double kappa, const int* upd,
                                                         int nblk) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  const int par = eo_block_parity(nblk);
  const int i = (blockIdx.x - par * nblk) * blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  if (!upd[gi] || i >= g.Vh) return;
  const int xs = xmap[gi] + s;
  const int act[1] = {1};
  cx<double> acc[1][NS][NC];
  hop_tile<ND, NC, SP64, SP64, false, false, 1>(g, hg, sub(x64, (int64_t)(1 - par) * nxs), xs, i, par, act, acc);
  cx<double> v[NCOMP];
  load_sp<SP64, NCOMP>(sub(x64, (int64_t)par * nxs), xs, i, v);
#pragma unroll
  for (int a = 0; a < NS; ++a)
#pragma unroll
    for (int c = 0; c < NC; ++c) v[a * NC + c] += kappa * acc[0][a][c];
  store_sp<SP64, NCOMP>(w64, par * G + gi, i, v);
}

// r64 = b - w64 - sigma_s x - kappa gamma_d H gamma_d w64 = b - (Q^2 + sigma_s) x ;
// res[gi] = |r64|^2
template <int ND, int NC>
__global__ void __launch_bounds__(128, 1) ms_res64_kernel(EoGeom g, HopGauge hg, EoField b64, int nbs,
                                                          const int* bmap, EoField x64, int nxs, const int* xmap,
                                                          int s, const MsShift* shf, int S, EoField w64, EoField r64,
                                                          int G, double kappa, const int* upd, double* partials,
                                                          unsigned* counters, double* res, int nblk) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  __shared__ double sh[32];
  const int par = eo_block_parity(nblk);
  const int i = (blockIdx.x - par * nblk) * blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  if (!upd[gi]) return;  // uniform per block
  double n[1] = {0.0};
  if (i < g.Vh) {
    const int act[1] = {1};
    cx<double> acc[1][NS][NC];
    hop_tile<ND, NC, SP64, SP64, false, true, 1>(g, hg, sub(w64, (int64_t)(1 - par) * G), gi, i, par, act, acc);
    const double sg = shf[(int64_t)gi * S + s].sigma;
    cx<double> bv[NCOMP], wv[NCOMP], xv[NCOMP];
    load_sp<SP64, NCOMP>(sub(b64, (int64_t)par * nbs), bmap[gi], i, bv);
    load_sp<SP64, NCOMP>(w64, par * G + gi, i, wv);
    load_sp<SP64, NCOMP>(sub(x64, (int64_t)par * nxs), xmap[gi] + s, i, xv);
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int m = a * NC + c;
        cx<double> h = acc[0][a][c];
        if (a >= NS / 2) h = -h;
        bv[m] = bv[m] - wv[m] - sg * xv[m] - kappa * h;
        n[0] += norm2(bv[m]);
      }
    store_sp<SP64, NCOMP>(r64, par * G + gi, i, bv);
  }
  if (grid_sum<1>(n, partials + (int64_t)gi * gridDim.x, counters + gi, sh) && threadIdx.x == 0) res[gi] = n[0];
}

// x64 += xs ; xs = 0 for every shift of the groups with upd; grid (2 nblk, G S)
template <int XP, int NCOMP>
__global__ void __launch_bounds__(128) ms_flush_kernel(int64_t Vh, int nblk, int G, int S, EoField xs, EoField x64,
                                                       int nxs, const int* xmap, const int* upd) {
  using XR = typename Prec<XP>::real;
  const int par = eo_block_parity(nblk);
  const int64_t cb = (blockIdx.x - par * nblk) * (int64_t)blockDim.x + threadIdx.x;
  const int slot = blockIdx.y, gi = slot / S, s = slot - gi * S;
  if (!upd[gi] || cb >= Vh) return;
  cx<XR> a[NCOMP];
  load_sp<XP, NCOMP>(xs, par * G * S + slot, cb, a);
  const EoField xv = sub(x64, (int64_t)par * nxs);
  cx<double> b[NCOMP];
  load_sp<SP64, NCOMP>(xv, xmap[gi] + s, cb, b);
  cx<XR> z[NCOMP];
#pragma unroll
  for (int k = 0; k < NCOMP; ++k) {
    b[k] += cx<double>{(double)a[k].re, (double)a[k].im};
    z[k] = czero<XR>();
  }
  store_sp<SP64, NCOMP>(xv, xmap[gi] + s, cb, b);
  store_sp<XP, NCOMP>(xs, par * G * S + slot, cb, z);
}

// r = r64 in the sloppy precision (into the ring slot of the group's
// iteration count) for groups with upd bit 1; with bit 2 also every
// direction p_k = r (a start or restart)
template <int SP, int NCOMP>
__global__ void __launch_bounds__(128) ms_sloppy_kernel(int64_t Vh, int nblk, int G, int S, EoField r64,
                                                        EoField ring, EoField pb, EoField ps, const int* upd,
                                                        const MsGroup* grp) {
  using RT = typename Prec<SP>::real;
  const int par = eo_block_parity(nblk);
  const int64_t cb = (blockIdx.x - par * nblk) * (int64_t)blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  const int u = upd[gi];
  if (!u || cb >= Vh) return;
  cx<double> v[NCOMP];
  load_sp<SP64, NCOMP>(r64, par * G + gi, cb, v);
  cx<RT> w[NCOMP];
#pragma unroll
  for (int k = 0; k < NCOMP; ++k) w[k] = {(RT)v[k].re, (RT)v[k].im};
  store_sp<SP, NCOMP>(sub(ring, (int64_t)(grp[gi].iters % kMsBlock) * 2 * G + par * G), gi, cb, w);
  if (u & 2) {
    store_sp<SP, NCOMP>(pb, par * G + gi, cb, w);
    for (int s = 0; s < S; ++s) store_sp<SP, NCOMP>(ps, par * G * S + gi * S + s, cb, w);
  }
}

// The directions of an FP64 workspace (Gi groups) in the inner precision of
// another (Go groups): the base direction and every shift's; grid (2 nblk, nreal)
template <int SP, int NCOMP>
__global__ void __launch_bounds__(128) ms_dirs_from64_kernel(int64_t Vh, int nblk, int Gi, int Go, int S,
                                                             EoField pbi, EoField psi, EoField pbo, EoField pso) {
  using RT = typename Prec<SP>::real;
  const int par = eo_block_parity(nblk);
  const int64_t cb = (blockIdx.x - par * nblk) * (int64_t)blockDim.x + threadIdx.x;
  const int gi = blockIdx.y;
  if (cb >= Vh) return;
  for (int s = -1; s < S; ++s) {
    cx<double> v[NCOMP];
    if (s < 0) load_sp<SP64, NCOMP>(pbi, par * Gi + gi, cb, v);
    else load_sp<SP64, NCOMP>(psi, par * Gi * S + gi * S + s, cb, v);
    cx<RT> w[NCOMP];
#pragma unroll
    for (int k = 0; k < NCOMP; ++k) w[k] = {(RT)v[k].re, (RT)v[k].im};
    if (s < 0) store_sp<SP, NCOMP>(pbo, par * Go + gi, cb, w);
    else store_sp<SP, NCOMP>(pso, par * Go * S + gi * S + s, cb, w);
  }
}

// reference layout (nrhs, ns, N, V) -> FP64 even-odd b64 (nbs slots per parity)
template <int ND, int NC>
__global__ void ms_from_ref_kernel(EoGeom g, int64_t V, const double2* __restrict__ ref, EoField b64, int nbs) {
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
  for (int c = 0; c < NCOMP; ++c) v[c] = ld(ref + ((int64_t)rhs * NCOMP + c) * V + lex);
  store_sp<SP64, NCOMP>(sub(b64, (int64_t)par * nbs), rhs, lex >> 1, v);
}

// x64 slot k (nxs per parity) -> reference-layout vector out_slot[k]
template <int ND, int NC>
__global__ void ms_to_ref_kernel(EoGeom g, int64_t V, EoField x64, int nxs, const int* out_slot,
                                 double2* __restrict__ ref) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  const int64_t lex = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (lex >= V) return;
  int x[ND];
  lex_coords<ND>(g, lex, x);
  int par = 0;
#pragma unroll
  for (int d = 0; d < ND; ++d) par += x[d];
  par &= 1;
  cx<double> v[NCOMP];
  load_sp<SP64, NCOMP>(sub(x64, (int64_t)par * nxs), k, lex >> 1, v);
  const int64_t o = out_slot[k];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c) st(ref + (o * NCOMP + c) * V + lex, v[c]);
}

// ---------------------------------------------------------------------------
// workspace
// ---------------------------------------------------------------------------
struct MsOps {
  void (*iterate)(MsWork&, cudaStream_t, int i);  // inner iteration i of a chunk (3 launches, +1 every kMsBlock)
  void (*dx64)(MsWork&, int s, cudaStream_t);
  void (*res64)(MsWork&, int s, cudaStream_t);
  void (*flush)(MsWork&, cudaStream_t);
  void (*sloppy)(MsWork&, cudaStream_t);
  void (*from_ref)(MsWork&, const void* ref, int nrhs, cudaStream_t);
  void (*to_ref)(MsWork&, void* ref, const int* out_slot, int nslot, cudaStream_t);
  void (*dirs_from64)(MsWork& dst, const MsWork& src, int nreal, cudaStream_t);
  void (*preload)();
};
constexpr int kMsLaunchesPerIteration = 3;  // plus one ms_xpm every kMsBlock iterations
constexpr size_t kMaxMsWorkspaces = 3;  // a solve uses up to three: FP64 head, inner precision, refinement

struct MsWork {
  lym_gauge* g = nullptr;
  int G = 0, cap = 0, S = 0;    // groups (capacity padded to a multiple of R), capacity, shifts per group
  int Greal = 0;                // groups of the current run (the rest idle)
  int sp = 0, xp = 0, R = 1;
  bool comp = false;
  int64_t Vh = 0;
  int nblk = 0;
  double kappa = 0;
  // FP64 sources and solutions: this workspace's own, or borrowed (phase 2)
  EoField b64, x64;
  int nbs = 0, nxs = 0;
  EoField own_b64, own_x64;  // allocated here (empty when this workspace only borrows)
  int own_nbs = 0, own_nxs = 0;
  EoField r64, w64;          // FP64 temporaries, G slots per parity
  EoField ring;              // sloppy residuals of the last kMsBlock iterations (kMsBlock x 2G slots)
  EoField pb, w;             // sloppy base direction and D p_0 (2G slots)
  EoField ps;                // every shift's direction at the last block boundary (2 G S slots)
  EoField xs;                // sloppy solution increments, FP32 for 16-bit inner precisions (2 G S slots)
  MsGroup* grp = nullptr;
  MsShift* shf = nullptr;
  int* upd = nullptr;
  int* xmap = nullptr;
  int* bmap = nullptr;
  int* oslot = nullptr;
  double* partials = nullptr;
  unsigned* counters = nullptr;
  double* res = nullptr;
  MsGroup* grp_h = nullptr;
  MsShift* shf_h = nullptr;
  int* upd_h = nullptr;
  int* map_h = nullptr;      // staging for xmap / bmap / oslot uploads
  double* res_h = nullptr;
  void* pool = nullptr;
  size_t pool_bytes = 0;
  HopGauge hg64, hgs;
  MsOps ops{};
  GraphRec rec;
  cudaGraphExec_t graph = nullptr;
  int graph_chunk = 0;
  double graph_kappa = 0;
  cudaStream_t graph_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int64_t launches = 0;
  int store_rhs = 0;  // right-hand sides the own FP64 store holds (0: none)
};

template <typename... KArgs, typename... Args>
static void ms_launch(MsWork& w, cudaStream_t st, void (*kernel)(KArgs...), dim3 grid, dim3 block, Args&&... args) {
  launch_rec(w.rec, st, kernel, grid, block, std::forward<Args>(args)...);
}

template <int ND, int NC, int SP, bool COMP, int R, int MX>
struct MsImpl {
  static constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC;
  static constexpr int GP = SP == SP64 ? SP64 : (SP == SP32 ? SP32 : SP16);
  static constexpr int XP = (SP == SP16 || SP == SPB16) ? SP32 : SP;

  static void iterate(MsWork& w, cudaStream_t st, int i) {
    dim3 tile(2 * w.nblk, w.G / R), grid(2 * w.nblk, w.G);
    ms_launch(w, st, ms_dp_kernel<ND, NC, SP, GP, COMP, R, MX>, tile, dim3(128), w.g->geom, w.hgs, w.pb, w.w, w.G,
              w.kappa, w.grp, w.partials, w.counters + w.G, w.nblk);
    ms_launch(w, st, ms_ap_kernel<ND, NC, SP, GP, COMP, R, MX>, tile, dim3(128), w.g->geom, w.hgs, w.w, w.pb, w.ring,
              w.G, w.S, w.kappa, w.grp, w.shf, w.partials, w.counters + w.G, w.nblk);
    ms_launch(w, st, ms_p0_kernel<SP, XP, NCOMP>, grid, dim3(128), w.Vh, w.nblk, w.G, w.S, w.ring, w.pb, w.xs, w.grp,
              w.counters);
    if ((i + 1) % kMsBlock == 0) {
      if constexpr (SP == SP64 || SP == SP32) {
        constexpr int NU = units_for(NCOMP, Prec<SP>::CPU), NG = ms_xpm_parts<NU>();
        ms_launch(w, st, ms_xpm_split_kernel<SP, NU, NG>, dim3(2 * w.nblk * NG, w.G), dim3(128), w.Vh, w.nblk, w.G,
                  w.S, w.ring, w.ps, w.xs, w.grp, (const MsShift*)w.shf, w.counters);
      } else {
        ms_launch(w, st, ms_xpm_kernel<SP, XP, NCOMP>, grid, dim3(128), w.Vh, w.nblk, w.G, w.S, w.ring, w.ps, w.xs,
                  w.grp, (const MsShift*)w.shf, w.counters);
      }
    }
  }
  static void dx64(MsWork& w, int s, cudaStream_t st) {
    w.launches += 1;
    ms_dx64_kernel<ND, NC><<<dim3(2 * w.nblk, w.G), 128, 0, st>>>(w.g->geom, w.hg64, w.x64, w.nxs, w.xmap, s, w.w64,
                                                                 w.G, w.kappa, w.upd, w.nblk);
  }
  static void res64(MsWork& w, int s, cudaStream_t st) {
    w.launches += 1;
    ms_res64_kernel<ND, NC><<<dim3(2 * w.nblk, w.G), 128, 0, st>>>(
        w.g->geom, w.hg64, w.b64, w.nbs, w.bmap, w.x64, w.nxs, w.xmap, s, w.shf, w.S, w.w64, w.r64, w.G, w.kappa,
        w.upd, w.partials, w.counters, w.res, w.nblk);
  }
  static void flush(MsWork& w, cudaStream_t st) {
    w.launches += 1;
    ms_flush_kernel<XP, NCOMP><<<dim3(2 * w.nblk, w.G * w.S), 128, 0, st>>>(w.Vh, w.nblk, w.G, w.S, w.xs, w.x64,
                                                                           w.nxs, w.xmap, w.upd);
  }
  static void sloppy(MsWork& w, cudaStream_t st) {
    w.launches += 1;
    ms_sloppy_kernel<SP, NCOMP><<<dim3(2 * w.nblk, w.G), 128, 0, st>>>(w.Vh, w.nblk, w.G, w.S, w.r64, w.ring,
                                                                      w.pb, w.ps, w.upd, w.grp);
  }
  static void from_ref(MsWork& w, const void* ref, int nrhs, cudaStream_t st) {
    w.launches += 1;
    ms_from_ref_kernel<ND, NC><<<dim3(grid_for(w.g->V, 128), nrhs), 128, 0, st>>>(
        w.g->geom, w.g->V, (const double2*)ref, w.own_b64, w.own_nbs);
  }
  static void to_ref(MsWork& w, void* ref, const int* out_slot, int nslot, cudaStream_t st) {
    w.launches += 1;
    ms_to_ref_kernel<ND, NC><<<dim3(grid_for(w.g->V, 128), nslot), 128, 0, st>>>(w.g->geom, w.g->V, w.own_x64,
                                                                                w.own_nxs, out_slot, (double2*)ref);
  }
  static void dirs_from64(MsWork& w, const MsWork& src, int nreal, cudaStream_t st) {
    w.launches += 1;
    ms_dirs_from64_kernel<SP, NCOMP><<<dim3(2 * w.nblk, nreal), 128, 0, st>>>(w.Vh, w.nblk, src.G, w.G, w.S, src.pb,
                                                                             src.ps, w.pb, w.ps);
  }
  static void preload() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, ms_dp_kernel<ND, NC, SP, GP, COMP, R, MX>);
    cudaFuncGetAttributes(&a, ms_ap_kernel<ND, NC, SP, GP, COMP, R, MX>);
    cudaFuncGetAttributes(&a, ms_p0_kernel<SP, XP, NCOMP>);
    if constexpr (SP == SP64 || SP == SP32) {
      constexpr int NU = units_for(NCOMP, Prec<SP>::CPU);
      cudaFuncGetAttributes(&a, ms_xpm_split_kernel<SP, NU, ms_xpm_parts<NU>()>);
    }
    else cudaFuncGetAttributes(&a, ms_xpm_kernel<SP, XP, NCOMP>);
  }
  static MsOps table() {
    return MsOps{&iterate, &dx64, &res64, &flush, &sloppy, &from_ref, &to_ref, &dirs_from64, &preload};
  }
};

// FP64: one group per thread; FP32: R groups per thread, 12-real links when
// the links allow; FP16: one group per thread, full links, mixed-precision hop
// (with neighbour indices from coordinate arithmetic on large lattices, arith);
// BF16: one group per thread, full links (the 16-bit choices are the fastest
// tiles of the CG's hop sweep)
template <int ND, int NC, int R>
static MsOps ms_pick_sp(int sp, bool comp, bool arith) {
  switch (sp) {
    case SP64: return MsImpl<ND, NC, SP64, false, 1, 0>::table();
    case SP32: return comp ? MsImpl<ND, NC, SP32, true, R, 0>::table() : MsImpl<ND, NC, SP32, false, R, 0>::table();
    case SP16: return arith ? MsImpl<ND, NC, SP16, false, 1, 4>::table() : MsImpl<ND, NC, SP16, false, 1, 1>::table();
    default: return MsImpl<ND, NC, SPB16, false, 1, 0>::table();
  }
}

template <int R>
static bool ms_pick_r(int nd, int nc, int sp, bool comp, bool arith, MsOps* out) {
  if (nd == 2 && nc == 2) *out = ms_pick_sp<2, 2, R>(sp, comp, arith);
  else if (nd == 2 && nc == 3) *out = ms_pick_sp<2, 3, R>(sp, comp, arith);
  else if (nd == 4 && nc == 2) *out = ms_pick_sp<4, 2, R>(sp, comp, arith);
  else if (nd == 4 && nc == 3) *out = ms_pick_sp<4, 3, R>(sp, comp, arith);
  else return false;
  return true;
}

static size_t ms_field_bytes(int sp, int ncomp, int64_t Vh, int64_t nslots) {
  const int cpu = sp == SP64 ? 1 : (sp == SP32 ? 2 : 4);
  size_t b = (size_t)units_for(ncomp, cpu) * 16 * Vh * nslots;
  if (sp == SP16 || sp == SPB16) b += sizeof(float) * Vh * nslots;
  return (b + 255) & ~(size_t)255;
}

static EoField ms_carve(char*& cur, int sp, int ncomp, int64_t Vh, int64_t nslots) {
  EoField f;
  const int cpu = sp == SP64 ? 1 : (sp == SP32 ? 2 : 4);
  f.nunits = units_for(ncomp, cpu);
  f.Vh = Vh;
  f.data = cur;
  size_t b = (size_t)f.nunits * 16 * Vh * nslots;
  if (sp == SP16 || sp == SPB16) {
    f.norm = reinterpret_cast<float*>(cur + b);
    b += sizeof(float) * Vh * nslots;
  }
  cur += (b + 255) & ~(size_t)255;
  return f;
}

static size_t ms_align(size_t b) { return (b + 255) & ~(size_t)255; }

// bytes a workspace of G groups x S shifts needs (store_rhs > 0: with its own
// FP64 store of store_rhs sources and store_rhs * S solutions)
static size_t ms_bytes(const lym_gauge* g, int G, int S, int sp, int store_rhs, int nblk) {
  const int nc = g->ncomp, xp = (sp == SP16 || sp == SPB16) ? SP32 : sp;
  const int64_t Vh = g->Vh;
  size_t b = 0;
  if (store_rhs > 0) {
    b += ms_field_bytes(SP64, nc, Vh, 2 * (int64_t)store_rhs);
    b += ms_field_bytes(SP64, nc, Vh, 2 * (int64_t)store_rhs * S);
  }
  b += 2 * ms_field_bytes(SP64, nc, Vh, 2 * (int64_t)G);
  b += ms_field_bytes(sp, nc, Vh, 2 * (int64_t)G * kMsBlock);
  b += 2 * ms_field_bytes(sp, nc, Vh, 2 * (int64_t)G);
  b += ms_field_bytes(sp, nc, Vh, 2 * (int64_t)G * S);
  b += ms_field_bytes(xp, nc, Vh, 2 * (int64_t)G * S);
  b += ms_align(sizeof(MsGroup) * G) + ms_align(sizeof(MsShift) * (size_t)G * S);
  b += ms_align(sizeof(int) * (size_t)G) + ms_align(sizeof(int) * 2 * (size_t)G);  // upd; xmap and bmap
  b += ms_align(sizeof(int) * (size_t)G * S);                                      // oslot
  b += ms_align(sizeof(double) * 4 * (size_t)G * nblk);
  b += ms_align(sizeof(unsigned) * 2 * (size_t)G);
  b += ms_align(sizeof(double) * (size_t)G);
  return b;
}

static void ms_free(MsWork* w) {
  if (!w) return;
  if (w->graph) cudaGraphExecDestroy(w->graph);
  if (w->stream) cudaStreamSynchronize(w->stream);
  if (w->pool) cudaFree(w->pool);
  if (w->ev_in) cudaEventDestroy(w->ev_in);
  if (w->ev_out) cudaEventDestroy(w->ev_out);
  if (w->stream) cudaStreamDestroy(w->stream);
  if (w->grp_h) cudaFreeHost(w->grp_h);
  if (w->shf_h) cudaFreeHost(w->shf_h);
  if (w->upd_h) cudaFreeHost(w->upd_h);
  if (w->map_h) cudaFreeHost(w->map_h);
  if (w->res_h) cudaFreeHost(w->res_h);
  delete w;
}

void free_ms_works(lym_gauge* g) {
  for (MsWork* w : g->ms_works) ms_free(w);
  g->ms_works.clear();
}

// A workspace for up to `cap` groups of S shifts (Greal is set per run).
// R: groups per hop-kernel thread (1, or 4 with the groups padded to a
// multiple of 4).  `keep` is never evicted (the workspace the others borrow from).
static int ms_get(lym_gauge* g, int cap, int S, int sp, int store_rhs, int want_r, const MsWork* keep,
                  MsWork** out) {
  const int R = (sp == SP32 && cap >= 4 && want_r != 1) ? 4 : 1;
  const int G = (cap + R - 1) / R * R;
  const bool comp = g->comp && sp == SP32;
  for (size_t i = 0; i < g->ms_works.size(); ++i) {
    MsWork* w = g->ms_works[i];
    if (w->cap == cap && w->S == S && w->sp == sp && w->store_rhs == store_rhs && w->R == R) {
      g->ms_works.erase(g->ms_works.begin() + i);  // most recently used first
      g->ms_works.insert(g->ms_works.begin(), w);
      w->Greal = cap;
      *out = w;
      return LYM_OK;
    }
  }
  while (g->ms_works.size() >= kMaxMsWorkspaces) {
    auto victim = g->ms_works.end() - 1;
    if (*victim == keep) --victim;
    ms_free(*victim);
    g->ms_works.erase(victim);
  }
  MsWork* w = new MsWork();
  w->g = g;
  w->G = G;
  w->cap = cap;
  w->Greal = cap;
  w->S = S;
  w->sp = sp;
  w->xp = (sp == SP16 || sp == SPB16) ? SP32 : sp;
  w->R = R;
  w->comp = comp;
  w->Vh = g->Vh;
  w->nblk = (int)grid_for(g->Vh, 128);
  w->store_rhs = store_rhs;
  // the CG's tile sweeps: arithmetic neighbours win from 24^3 x 48 (V/2 = 331 776) up,
  // the neighbour table at 16^4 (V/2 = 32 768)
  const bool arith = g->Vh >= (int64_t(1) << 17);
  const bool ok = R == 4 ? ms_pick_r<4>(g->nd, g->nc, sp, comp, arith, &w->ops)
                         : ms_pick_r<1>(g->nd, g->nc, sp, comp, arith, &w->ops);
  if (!ok) {
    delete w;
    set_error("unsupported (nd=%d, N=%d) for the even-odd multishift", g->nd, g->nc);
    return LYM_ERR_UNSUPPORTED;
  }
  const size_t bytes = ms_bytes(g, G, S, sp, store_rhs, w->nblk);
  if (cudaMalloc(&w->pool, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete w;
    set_error("multishift workspace of %zu bytes does not fit", bytes);
    return LYM_ERR_OOM;
  }
  w->pool_bytes = bytes;
  const int nc = g->ncomp;
  const int64_t Vh = g->Vh;
  char* cur = (char*)w->pool;
  if (store_rhs > 0) {
    w->own_b64 = ms_carve(cur, SP64, nc, Vh, 2 * (int64_t)store_rhs);
    w->own_nbs = store_rhs;
    w->own_x64 = ms_carve(cur, SP64, nc, Vh, 2 * (int64_t)store_rhs * S);
    w->own_nxs = store_rhs * S;
  }
  w->r64 = ms_carve(cur, SP64, nc, Vh, 2 * (int64_t)G);
  w->w64 = ms_carve(cur, SP64, nc, Vh, 2 * (int64_t)G);
  w->ring = ms_carve(cur, sp, nc, Vh, 2 * (int64_t)G * kMsBlock);
  w->pb = ms_carve(cur, sp, nc, Vh, 2 * (int64_t)G);
  w->w = ms_carve(cur, sp, nc, Vh, 2 * (int64_t)G);
  w->ps = ms_carve(cur, sp, nc, Vh, 2 * (int64_t)G * S);
  w->xs = ms_carve(cur, w->xp, nc, Vh, 2 * (int64_t)G * S);
  w->grp = reinterpret_cast<MsGroup*>(cur);
  cur += ms_align(sizeof(MsGroup) * G);
  w->shf = reinterpret_cast<MsShift*>(cur);
  cur += ms_align(sizeof(MsShift) * (size_t)G * S);
  w->upd = reinterpret_cast<int*>(cur);
  cur += ms_align(sizeof(int) * (size_t)G);
  w->xmap = reinterpret_cast<int*>(cur);
  w->bmap = w->xmap + G;
  cur += ms_align(sizeof(int) * 2 * (size_t)G);
  w->oslot = reinterpret_cast<int*>(cur);
  cur += ms_align(sizeof(int) * (size_t)G * S);
  w->partials = reinterpret_cast<double*>(cur);
  cur += ms_align(sizeof(double) * 4 * (size_t)G * w->nblk);
  w->counters = reinterpret_cast<unsigned*>(cur);
  cur += ms_align(sizeof(unsigned) * 2 * (size_t)G);
  w->res = reinterpret_cast<double*>(cur);
  // zero everything (reduction counters, padding groups) on the workspace's own
  // stream, complete before any other stream uses the pool
  if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMemsetAsync(w->pool, 0, bytes, w->stream) != cudaSuccess ||
      cudaStreamSynchronize(w->stream) != cudaSuccess ||
      cudaMallocHost(&w->grp_h, sizeof(MsGroup) * G) != cudaSuccess ||
      cudaMallocHost(&w->shf_h, sizeof(MsShift) * (size_t)G * S) != cudaSuccess ||
      cudaMallocHost(&w->upd_h, sizeof(int) * G) != cudaSuccess ||
      cudaMallocHost(&w->map_h, sizeof(int) * std::max<size_t>(2 * (size_t)G, (size_t)G * S)) != cudaSuccess ||
      cudaMallocHost(&w->res_h, sizeof(double) * G) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    ms_free(w);
    set_error("multishift workspace host buffers");
    return LYM_ERR_OOM;
  }
  w->hg64 = HopGauge{g->u64, g->nc * g->nc, 1.0, 0.0};
  if (sp == SP64) w->hgs = w->hg64;
  else if (sp == SP32) w->hgs = comp ? HopGauge{g->u32, g->n32, g->bcr, g->bci} : HopGauge{g->u32f, g->n32f, 1.0, 0.0};
  else w->hgs = comp ? HopGauge{g->u16, g->n16, g->bcr, g->bci} : HopGauge{g->u16f, g->n16f, 1.0, 0.0};
  g->ms_works.insert(g->ms_works.begin(), w);
  *out = w;
  return LYM_OK;
}

static int ms_build_graph(MsWork& w, int chunk, cudaStream_t st) {
  if (w.graph && w.graph_chunk == chunk && w.graph_kappa == w.kappa && w.graph_stream == st) return LYM_OK;
  if (w.graph) {
    cudaGraphExecDestroy(w.graph);
    w.graph = nullptr;
  }
  w.ops.preload();
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaGraphCreate(&graph, 0);
  if (e == cudaSuccess) {
    w.rec = GraphRec{graph, nullptr, cudaSuccess};
    for (int i = 0; i < chunk; ++i) w.ops.iterate(w, st, i);
    e = w.rec.err;
    w.rec = GraphRec{};
  }
  if (e == cudaSuccess) {
    e = cudaGraphInstantiate(&w.graph, graph, 0);
    if (e != cudaSuccess) w.graph = nullptr;
  }
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) cudaGetLastError();  // plain launches instead (w.graph stays null)
  w.graph_chunk = chunk;
  w.graph_kappa = w.kappa;
  w.graph_stream = st;
  return LYM_OK;
}

// FP64 true residual of shift s of every group with upd (after flushing the
// sloppy increments when `flush`): res_h[g] = |b - (Q^2 + sigma_s) x_s|^2.
static int ms_true_residual(MsWork& w, int s, bool flush, cudaStream_t st) {
  if (flush) w.ops.flush(w, st);
  w.ops.dx64(w, s, st);
  w.ops.res64(w, s, st);
  LYM_CHECK_LAUNCH();
  LYM_CUDA(cudaMemcpyAsync(w.res_h, w.res, sizeof(double) * w.G, cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  return LYM_OK;
}

struct MsOutcome {
  std::vector<int> done;      // true residual of the base below tol
  std::vector<int> updates;   // FP64 reliable updates
  std::vector<double> tres;   // last true relative residual of the base
};

// Runs the group CGs of w (grp_h / shf_h hold sigma and the zeroed recurrences,
// or with `resume` the state another workspace left; x64 holds each group's
// start) until each group's base true residual is below group_tol |b|
// (bnorm2: |b|^2 per group, < 0 to take it from the first residual, i.e. a
// zero start), it stalls (a group of several shifts: phase 2 takes over) or
// runs out of iterations.  The shifted systems stop on the final prm->tol.
static int ms_run(MsWork& w, const lym_solver_params* prm, double group_tol, bool resume,
                  std::vector<double>& bnorm2, MsOutcome& out, cudaStream_t st) {
  const int G = w.G, Gr = w.Greal, S = w.S;
  const double tol2 = group_tol * group_tol, final2 = prm->tol * prm->tol;
  const double delta = prm->delta > 0 && prm->delta < 1 ? prm->delta : 0.1;
  // a chunk ends on a block boundary, so no shift update is pending between chunks
  const int chunk = (std::max(1, prm->chunk > 0 ? std::min(prm->chunk, 256) : 8) + kMsBlock - 1) / kMsBlock * kMsBlock;
  const int max_interval = w.sp == SP64 ? (1 << 30) : 50;
  out.done.assign(G, 0);
  out.updates.assign(G, 0);
  out.tres.assign(G, 0.0);
  std::vector<int> ended(G, 0), restart(G, 0), iters_at_update(G, -1);
  std::vector<double> prev_q2(G, 0.0);
  for (int i = 0; i < G; ++i) {
    w.upd_h[i] = i < Gr ? 3 : 0;  // the first residual (and with a fresh start, every direction)
    if (i >= Gr) ended[i] = 1;
  }
  auto plan = [&](int i, double q2) {
    MsGroup& M = w.grp_h[i];
    const double want = tol2 * bnorm2[i];
    out.tres[i] = bnorm2[i] > 0 ? std::sqrt(q2 / bnorm2[i]) : 0.0;
    restart[i] = 0;
    // no iteration since the previous update (a zero or non-finite direction
    // or residual): nothing more will happen for this group
    const bool stuck = iters_at_update[i] == M.iters;
    iters_at_update[i] = M.iters;
    if (ms_trace())
      std::fprintf(stderr, "lym_ms: S=%d group %d iters %d true rel residual %.3e (previous %.3e)\n", S, i, M.iters,
                   out.tres[i], bnorm2[i] > 0 && prev_q2[i] > 0 ? std::sqrt(prev_q2[i] / bnorm2[i]) : 0.0);
    if (q2 <= want || q2 == 0.0) {
      out.done[i] = 1;
      M.active = 0;
      return;
    }
    if (stuck || !std::isfinite(q2)) {
      ended[i] = 1;
      M.active = 0;
      return;
    }
    if (prev_q2[i] > 0.0 && q2 > 0.25 * prev_q2[i]) {  // the true residual stalled
      if (S > 1) {  // the shifted solutions are refined one by one
        if (ms_trace()) std::fprintf(stderr, "lym_ms: group %d stalled, ends\n", i);
        ended[i] = 1;
        M.active = 0;
        return;
      }
      restart[i] = 1;  // one shift: restart the direction from the true residual
    }
    prev_q2[i] = q2;
    M.rr = q2;
    M.pause2 = w.sp == SP64 ? 0.25 * want : std::max(0.25 * want, delta * delta * q2);
    M.pause_iter = M.iters + max_interval;
    M.active = M.iters >= M.max_iter ? 0 : 1;
    if (!M.active) ended[i] = 1;
  };
  LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_h, sizeof(int) * G, cudaMemcpyHostToDevice, st));
  // the residual kernel reads each group's shift from the device copy
  LYM_CUDA(cudaMemcpyAsync(w.shf, w.shf_h, sizeof(MsShift) * (size_t)G * S, cudaMemcpyHostToDevice, st));
  int rc = ms_true_residual(w, 0, false, st);
  if (rc) return rc;
  for (int i = 0; i < Gr; ++i) {
    if (bnorm2[i] < 0) bnorm2[i] = w.res_h[i];
    for (int s = 1; s < S; ++s) w.shf_h[(size_t)i * S + s].stop2 = 0.25 * final2 * bnorm2[i];
    plan(i, w.res_h[i]);
    w.upd_h[i] = out.done[i] ? 0 : (resume ? 1 : 3);
  }
  LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_h, sizeof(int) * G, cudaMemcpyHostToDevice, st));
  LYM_CUDA(cudaMemcpyAsync(w.grp, w.grp_h, sizeof(MsGroup) * G, cudaMemcpyHostToDevice, st));
  LYM_CUDA(cudaMemcpyAsync(w.shf, w.shf_h, sizeof(MsShift) * (size_t)G * S, cudaMemcpyHostToDevice, st));
  w.ops.sloppy(w, st);
  LYM_CHECK_LAUNCH();
  rc = ms_build_graph(w, chunk, st);
  if (rc) return rc;
  while (true) {
    bool any_active = false;
    for (int i = 0; i < Gr; ++i) any_active = any_active || w.grp_h[i].active;
    if (!any_active) break;
    while (true) {
      if (w.graph) {
        LYM_CUDA(cudaGraphLaunch(w.graph, st));
      } else {
        for (int i = 0; i < chunk; ++i) w.ops.iterate(w, st, i);
        LYM_CHECK_LAUNCH();
      }
      w.launches += (int64_t)chunk * kMsLaunchesPerIteration + chunk / kMsBlock;
      LYM_CUDA(cudaMemcpyAsync(w.grp_h, w.grp, sizeof(MsGroup) * G, cudaMemcpyDeviceToHost, st));
      LYM_CUDA(cudaStreamSynchronize(st));
      bool running = false;
      for (int i = 0; i < Gr; ++i) running = running || w.grp_h[i].active;
      if (!running) break;
    }
    // reliable update of every group still going
    bool any = false;
    for (int i = 0; i < G; ++i) {
      w.upd_h[i] = (i < Gr && !out.done[i] && !ended[i]) ? 1 : 0;
      any = any || w.upd_h[i];
    }
    if (!any) break;
    LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_h, sizeof(int) * G, cudaMemcpyHostToDevice, st));
    rc = ms_true_residual(w, 0, true, st);
    if (rc) return rc;
    for (int i = 0; i < Gr; ++i) {
      if (!w.upd_h[i]) continue;
      out.updates[i] += 1;
      plan(i, w.res_h[i]);
      w.upd_h[i] = (out.done[i] || ended[i]) ? 0 : (restart[i] ? 3 : 1);
    }
    LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_h, sizeof(int) * G, cudaMemcpyHostToDevice, st));
    LYM_CUDA(cudaMemcpyAsync(w.grp, w.grp_h, sizeof(MsGroup) * G, cudaMemcpyHostToDevice, st));
    w.ops.sloppy(w, st);
    LYM_CHECK_LAUNCH();
  }
  // flush what the groups that ended without a final update still hold
  for (int i = 0; i < G; ++i) w.upd_h[i] = i < Gr ? 1 : 0;
  LYM_CUDA(cudaMemcpyAsync(w.upd, w.upd_h, sizeof(int) * G, cudaMemcpyHostToDevice, st));
  w.ops.flush(w, st);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

static void ms_init_states(MsWork& w, const std::vector<double>& group_base_sigma,
                           const std::vector<double>& shift_sigma /* G*S */, int max_iter) {
  for (int i = 0; i < w.G; ++i) {
    MsGroup& M = w.grp_h[i];
    std::memset(&M, 0, sizeof(M));
    M.alpha_prev = 1.0;
    M.beta_prev = 0.0;
    M.sigma = i < w.Greal ? group_base_sigma[i] : 0.0;
    M.max_iter = max_iter;
    for (int s = 0; s < w.S; ++s) {
      MsShift& T = w.shf_h[(size_t)i * w.S + s];
      std::memset(&T, 0, sizeof(T));
      T.sigma = i < w.Greal ? shift_sigma[(size_t)i * w.S + s] : 0.0;
      T.z = T.zprev = 1.0;
      T.active = i < w.Greal ? 1 : 0;
    }
  }
}

// Orders the caller's later work after everything the solve enqueued on its
// own stream, on every way out of the solve (errors included).
struct MsFence {
  cudaEvent_t ev;
  cudaStream_t from, to;
  ~MsFence() {
    cudaEventRecord(ev, from);
    cudaStreamWaitEvent(to, ev, 0);
  }
};

static int ms_solve_on(lym_gauge* g, double kappa, int nrhs, int nshift, const double* shifts, const void* b,
                       void* xs, const lym_solver_params* prm, lym_solver_report* rep, cudaStream_t caller) {
  const int sp = prm->precision;
  // internal shift order: the smallest first (the base), the rest ascending
  std::vector<int> order(nshift);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return shifts[a] < shifts[c]; });
  MsWork* w1p;
  int rc = ms_get(g, nrhs, nshift, sp, nrhs, prm->rhs_per_thread, nullptr, &w1p);
  if (rc) return rc;
  MsWork& w1 = *w1p;
  const int S = nshift;
  cudaStream_t st = w1.stream;
  LYM_CUDA(cudaEventRecord(w1.ev_in, caller));
  LYM_CUDA(cudaStreamWaitEvent(st, w1.ev_in, 0));
  const MsFence fence{w1.ev_out, st, caller};
  w1.kappa = kappa;
  w1.launches = 0;
  w1.b64 = w1.own_b64;
  w1.nbs = w1.own_nbs;
  w1.x64 = w1.own_x64;
  w1.nxs = w1.own_nxs;
  // sources, zero starts
  w1.ops.from_ref(w1, b, nrhs, st);
  LYM_CUDA(cudaMemsetAsync(w1.own_x64.data, 0, ms_field_bytes(SP64, g->ncomp, g->Vh, 2 * (int64_t)w1.own_nxs), st));
  LYM_CUDA(cudaMemsetAsync(w1.xs.data, 0, ms_field_bytes(w1.xp, g->ncomp, g->Vh, 2 * (int64_t)w1.G * S), st));
  for (int i = 0; i < w1.G; ++i) {
    w1.map_h[i] = std::min(i, nrhs - 1) * S;  // xmap: the padding groups never run
    w1.map_h[w1.G + i] = std::min(i, nrhs - 1);  // bmap
  }
  LYM_CUDA(cudaMemcpyAsync(w1.xmap, w1.map_h, sizeof(int) * 2 * w1.G, cudaMemcpyHostToDevice, st));
  std::vector<double> base_sigma(nrhs, shifts[order[0]]), shift_sigma((size_t)nrhs * S);
  for (int i = 0; i < nrhs; ++i)
    for (int s = 0; s < S; ++s) shift_sigma[(size_t)i * S + s] = shifts[order[s]];
  ms_init_states(w1, base_sigma, shift_sigma, prm->max_iter);
  std::vector<double> bnorm2(w1.G, -1.0);
  MsOutcome o1;
  const auto t0 = std::chrono::steady_clock::now();
  auto trace_ms = [&]() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };
  // FP64 head (reduced inner precisions): the same groups in an FP64 workspace
  // until the base true residual is below the switch point
  double sw = prm->switch_residual;
  if (sw == 0.0) sw = sp == SP32 ? 1e-4 : (sp == SP16 ? 1e-6 : 1e-7);
  const bool head = sp != SP64 && sw > prm->tol;
  std::vector<int> head_updates(nrhs, 0);
  if (head) {
    MsWork* whp;
    rc = ms_get(g, nrhs, nshift, SP64, 0, prm->rhs_per_thread, &w1, &whp);
    if (rc) return rc;
    MsWork& wh = *whp;
    wh.kappa = kappa;
    wh.launches = 0;
    wh.b64 = w1.own_b64;
    wh.nbs = w1.own_nbs;
    wh.x64 = w1.own_x64;
    wh.nxs = w1.own_nxs;
    wh.Greal = nrhs;
    for (int i = 0; i < wh.G; ++i) {
      wh.map_h[i] = std::min(i, nrhs - 1) * S;
      wh.map_h[wh.G + i] = std::min(i, nrhs - 1);
    }
    LYM_CUDA(cudaMemcpyAsync(wh.xmap, wh.map_h, sizeof(int) * 2 * wh.G, cudaMemcpyHostToDevice, st));
    LYM_CUDA(cudaMemsetAsync(wh.xs.data, 0, ms_field_bytes(SP64, g->ncomp, g->Vh, 2 * (int64_t)wh.G * S), st));
    ms_init_states(wh, base_sigma, shift_sigma, prm->max_iter);
    std::vector<double> bn_h(wh.G, -1.0);
    MsOutcome oh;
    rc = ms_run(wh, prm, sw, false, bn_h, oh, st);
    if (rc) return rc;
    // the state moves to the inner-precision workspace
    LYM_CUDA(cudaMemcpyAsync(wh.shf_h, wh.shf, sizeof(MsShift) * (size_t)wh.G * S, cudaMemcpyDeviceToHost, st));
    LYM_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < nrhs; ++i) {
      w1.grp_h[i] = wh.grp_h[i];
      w1.grp_h[i].nstep = 0;
      for (int s = 0; s < S; ++s) w1.shf_h[(size_t)i * S + s] = wh.shf_h[(size_t)i * S + s];
      bnorm2[i] = bn_h[i];
      head_updates[i] = oh.updates[i];
    }
    w1.ops.dirs_from64(w1, wh, nrhs, st);
    LYM_CHECK_LAUNCH();
    w1.launches += wh.launches;
    if (ms_trace()) std::fprintf(stderr, "lym_ms: FP64 head done at %.2f ms\n", trace_ms());
  }
  rc = ms_run(w1, prm, prm->tol, head, bnorm2, o1, st);
  if (rc) return rc;
  for (int i = 0; i < nrhs; ++i) o1.updates[i] += head_updates[i];
  if (ms_trace()) std::fprintf(stderr, "lym_ms: phase 1 done at %.2f ms\n", trace_ms());
  if (ms_trace()) {
    LYM_CUDA(cudaMemcpyAsync(w1.shf_h, w1.shf, sizeof(MsShift) * (size_t)w1.G * S, cudaMemcpyDeviceToHost, st));
    LYM_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < nrhs; ++i)
      for (int s = 0; s < S; ++s) {
        const MsShift& T = w1.shf_h[(size_t)i * S + s];
        std::fprintf(stderr, "lym_ms: phase 1 rhs %d shift %.3e active %d zeta %.3e\n", i, T.sigma, T.active, T.z);
      }
  }
  // verification: FP64 true residual of every (rhs, shift)
  std::vector<double> q2((size_t)nrhs * S, 0.0);
  for (int i = 0; i < w1.G; ++i) w1.upd_h[i] = i < nrhs ? 1 : 0;
  LYM_CUDA(cudaMemcpyAsync(w1.upd, w1.upd_h, sizeof(int) * w1.G, cudaMemcpyHostToDevice, st));
  for (int s = 0; s < S; ++s) {
    rc = ms_true_residual(w1, s, false, st);
    if (rc) return rc;
    for (int i = 0; i < nrhs; ++i) q2[(size_t)i * S + s] = w1.res_h[i];
  }
  std::vector<int> iters((size_t)nrhs * S), updates((size_t)nrhs * S), status((size_t)nrhs * S, LYM_OK);
  std::vector<double> tres((size_t)nrhs * S);
  std::vector<int> todo;
  for (int i = 0; i < nrhs; ++i)
    for (int s = 0; s < S; ++s) {
      const size_t k = (size_t)i * S + s;
      iters[k] = w1.grp_h[i].iters;
      updates[k] = o1.updates[i];
      tres[k] = bnorm2[i] > 0 ? std::sqrt(q2[k] / bnorm2[i]) : 0.0;
      if (ms_trace())
        std::fprintf(stderr, "lym_ms: verify rhs %d shift %.3e iters %d true rel residual %.3e\n", i,
                     shifts[order[s]], iters[k], tres[k]);
      if (q2[k] > prm->tol * prm->tol * bnorm2[i]) todo.push_back((int)k);
    }
  if (ms_trace()) std::fprintf(stderr, "lym_ms: verification done at %.2f ms, %zu pairs to refine\n", trace_ms(),
                               todo.size());
  int64_t launches = 0;
  // phase 2: the pairs above tol, each a CG of its own, in batches of the
  // first batch's size (what fits in free memory, at most 64)
  size_t at = 0;
  int cap2 = 0;
  while (at < todo.size()) {
    if (cap2 == 0) {
      size_t free_b = 0, total_b = 0;
      cudaMemGetInfo(&free_b, &total_b);
      const size_t per = ms_bytes(g, 4, 1, sp, 0, w1.nblk) / 4 + 1;
      cap2 = (int)std::min<size_t>(todo.size(), 64);
      cap2 = (int)std::max<size_t>(1, std::min<size_t>(cap2, (size_t)(0.6 * (double)free_b) / per));
    }
    const int batch = (int)std::min<size_t>(todo.size() - at, cap2);
    MsWork* w2p;
    rc = ms_get(g, cap2, 1, sp, 0, prm->rhs_per_thread, &w1, &w2p);
    if (rc) return rc;
    MsWork& w2 = *w2p;
    w2.Greal = batch;
    w2.kappa = kappa;
    w2.launches = 0;
    w2.b64 = w1.own_b64;
    w2.nbs = w1.own_nbs;
    w2.x64 = w1.own_x64;
    w2.nxs = w1.own_nxs;
    std::vector<double> bs(batch), ss(batch), bn2(w2.G, -1.0);
    for (int j = 0; j < w2.G; ++j) {
      const int k = todo[at + std::min(j, batch - 1)];
      const int i = k / S, s = k % S;
      w2.map_h[j] = i * S + s;   // xmap
      w2.map_h[w2.G + j] = i;    // bmap
      if (j < batch) {
        bs[j] = shifts[order[s]];
        ss[j] = shifts[order[s]];
        bn2[j] = bnorm2[i];
      }
    }
    // w2 runs on w1's stream (the fields it borrows are w1's)
    LYM_CUDA(cudaMemcpyAsync(w2.xmap, w2.map_h, sizeof(int) * 2 * w2.G, cudaMemcpyHostToDevice, st));
    LYM_CUDA(cudaMemsetAsync(w2.xs.data, 0, ms_field_bytes(w2.xp, g->ncomp, g->Vh, 2 * (int64_t)w2.G), st));
    ms_init_states(w2, bs, ss, std::max(1, prm->max_iter));
    MsOutcome o2;
    rc = ms_run(w2, prm, prm->tol, false, bn2, o2, st);
    if (rc) return rc;
    for (int j = 0; j < batch; ++j) {
      const int k = todo[at + j];
      iters[k] += w2.grp_h[j].iters;
      updates[k] += o2.updates[j];
      tres[k] = o2.tres[j];
      if (!o2.done[j]) status[k] = LYM_ERR_NOT_CONVERGED;
    }
    launches += w2.launches;
    at += batch;
    if (ms_trace()) std::fprintf(stderr, "lym_ms: phase 2 batch of %d done at %.2f ms\n", batch, trace_ms());
  }
  // solutions back in the caller's shift order
  for (int i = 0; i < nrhs; ++i)
    for (int s = 0; s < S; ++s) w1.map_h[(size_t)i * S + s] = i * S + order[s];
  LYM_CUDA(cudaMemcpyAsync(w1.oslot, w1.map_h, sizeof(int) * (size_t)nrhs * S, cudaMemcpyHostToDevice, st));
  w1.ops.to_ref(w1, xs, w1.oslot, nrhs * S, st);
  LYM_CHECK_LAUNCH();
  LYM_CUDA(cudaStreamSynchronize(st));
  launches += w1.launches;
  int result = LYM_OK;
  for (int i = 0; i < nrhs; ++i)
    for (int s = 0; s < S; ++s) {
      const size_t k = (size_t)i * S + s;
      lym_solver_report& R = rep[(size_t)i * S + order[s]];
      std::memset(&R, 0, sizeof(R));
      R.status = status[k];
      R.iterations = iters[k];
      R.reliable_updates = updates[k];
      R.true_residual = tres[k];
      R.kernel_launches = launches;
      R.rhs_per_thread = w1.R;
      R.compressed_links = w1.comp ? 1 : 0;
      R.mixed_fma = 0;
      if (status[k] != LYM_OK) result = LYM_ERR_NOT_CONVERGED;
    }
  return result;
}

}  // namespace lym

using namespace lym;

extern "C" {

int lym_multishift_solve_eo(lym_gauge* g, double kappa, int nrhs, int nshift, const double* shifts, const void* b,
                            void* xs, const lym_solver_params* params, lym_solver_report* reports, void* stream) {
  LYM_REQUIRE(g && shifts && b && xs && params && reports, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nrhs >= 1 && nrhs <= 1024, LYM_ERR_BAD_ARG, "nrhs out of range");
  LYM_REQUIRE(g->nd != 3, LYM_ERR_UNSUPPORTED,
              "Q^2 + sigma needs the hermitian Q = gamma_d D, which three dimensions do not have");
  LYM_REQUIRE(nshift >= 1 && nshift <= kMsMaxShifts, LYM_ERR_BAD_ARG, "nshift must be in [1, %d]", kMsMaxShifts);
  LYM_REQUIRE(params->tol > 0 && params->max_iter > 0, LYM_ERR_BAD_ARG, "tol and max_iter must be positive");
  LYM_REQUIRE(params->precision >= 0 && params->precision <= 3, LYM_ERR_BAD_ARG, "bad precision");
  LYM_REQUIRE(params->precision == SP64 || (g->prec_mask >> params->precision) & 1u, LYM_ERR_BAD_ARG,
              "precision %d was not enabled in lym_gauge_create", params->precision);
  for (int s = 0; s < nshift; ++s)
    LYM_REQUIRE(shifts[s] >= 0, LYM_ERR_BAD_ARG, "negative shifts need BiCGStab (dirac_solver.py:26-30)");
  std::lock_guard<std::recursive_mutex> own(g->mu);
  return ms_solve_on(g, kappa, nrhs, nshift, shifts, b, xs, params, reports, (cudaStream_t)stream);
}

}  // extern "C"
