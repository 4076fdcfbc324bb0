// Even-odd (checkerboard) layouts and the hopping-term core for the solvers.
//
// Ordering (builder-defined; the reference has no even-odd preconditioning):
// parity(x) = sum_i x_i mod 2; within a parity, sites keep the reference's
// lexicographic order, so the checkerboard index is lex / 2 (all extents even).
//
// Spinor field of one parity, nrhs vectors:  unit[(rhs * nunits + u) * Vh + cb]
//   FP64 : double2 units, 1 complex each
//   FP32 : float4 units, 2 complex each
//   FP16 / BF16 : uint4 units, 4 complex each, plus a float norm per site
//          (values stored divided by the site's max |re|,|im|)
// Gauge field: unit[((mu * 2 + parity) * nunits + u) * Vh + cb] holding
//   U_mu(x) for x of that parity; full N x N, or compressed to the first
//   N-1 rows (SU(3): 12 reals, third row = conj(row0 x row1); SU(2): 4 reals,
//   row1 = (-conj(b), conj(a))).  FP64 and full links have the boundary
//   factor folded in; compressed links get it at load time.
#pragma once

#include "lym_internal.cuh"

namespace lym {

enum { SP64 = 0, SP32 = 1, SP16 = 2, SPB16 = 3 };

template <int SP> struct Prec;
template <> struct Prec<SP64> { using real = double; using unit = double2; static constexpr int CPU = 1; };
template <> struct Prec<SP32> { using real = float; using unit = float4; static constexpr int CPU = 2; };
template <> struct Prec<SP16> { using real = float; using unit = uint4; static constexpr int CPU = 4; };
template <> struct Prec<SPB16> { using real = float; using unit = uint4; static constexpr int CPU = 4; };

constexpr int units_for(int ncomplex, int cpu) { return (ncomplex + cpu - 1) / cpu; }

struct EoField {
  void* data = nullptr;
  float* norm = nullptr;
  int nunits = 0;
  int64_t Vh = 0;
};

// --- half / bfloat16 packing ------------------------------------------------
template <int SP> LYM_D unsigned pack2(float a, float b);
template <> LYM_D unsigned pack2<SP16>(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<unsigned*>(&h);
}
template <> LYM_D unsigned pack2<SPB16>(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<unsigned*>(&h);
}
template <int SP> LYM_D cx<float> unpack2(unsigned w);
template <> LYM_D cx<float> unpack2<SP16>(unsigned w) {
  __half2 h = *reinterpret_cast<__half2*>(&w);
  float2 f = __half22float2(h);
  return {f.x, f.y};
}
template <> LYM_D cx<float> unpack2<SPB16>(unsigned w) {
  __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&w);
  float2 f = __bfloat1622float2(h);
  return {f.x, f.y};
}

// --- spinor load / store ------------------------------------------------------
template <int SP, int NCOMP>
LYM_D void load_sp(const EoField& f, int rhs, int64_t cb, cx<typename Prec<SP>::real> (&v)[NCOMP]) {
  using U = typename Prec<SP>::unit;
  const U* base = reinterpret_cast<const U*>(f.data) + (int64_t)rhs * f.nunits * f.Vh + cb;
  if constexpr (SP == SP64) {
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
      double2 t = __ldg(base + c * f.Vh);
      v[c] = {t.x, t.y};
    }
  } else if constexpr (SP == SP32) {
#pragma unroll
    for (int u = 0; u < units_for(NCOMP, 2); ++u) {
      float4 t = __ldg(base + u * f.Vh);
      v[2 * u] = {t.x, t.y};
      if (2 * u + 1 < NCOMP) v[2 * u + 1] = {t.z, t.w};
    }
  } else {
    const float nrm = __ldg(f.norm + (int64_t)rhs * f.Vh + cb);
#pragma unroll
    for (int u = 0; u < units_for(NCOMP, 4); ++u) {
      uint4 t = __ldg(base + u * f.Vh);
      const unsigned w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (4 * u + k < NCOMP) v[4 * u + k] = nrm * unpack2<SP>(w[k]);
    }
  }
}

template <int SP, int NCOMP>
LYM_D void store_sp(const EoField& f, int rhs, int64_t cb, const cx<typename Prec<SP>::real> (&v)[NCOMP]) {
  using U = typename Prec<SP>::unit;
  U* base = reinterpret_cast<U*>(f.data) + (int64_t)rhs * f.nunits * f.Vh + cb;
  if constexpr (SP == SP64) {
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) base[c * f.Vh] = make_double2(v[c].re, v[c].im);
  } else if constexpr (SP == SP32) {
#pragma unroll
    for (int u = 0; u < units_for(NCOMP, 2); ++u) {
      cx<float> b = (2 * u + 1 < NCOMP) ? v[2 * u + 1] : cx<float>{0.f, 0.f};
      base[u * f.Vh] = make_float4(v[2 * u].re, v[2 * u].im, b.re, b.im);
    }
  } else {
    float m = 0.f;
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) m = fmaxf(m, fmaxf(fabsf(v[c].re), fabsf(v[c].im)));
    const float inv = m > 0.f ? 1.0f / m : 0.f;
    f.norm[(int64_t)rhs * f.Vh + cb] = m;
#pragma unroll
    for (int u = 0; u < units_for(NCOMP, 4); ++u) {
      unsigned w[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        cx<float> c = (4 * u + k < NCOMP) ? v[4 * u + k] : cx<float>{0.f, 0.f};
        w[k] = pack2<SP>(c.re * inv, c.im * inv);
      }
      base[u * f.Vh] = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Raw load: values as stored (not multiplied by the site norm) and the norm
// (1 for FP64 / FP32), so callers can fold the norm into fewer multiplies.
// 32-bit offsets within one rhs (nunits * Vh < 2^31 is checked at creation).
template <int SP, int NCOMP>
LYM_D float load_sp_raw(const EoField& f, int rhs, int cb, cx<typename Prec<SP>::real> (&v)[NCOMP]) {
  using U = typename Prec<SP>::unit;
  const int vh = (int)f.Vh;
  const U* base = reinterpret_cast<const U*>(f.data) + (size_t)rhs * f.nunits * f.Vh;
  if constexpr (SP == SP64) {
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
      double2 t = __ldg(base + c * vh + cb);
      v[c] = {t.x, t.y};
    }
    return 1.0f;
  } else if constexpr (SP == SP32) {
#pragma unroll
    for (int u = 0; u < units_for(NCOMP, 2); ++u) {
      float4 t = __ldg(base + u * vh + cb);
      v[2 * u] = {t.x, t.y};
      if (2 * u + 1 < NCOMP) v[2 * u + 1] = {t.z, t.w};
    }
    return 1.0f;
  } else {
#pragma unroll
    for (int u = 0; u < units_for(NCOMP, 4); ++u) {
      uint4 t = __ldg(base + u * vh + cb);
      const unsigned w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (4 * u + k < NCOMP) v[4 * u + k] = unpack2<SP>(w[k]);
    }
    return __ldg(f.norm + (size_t)rhs * f.Vh + cb);
  }
}

// --- gauge load -----------------------------------------------------------
// GP: storage precision (SP64 double2, SP32 float4, SP16 uint2 of 2 half2)
// COMP: compressed to N-1 rows
template <int GP> struct GPrec;
template <> struct GPrec<SP64> { using real = double; using unit = double2; static constexpr int CPU = 1; };
template <> struct GPrec<SP32> { using real = float; using unit = float4; static constexpr int CPU = 2; };
template <> struct GPrec<SP16> { using real = float; using unit = uint2; static constexpr int CPU = 2; };

template <int NC, bool COMP> constexpr int link_complex() { return COMP ? (NC - 1) * NC : NC * NC; }

template <int GP, int NC, bool COMP>
LYM_D void load_link_eo(const void* g, int nunits, int64_t Vh, int mu, int par, int64_t cb,
                        cx<typename GPrec<GP>::real> (&u)[NC][NC]) {
  using R = typename GPrec<GP>::real;
  using U = typename GPrec<GP>::unit;
  constexpr int NCX = link_complex<NC, COMP>();
  const U* base = reinterpret_cast<const U*>(g) + ((int64_t)(mu * 2 + par) * nunits) * Vh + cb;
  cx<R> e[NCX];
  if constexpr (GP == SP64) {
#pragma unroll
    for (int k = 0; k < NCX; ++k) {
      double2 t = __ldg(base + k * Vh);
      e[k] = {t.x, t.y};
    }
  } else if constexpr (GP == SP32) {
#pragma unroll
    for (int k = 0; k < units_for(NCX, 2); ++k) {
      float4 t = __ldg(base + k * Vh);
      e[2 * k] = {t.x, t.y};
      if (2 * k + 1 < NCX) e[2 * k + 1] = {t.z, t.w};
    }
  } else {
#pragma unroll
    for (int k = 0; k < units_for(NCX, 2); ++k) {
      uint2 t = __ldg(base + k * Vh);
      e[2 * k] = unpack2<SP16>(t.x);
      if (2 * k + 1 < NCX) e[2 * k + 1] = unpack2<SP16>(t.y);
    }
  }
  if constexpr (!COMP) {
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) u[i][j] = e[i * NC + j];
  } else if constexpr (NC == 2) {
    u[0][0] = e[0];
    u[0][1] = e[1];
    u[1][0] = -conj(e[1]);
    u[1][1] = conj(e[0]);
  } else {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      u[0][j] = e[j];
      u[1][j] = e[3 + j];
    }
    // row2 = conj(row0 x row1)
    cx<R> t0 = u[0][1] * u[1][2], t1 = u[0][2] * u[1][0], t2 = u[0][0] * u[1][1];
    cmac(t0, -u[0][2], u[1][1]);
    cmac(t1, -u[0][0], u[1][2]);
    cmac(t2, -u[0][1], u[1][0]);
    u[2][0] = conj(t0);
    u[2][1] = conj(t1);
    u[2][2] = conj(t2);
  }
}

// --- geometry of the checkerboard ------------------------------------------
struct EoGeom {
  int nd;
  int dims[4];
  int stride[4];  // lexicographic strides (last coordinate fastest)
  int Lh;         // dims[nd-1] / 2
  int64_t Vh;
  // Neighbour table of the checkerboard, nbr[(par * 2 nd + 2 mu + dir) * Vh + cb]:
  // the checkerboard index of x +- mu (dir 0: +, 1: -) for x of parity par,
  // with bit 31 set when the hop crosses the time boundary (mu = nd-1 and the
  // link involved sits on the last time slice).  Built once per gauge object.
  const int* nbr;
};
constexpr int kNbrBoundary = int(0x80000000u);

// coordinates and lexicographic index of checkerboard site (cb, parity);
// 32-bit arithmetic throughout (the volume is below 2^31)
template <int ND>
LYM_D int eo_coords(const EoGeom& g, int cb, int par, int (&x)[ND]) {
  const int Lt = g.dims[ND - 1];
  const unsigned row = (unsigned)cb / (unsigned)g.Lh;
  const int th = cb - (int)row * g.Lh;
  unsigned r = row;
  int sum = 0;
#pragma unroll
  for (int d = ND - 2; d >= 0; --d) {
    const unsigned q = r / (unsigned)g.dims[d];
    x[d] = (int)(r - q * (unsigned)g.dims[d]);
    r = q;
    sum += x[d];
  }
  x[ND - 1] = 2 * th + ((par + sum) & 1);
  return (int)row * Lt + x[ND - 1];
}

// coordinates of lexicographic site lex (last coordinate fastest)
template <int ND>
LYM_D void lex_coords(const EoGeom& g, int64_t lex, int (&x)[ND]) {
  int64_t r = lex;
#pragma unroll
  for (int d = ND - 1; d >= 0; --d) {
    x[d] = (int)(r % g.dims[d]);
    r /= g.dims[d];
  }
}

template <int ND>
LYM_D int nb_fwd(const EoGeom& g, int lex, const int (&x)[ND], int mu) {
  return (x[mu] == g.dims[mu] - 1) ? lex - (g.dims[mu] - 1) * g.stride[mu] : lex + g.stride[mu];
}
template <int ND>
LYM_D int nb_bwd(const EoGeom& g, int lex, const int (&x)[ND], int mu) {
  return (x[mu] == 0) ? lex + (g.dims[mu] - 1) * g.stride[mu] : lex - g.stride[mu];
}

// --- hopping term -----------------------------------------------------------
struct HopGauge {
  const void* data;
  int nunits;
  double bcr, bci;  // boundary factor applied at load time (compressed links only)
};

// acc = sum_mu [U_mu(x)(1-g_mu) psi(x+mu) + U_mu(x-mu)^dag (1+g_mu) psi(x-mu)]
// for x of parity `par`; psi is the opposite-parity field.  G5IN: psi is
// replaced by gamma_d psi (lower spin components negated) on load.
template <int ND, int NC, int SP, int GP, bool COMP, bool G5IN>
LYM_D void hop_site(const EoGeom& g, const HopGauge& hg, const EoField& in, int rhs, int64_t cb, int par,
                    cx<typename Prec<SP>::real> (&acc)[Gamma<ND>::NS][NC]) {
  using R = typename Prec<SP>::real;
  using GR = typename GPrec<GP>::real;
  constexpr int NS = Gamma<ND>::NS;
  int x[ND];
  const int lex = eo_coords<ND>(g, (int)cb, par, x);
#pragma unroll
  for (int a = 0; a < NS; ++a)
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[a][c] = czero<R>();
#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int nlex = fwd ? nb_fwd<ND>(g, lex, x, mu) : nb_bwd<ND>(g, lex, x, mu);
      const int ncb = nlex >> 1;
      cx<GR> ug[NC][NC];
      // forward link lives on x (parity par), backward link on x - mu (parity 1-par)
      load_link_eo<GP, NC, COMP>(hg.data, hg.nunits, g.Vh, mu, fwd ? par : 1 - par, fwd ? cb : ncb, ug);
      cx<R> u[NC][NC];
#pragma unroll
      for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) u[i][j] = {(R)ug[i][j].re, (R)ug[i][j].im};
      if (COMP && mu == ND - 1 && x[ND - 1] == (fwd ? g.dims[ND - 1] - 1 : 0)) {
        const cx<R> bc{(R)hg.bcr, (R)hg.bci};
#pragma unroll
        for (int i = 0; i < NC; ++i)
#pragma unroll
          for (int j = 0; j < NC; ++j) u[i][j] = bc * u[i][j];
      }
      cx<R> psi[NS * NC];
      load_sp<SP, NS * NC>(in, rhs, ncb, psi);
      if constexpr (ND == 3) {
        // two-component spinors: G5IN selects the adjoint hop (gamma -> -gamma)
        const int s3 = (fwd != G5IN) ? 1 : -1;
        cx<R> p0[NC], p1[NC], h[NC], t[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          p0[c] = psi[c];
          p1[c] = psi[NC + c];
        }
        proj3<R, NC>(mu, s3, p0, p1, h);
#pragma unroll
        for (int i = 0; i < NC; ++i) {
          if (fwd) {
            t[i] = u[i][0] * h[0];
#pragma unroll
            for (int j = 1; j < NC; ++j) cmac(t[i], u[i][j], h[j]);
          } else {
            t[i] = cmul_cj(u[0][i], h[0]);
#pragma unroll
            for (int j = 1; j < NC; ++j) cmac_cj(t[i], u[j][i], h[j]);
          }
        }
        recon3<R, NC>(mu, s3, t, acc[0], acc[1]);
        continue;
      }
      if (G5IN) {
#pragma unroll
        for (int k = (NS / 2) * NC; k < NS * NC; ++k) psi[k] = -psi[k];
      }
      const R sgn = fwd ? R(1) : R(-1);
#pragma unroll
      for (int a = 0; a < NS / 2; ++a) {
        const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
        cx<R> h[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) h[c] = psi[a * NC + c] - sgn * mul_phase(ph, psi[jb * NC + c]);
        // lower row factor: -s conj(g_a)
        const int lph = fwd ? phase_neg(phase_conj(ph)) : phase_conj(ph);
#pragma unroll
        for (int i = 0; i < NC; ++i) {
          cx<R> t;
          if (fwd) {
            t = u[i][0] * h[0];
#pragma unroll
            for (int j = 1; j < NC; ++j) cmac(t, u[i][j], h[j]);
          } else {
            t = cmul_cj(u[0][i], h[0]);
#pragma unroll
            for (int j = 1; j < NC; ++j) cmac_cj(t, u[j][i], h[j]);
          }
          acc[a][i] += t;
          acc[jb][i] += mul_phase(lph, t);
        }
      }
    }
  }
}

// Register-tiled hop: one thread, one site, R right-hand sides rhs0..rhs0+R-1.
// The link of each direction is loaded and decompressed once and reused for
// the R spinors; the half-spinor projection is formed from the raw stored
// values and scaled once by the neighbour's norm.  act[r] == 0 skips rhs r
// (uniform across a block, since the rhs tile is blockIdx.y).
template <int ND, int NC, int SP, int GP, bool COMP, bool G5IN, int R>
LYM_D void hop_tile(const EoGeom& g, const HopGauge& hg, const EoField& in, int rhs0, int cb, int par,
                    const int (&act)[R], cx<typename Prec<SP>::real> (&acc)[R][Gamma<ND>::NS][NC]) {
  using RT = typename Prec<SP>::real;
  using GR = typename GPrec<GP>::real;
  constexpr int NS = Gamma<ND>::NS;
  const int vh = (int)g.Vh;
  const int* nb = g.nbr + par * 2 * ND * vh + cb;
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[r][a][c] = czero<RT>();
#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int code = __ldg(nb + (2 * mu + dir) * vh);
      const int ncb = code & 0x7fffffff;
      cx<GR> ug[NC][NC];
      load_link_eo<GP, NC, COMP>(hg.data, hg.nunits, g.Vh, mu, fwd ? par : 1 - par, fwd ? cb : ncb, ug);
      cx<RT> u[NC][NC];
#pragma unroll
      for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) u[i][j] = {(RT)ug[i][j].re, (RT)ug[i][j].im};
      if (COMP && mu == ND - 1 && (code & kNbrBoundary)) {
        const cx<RT> bc{(RT)hg.bcr, (RT)hg.bci};
#pragma unroll
        for (int i = 0; i < NC; ++i)
#pragma unroll
          for (int j = 0; j < NC; ++j) u[i][j] = bc * u[i][j];
      }
      const RT sgn = fwd ? RT(1) : RT(-1);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!act[r]) continue;
        cx<RT> psi[NS * NC];
        const float nrm = load_sp_raw<SP, NS * NC>(in, rhs0 + r, ncb, psi);
        if constexpr (ND == 3) {
          // two-component spinors: G5IN selects the adjoint hop (gamma -> -gamma)
          const int s3 = (fwd != G5IN) ? 1 : -1;
          cx<RT> p0[NC], p1[NC], h[NC], t[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            p0[c] = psi[c];
            p1[c] = psi[NC + c];
          }
          proj3<RT, NC>(mu, s3, p0, p1, h);
          if constexpr (SP == SP16 || SP == SPB16) {
#pragma unroll
            for (int c = 0; c < NC; ++c) h[c] = (RT)nrm * h[c];
          }
#pragma unroll
          for (int i = 0; i < NC; ++i) {
            if (fwd) {
              t[i] = u[i][0] * h[0];
#pragma unroll
              for (int j = 1; j < NC; ++j) cmac(t[i], u[i][j], h[j]);
            } else {
              t[i] = cmul_cj(u[0][i], h[0]);
#pragma unroll
              for (int j = 1; j < NC; ++j) cmac_cj(t[i], u[j][i], h[j]);
            }
          }
          recon3<RT, NC>(mu, s3, t, acc[r][0], acc[r][1]);
          continue;
        }
#pragma unroll
        for (int a = 0; a < NS / 2; ++a) {
          const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
          // G5IN flips the lower component psi_{jb} before projecting
          const RT s2 = G5IN ? -sgn : sgn;
          cx<RT> h[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            h[c] = psi[a * NC + c] - s2 * mul_phase(ph, psi[jb * NC + c]);
            if constexpr (SP == SP16 || SP == SPB16) h[c] = (RT)nrm * h[c];
          }
          const int lph = fwd ? phase_neg(phase_conj(ph)) : phase_conj(ph);
#pragma unroll
          for (int i = 0; i < NC; ++i) {
            cx<RT> t;
            if (fwd) {
              t = u[i][0] * h[0];
#pragma unroll
              for (int j = 1; j < NC; ++j) cmac(t, u[i][j], h[j]);
            } else {
              t = cmul_cj(u[0][i], h[0]);
#pragma unroll
              for (int j = 1; j < NC; ++j) cmac_cj(t, u[j][i], h[j]);
            }
            acc[r][a][i] += t;
            acc[r][jb][i] += mul_phase(lph, t);
          }
        }
      }
    }
  }
}

// raw spinor units of one site (values as stored) and its norm (1 for FP32)
template <int SP, int NCOMP>
LYM_D float load_sp_units(const EoField& f, int rhs, int cb,
                          typename Prec<SP>::unit (&u)[units_for(NCOMP, Prec<SP>::CPU)]) {
  using U = typename Prec<SP>::unit;
  const int vh = (int)f.Vh;
  const U* base = reinterpret_cast<const U*>(f.data) + (size_t)rhs * f.nunits * f.Vh;
#pragma unroll
  for (int k = 0; k < units_for(NCOMP, Prec<SP>::CPU); ++k) u[k] = __ldg(base + k * vh + cb);
  if constexpr (SP == SP16 || SP == SPB16) return __ldg(f.norm + (size_t)rhs * f.Vh + cb);
  return 1.0f;
}

// --- FP16 hop in mixed precision --------------------------------------------
// For FP16 spinors and FP16 full links.  The half spinor h = psi_a + k psi_jb
// (k = +-1, +-i) is formed in packed FP16 (one __hadd2 / __hfma2 per complex, the
// factors +-1 exact), and U h accumulates in FP32 through the sm_100 mixed-
// precision FMA fma.rn.f32.f16 (f16 x f16 + f32; the product of two halves is
// exact in FP32).  No value is converted to FP32 on its own, which takes the
// conversions off the FMA-heavy pipe that bounds the FP32-arithmetic hop.  The
// only extra rounding against hop_tile is h's to FP16 (2^-11 relative, the
// storage precision).  The neighbour's norm scales the FP32 result.
LYM_D float fma_hh(__half a, __half b, float c) {
  float d;
  asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"(__half_as_ushort(a)), "h"(__half_as_ushort(b)), "f"(c));
  return d;
}
LYM_D __half2 as_h2(unsigned w) { return *reinterpret_cast<__half2*>(&w); }

// a + k b for the unit phase k (0:+1, 1:+i, 2:-1, 3:-i), (re, im) half2 pairs
LYM_D __half2 proj_h2(__half2 a, __half2 b, int k) {
  switch (k & 3) {
    case 0: return __hadd2(a, b);
    case 2: return __hsub2(a, b);
    case 1: return __hfma2(__lowhigh2highlow(b), __halves2half2(__float2half_rn(-1.f), __float2half_rn(1.f)), a);
    default: return __hfma2(__lowhigh2highlow(b), __halves2half2(__float2half_rn(1.f), __float2half_rn(-1.f)), a);
  }
}

// acc += s k t for the unit phase k and the real scale s (ns = -s)
LYM_D void acc_phase(cx<float>& acc, int k, float s, float ns, float tr, float ti) {
  switch (k & 3) {
    case 0: acc.re = fmaf(s, tr, acc.re); acc.im = fmaf(s, ti, acc.im); break;
    case 1: acc.re = fmaf(ns, ti, acc.re); acc.im = fmaf(s, tr, acc.im); break;
    case 2: acc.re = fmaf(ns, tr, acc.re); acc.im = fmaf(ns, ti, acc.im); break;
    default: acc.re = fmaf(s, ti, acc.re); acc.im = fmaf(ns, tr, acc.im); break;
  }
}

// Same result per site as hop_tile<ND, NC, SP16, SP16, false, G5IN, R> up to
// the rounding of h; R right-hand sides share each link.  ARITH: the neighbours'
// checkerboard indices come from the site's coordinates instead of the neighbour
// table (no dependent index load per direction; measured faster at 32^4, not at 16^4).
// TSH (with ARITH): the +t and -t neighbours' spinors come from the input field at the
// site's own checkerboard index, loaded once, and from the neighbouring lane of the same
// t row by a warp shuffle -- one coalesced load instead of two gathers.  The output site
// at t = 2 th + o (o = its row's parity offset) has its -t (o = 1) or +t (o = 0)
// neighbour at its own index th and the other one at th -+ 1 (periodic in the row).
// Needs every warp full and the rows of Lh = Lt/2 sites aligned to warps: Lh a power of
// two <= 32 and Vh a multiple of 32 (the host registers the form only then).
template <int ND, int NC, bool G5IN, int R, bool ARITH = false, bool TSH = false>
LYM_D void hop_tile_mx(const EoGeom& g, const HopGauge& hg, const EoField& in, int rhs0, int cb, int par,
                       const int (&act)[R], cx<float> (&acc)[R][Gamma<ND>::NS][NC]) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC, NU = units_for(NCOMP, 4);
  constexpr int NCX = NC * NC, NLU = units_for(NCX, 2);
  const int vh = (int)g.Vh;
  const int* nb = g.nbr + par * 2 * ND * vh + cb;
  static_assert(!TSH || ARITH, "the t-shuffle form takes the coordinates of the arithmetic form");
  int xc[ND];
  int lex = 0;
  if constexpr (ARITH) lex = eo_coords<ND>(g, cb, par, xc);
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[r][a][c] = czero<float>();
  const __half2 conj_f = __halves2half2(__float2half_rn(1.f), __float2half_rn(-1.f));
  const __half2 negre_f = __halves2half2(__float2half_rn(-1.f), __float2half_rn(1.f));
  // t direction by shuffle: the input spinors at the own index, the lanes holding the
  // row neighbours, and this site's row parity offset
  uint4 own[R][NU];
  float own_n[R];
  int srcf = 0, srcb = 0, lhm = 0;
  bool odd = false;
  if constexpr (TSH) {
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (act[r]) own_n[r] = load_sp_units<SP16, NCOMP>(in, rhs0 + r, cb, own[r]);
    const int lane = (int)(threadIdx.x & 31u);
    lhm = g.Lh - 1;
    const int seg = lane & ~lhm;
    srcf = seg | ((lane + 1) & lhm);
    srcb = seg | ((lane - 1) & lhm);
    odd = (xc[ND - 1] & 1) != 0;
  }
  // with TSH the t direction (mu = ND - 1) goes first, so the own-index loads die early
#pragma unroll
  for (int m = 0; m < ND; ++m) {
    const int mu = TSH ? (m == 0 ? ND - 1 : m - 1) : m;
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const bool tsh = TSH && mu == ND - 1;
      int ncb;
      if constexpr (TSH) {
        if (tsh)  // the -t neighbour's index (its link is read there); +t: not needed
          ncb = (cb & ~lhm) | ((cb - (odd ? 0 : 1)) & lhm);
        else
          ncb = (fwd ? nb_fwd<ND>(g, lex, xc, mu) : nb_bwd<ND>(g, lex, xc, mu)) >> 1;
      } else if constexpr (ARITH) {
        ncb = (fwd ? nb_fwd<ND>(g, lex, xc, mu) : nb_bwd<ND>(g, lex, xc, mu)) >> 1;
      } else {
        ncb = __ldg(nb + (2 * mu + dir) * vh) & 0x7fffffff;
      }
      // full N x N link, boundary factor folded in; forward link on x (parity
      // par), backward link on x - mu (parity 1-par)
      const uint2* lp = reinterpret_cast<const uint2*>(hg.data) +
                        (size_t)((mu * 2 + (fwd ? par : 1 - par)) * hg.nunits) * vh + (fwd ? cb : ncb);
      __half2 u[NCX];
#pragma unroll
      for (int k = 0; k < NLU; ++k) {
        const uint2 t = __ldg(lp + k * vh);
        u[2 * k] = as_h2(t.x);
        if (2 * k + 1 < NCX) u[2 * k + 1] = as_h2(t.y);
      }
      const bool s2pos = fwd != G5IN;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!act[r]) continue;
        uint4 raw[NU];
        float nrm;
        if (tsh) {
          // every lane of the warp takes part (act is uniform over the block)
          const int src = fwd ? srcf : srcb;
          const bool mine = fwd ? !odd : odd;
#pragma unroll
          for (int k = 0; k < NU; ++k) {
            uint4 t;
            t.x = __shfl_sync(0xffffffffu, own[r][k].x, src);
            t.y = __shfl_sync(0xffffffffu, own[r][k].y, src);
            t.z = __shfl_sync(0xffffffffu, own[r][k].z, src);
            t.w = __shfl_sync(0xffffffffu, own[r][k].w, src);
            raw[k] = mine ? own[r][k] : t;
          }
          const float tn = __shfl_sync(0xffffffffu, own_n[r], src);
          nrm = mine ? own_n[r] : tn;
        } else {
          nrm = load_sp_units<SP16, NCOMP>(in, rhs0 + r, ncb, raw);
        }
        const float nnrm = -nrm;
        __half2 psi[NCOMP];
#pragma unroll
        for (int k = 0; k < NU; ++k) {
          const unsigned w[4] = {raw[k].x, raw[k].y, raw[k].z, raw[k].w};
#pragma unroll
          for (int m = 0; m < 4; ++m)
            if (4 * k + m < NCOMP) psi[4 * k + m] = as_h2(w[m]);
        }
#pragma unroll
        for (int a = 0; a < NS / 2; ++a) {
          const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
          // h = psi_a - s2 g_a psi_jb
          const int kph = s2pos ? phase_neg(ph) : ph;
          __half2 h[NC], hx[NC];  // hx: forward (re, -im), backward (-re, im)
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            h[c] = proj_h2(psi[a * NC + c], psi[jb * NC + c], kph);
            hx[c] = __hmul2(h[c], fwd ? conj_f : negre_f);
          }
          // lower row factor: -s conj(g_a)
          const int lph = fwd ? phase_neg(phase_conj(ph)) : phase_conj(ph);
#pragma unroll
          for (int i = 0; i < NC; ++i) {
            float tr = 0.f, ti = 0.f;
#pragma unroll
            for (int j = 0; j < NC; ++j) {
              const __half2 uu = fwd ? u[i * NC + j] : u[j * NC + i];
              const __half ure = __low2half(uu), uim = __high2half(uu);
              if (fwd) {  // U h: (u.re h.re - u.im h.im, u.re h.im + u.im h.re)
                tr = fma_hh(ure, __low2half(h[j]), tr);
                tr = fma_hh(uim, __high2half(hx[j]), tr);
                ti = fma_hh(ure, __high2half(h[j]), ti);
                ti = fma_hh(uim, __low2half(h[j]), ti);
              } else {  // U^dag h: (u.re h.re + u.im h.im, u.re h.im - u.im h.re)
                tr = fma_hh(ure, __low2half(h[j]), tr);
                tr = fma_hh(uim, __high2half(h[j]), tr);
                ti = fma_hh(ure, __high2half(h[j]), ti);
                ti = fma_hh(uim, __low2half(hx[j]), ti);
              }
            }
            acc_phase(acc[r][a][i], 0, nrm, nnrm, tr, ti);
            acc_phase(acc[r][jb][i], lph, nrm, nnrm, tr, ti);
          }
        }
      }
    }
  }
}

// --- FP16 hop with packed half arithmetic ---------------------------------------
// As hop_tile_mx, but the colour contraction t = U h of each direction runs on packed
// FP16 pairs: t = sum_j (u_re, u_re) * (h_re, h_im) + (u_im, u_im) * hs_j with
// hs = (-h_im, h_re) for U and (h_im, -h_re) for U^dag, two fused half FMAs per
// complex term (__hfma2, one rounding each) and no value converted on its own.  Each
// t (at most |U| |h| <= 6 in magnitude: links unitary, stored spinors scaled to
// |component| <= 1) is converted to FP32 once and accumulated over the directions in
// FP32 with the neighbour's norm, as in hop_tile_mx.  Against hop_tile_mx the added
// rounding is that of the three-term sums (about 2^-11 relative each).
template <int ND, int NC, bool G5IN, int R>
LYM_D void hop_tile_h2(const EoGeom& g, const HopGauge& hg, const EoField& in, int rhs0, int cb, int par,
                       const int (&act)[R], cx<float> (&acc)[R][Gamma<ND>::NS][NC]) {
  constexpr int NS = Gamma<ND>::NS, NCOMP = NS * NC, NU = units_for(NCOMP, 4);
  constexpr int NCX = NC * NC, NLU = units_for(NCX, 2);
  const int vh = (int)g.Vh;
  const int* nb = g.nbr + par * 2 * ND * vh + cb;
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[r][a][c] = czero<float>();
  // hs = swap(h) * (-1, 1) for U, swap(h) * (1, -1) for U^dag
  const __half2 sw_f = __halves2half2(__float2half_rn(-1.f), __float2half_rn(1.f));
  const __half2 sw_b = __halves2half2(__float2half_rn(1.f), __float2half_rn(-1.f));
#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int code = __ldg(nb + (2 * mu + dir) * vh);
      const int ncb = code & 0x7fffffff;
      const uint2* lp = reinterpret_cast<const uint2*>(hg.data) +
                        (size_t)((mu * 2 + (fwd ? par : 1 - par)) * hg.nunits) * vh + (fwd ? cb : ncb);
      __half2 u[NCX];
#pragma unroll
      for (int k = 0; k < NLU; ++k) {
        const uint2 t = __ldg(lp + k * vh);
        u[2 * k] = as_h2(t.x);
        if (2 * k + 1 < NCX) u[2 * k + 1] = as_h2(t.y);
      }
      const bool s2pos = fwd != G5IN;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!act[r]) continue;
        uint4 raw[NU];
        const float nrm = load_sp_units<SP16, NCOMP>(in, rhs0 + r, ncb, raw);
        const float nnrm = -nrm;
        __half2 psi[NCOMP];
#pragma unroll
        for (int k = 0; k < NU; ++k) {
          const unsigned w[4] = {raw[k].x, raw[k].y, raw[k].z, raw[k].w};
#pragma unroll
          for (int m = 0; m < 4; ++m)
            if (4 * k + m < NCOMP) psi[4 * k + m] = as_h2(w[m]);
        }
#pragma unroll
        for (int a = 0; a < NS / 2; ++a) {
          const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
          const int kph = s2pos ? phase_neg(ph) : ph;
          __half2 h[NC], hs[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            h[c] = proj_h2(psi[a * NC + c], psi[jb * NC + c], kph);
            hs[c] = __hmul2(__lowhigh2highlow(h[c]), fwd ? sw_f : sw_b);
          }
          const int lph = fwd ? phase_neg(phase_conj(ph)) : phase_conj(ph);
#pragma unroll
          for (int i = 0; i < NC; ++i) {
            __half2 t = __float2half2_rn(0.f);
#pragma unroll
            for (int j = 0; j < NC; ++j) {
              const __half2 uu = fwd ? u[i * NC + j] : u[j * NC + i];
              t = __hfma2(__low2half2(uu), h[j], t);
              t = __hfma2(__high2half2(uu), hs[j], t);
            }
            const float2 tf = __half22float2(t);
            acc_phase(acc[r][a][i], 0, nrm, nnrm, tf.x, tf.y);
            acc_phase(acc[r][jb][i], lph, nrm, nnrm, tf.x, tf.y);
          }
        }
      }
    }
  }
}

// The hop of the solver kernels for R right-hand sides at one site: FP32
// arithmetic (MX = 0, hop_tile), or for FP16 spinors with full links the
// mixed-precision form (MX = 1: f16 x f16 + f32 FMAs, hop_tile_mx; MX = 4: the same
// with neighbour indices from coordinate arithmetic; MX = 5: that with the t direction
// by warp shuffle) or the packed-half form (MX = 3: half2 FMAs within a direction,
// hop_tile_h2).
template <int ND, int NC, int SP, int GP, bool COMP, bool G5IN, int R, int MX>
LYM_D void hop_any(const EoGeom& g, const HopGauge& hg, const EoField& in, int rhs0, int cb, int par,
                   const int (&act)[R], cx<typename Prec<SP>::real> (&acc)[R][Gamma<ND>::NS][NC]) {
  if constexpr (MX != 0) {
    static_assert(SP == SP16 && GP == SP16 && !COMP, "the mixed-precision hop takes FP16 spinors and full links");
    static_assert(ND != 3, "the mixed-precision hop has no three-dimensional form");
    if constexpr (MX == 3)
      hop_tile_h2<ND, NC, G5IN, R>(g, hg, in, rhs0, cb, par, act, acc);
    else
      hop_tile_mx<ND, NC, G5IN, R, MX == 4 || MX == 5, MX == 5>(g, hg, in, rhs0, cb, par, act, acc);
  } else {
    hop_tile<ND, NC, SP, GP, COMP, G5IN, R>(g, hg, in, rhs0, cb, par, act, acc);
  }
}

}  // namespace lym
