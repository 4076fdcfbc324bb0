// Adjoint-representation Wilson fermions: operator, adjoint links and fermion
// force (reference dirac.py:358-370, 380-456, 525-565; lie_generators.py).
//
// Spinors are matrix valued, (ns, N, N, V) complex128 planes in the reference
// layout; the adjoint links are (nd, N^2-1, N^2-1, V).  The generator basis is
// the reference's (lie_generators.py:3-17, T^a = lambda^a / 2 in its order), so
// lym_adjoint_links reproduces the reference's fermion_gauge_field entry by
// entry; the force does not depend on the basis.
#include <cmath>

#include "lym_internal.cuh"
#include "lym_su.cuh"

namespace lym {

namespace {

constexpr int kAdjBlock = 128;

// fundamental generator a, element (i, j), in the reference's basis and order
template <int NC>
LYM_D cx<double> gen(int a, int i, int j);

template <>
LYM_D cx<double> gen<2>(int a, int i, int j) {
  // Pauli / 2: sigma_x, sigma_y, sigma_z
  if (a == 0) return {(i != j) ? 0.5 : 0.0, 0.0};
  if (a == 1) return {0.0, (i == 0 && j == 1) ? -0.5 : ((i == 1 && j == 0) ? 0.5 : 0.0)};
  return {(i == j) ? (i == 0 ? 0.5 : -0.5) : 0.0, 0.0};
}

template <>
LYM_D cx<double> gen<3>(int a, int i, int j) {
  // lambda_1, lambda_4, lambda_6, lambda_2, lambda_5, lambda_7, lambda_3, lambda_8 (each / 2)
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  if (a < 6) {
    const int pi = (a % 3 == 0) ? 0 : ((a % 3 == 1) ? 0 : 1);
    const int pj = (a % 3 == 0) ? 1 : ((a % 3 == 1) ? 2 : 2);
    if (lo != pi || hi != pj) return {0.0, 0.0};
    if (a < 3) return {0.5, 0.0};
    return {0.0, i < j ? -0.5 : 0.5};
  }
  if (i != j) return {0.0, 0.0};
  if (a == 6) return {i == 0 ? 0.5 : (i == 1 ? -0.5 : 0.0), 0.0};
  const double s3 = 0.5 / sqrt(3.0);
  return {i == 2 ? -2.0 * s3 : s3, 0.0};
}

// The block's copies of the generators and of the adjoint generators
// (T_adj^k)_{ij} = -2 Tr([T_k, T_i] T_j) (lie_generators.py:22-36), built once
// per block in shared memory.
template <int NC>
struct AdjTables {
  static constexpr int A = NC * NC - 1;
  cx<double> T[A][NC][NC];
  cx<double> TA[A][A][A];
};

template <int NC>
LYM_D void build_tables(AdjTables<NC>& tb) {
  constexpr int A = NC * NC - 1;
  for (int e = threadIdx.x; e < A * NC * NC; e += blockDim.x) {
    const int a = e / (NC * NC), i = (e / NC) % NC, j = e % NC;
    tb.T[a][i][j] = gen<NC>(a, i, j);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < A * A * A; e += blockDim.x) {
    const int k = e / (A * A), i = (e / A) % A, j = e % A;
    // Tr([T_k, T_i] T_j) = sum_{p,q,r} (T_k[p][q] T_i[q][r] - T_i[p][q] T_k[q][r]) T_j[r][p]
    cx<double> t = czero<double>();
    for (int p = 0; p < NC; ++p)
      for (int q = 0; q < NC; ++q)
        for (int r = 0; r < NC; ++r) {
          const cx<double> c = tb.T[k][p][q] * tb.T[i][q][r] - tb.T[i][p][q] * tb.T[k][q][r];
          t += c * tb.T[j][r][p];
        }
    tb.TA[k][i][j] = -2.0 * t;
  }
  __syncthreads();
}

// (1 -+ gamma_mu), times gamma_d when hermitian (dirac.py:310-320), element (m, n)
template <int ND, bool HERM>
LYM_D cx<double> projector(int mu, double sgn, int m, int n) {
  constexpr int NS = Gamma<ND>::NS;
  cx<double> g = czero<double>();
#pragma unroll
  for (int a = 0; a < NS / 2; ++a) {
    const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
    if (m == a && n == jb) g = mul_phase(ph, cx<double>{1.0, 0.0});
    if (m == jb && n == a) g = mul_phase(phase_conj(ph), cx<double>{1.0, 0.0});
  }
  cx<double> p = {(m == n ? 1.0 : 0.0) - sgn * g.re, -sgn * g.im};
  if (HERM && m >= NS / 2) p = -p;
  return p;
}

LYM_D size_t adj_index(int s, int i, int j, int NC, int64_t V, int64_t x) {
  return ((size_t)(s * NC + i) * NC + j) * V + x;
}

}  // namespace

// ---------------------------------------------------------------------------
// operator: one thread per (site, colour row i, vector)
// ---------------------------------------------------------------------------
template <int ND, int NC, bool HERM>
__global__ void __launch_bounds__(kAdjBlock, 1) wilson_adjoint_kernel(
    const int32_t* __restrict__ tab, int V, int Lt, double kappa, double bcr, double bci,
    const double2* __restrict__ UL, const double2* __restrict__ UR, const double2* __restrict__ in,
    double2* __restrict__ out) {
  constexpr int NS = Gamma<ND>::NS;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (x >= V) return;
  const size_t vec = (size_t)NS * NC * NC * V;
  const double2* psi = in + blockIdx.z * vec;
  double2* res = out + blockIdx.z * vec;
  const cx<double> bc{bcr, bci};
  cx<double> acc[NS][NC];
#pragma unroll
  for (int s = 0; s < NS; ++s)
#pragma unroll
    for (int l = 0; l < NC; ++l) acc[s][l] = czero<double>();

#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int y = tab[(fwd ? 0 : ND) * V + mu * V + x];
      const int site = fwd ? x : y;  // the link's site: x forward, x - mu backward
      const bool boundary = mu == ND - 1 && (fwd ? (x % Lt) == Lt - 1 : (x % Lt) == 0);
      // left factor: row i of L (forward) or of L^dag (backward); right factor R in full
      cx<double> lrow[NC];
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        cx<double> v = fwd ? ld(UL + ((size_t)(mu * NC + i) * NC + j) * V + site)
                           : conj(ld(UL + ((size_t)(mu * NC + j) * NC + i) * V + site));
        if (boundary) v = fwd ? bc * v : conj(bc) * v;
        lrow[j] = v;
      }
      cx<double> r[NC][NC];
#pragma unroll
      for (int p = 0; p < NC; ++p)
#pragma unroll
        for (int q = 0; q < NC; ++q) r[p][q] = ld(UR + ((size_t)(mu * NC + p) * NC + q) * V + site);
      const double sgn = fwd ? 1.0 : -1.0;
#pragma unroll
      for (int a = 0; a < NS / 2; ++a) {
        const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
        // w = lrow . h with h = psi_a - s g_a psi_jb (N x N); then o = w R^dag (forward) or w R
        cx<double> w[NC];
#pragma unroll
        for (int l = 0; l < NC; ++l) w[l] = czero<double>();
#pragma unroll
        for (int j = 0; j < NC; ++j)
#pragma unroll
          for (int l = 0; l < NC; ++l) {
            const cx<double> h = ld(psi + adj_index(a, j, l, NC, V, y)) -
                                 sgn * mul_phase(ph, ld(psi + adj_index(jb, j, l, NC, V, y)));
            cmac(w[l], lrow[j], h);
          }
        const int lph = fwd ? phase_neg(phase_conj(ph)) : phase_conj(ph);
#pragma unroll
        for (int l = 0; l < NC; ++l) {
          cx<double> o = czero<double>();
#pragma unroll
          for (int q = 0; q < NC; ++q) {
            if (fwd) cmac(o, w[q], conj(r[l][q]));  // (w R^dag)_l = sum_q w_q conj(R[l][q])
            else cmac(o, w[q], r[q][l]);            // (w R)_l
          }
          acc[a][l] += o;
          acc[jb][l] += mul_phase(lph, o);
        }
      }
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s)
#pragma unroll
    for (int l = 0; l < NC; ++l) {
      const size_t k = adj_index(s, i, l, NC, V, x);
      cx<double> v = ld(psi + k) + kappa * acc[s][l];
      if (HERM && s >= NS / 2) v = -v;
      st(res + k, v);
    }
}

// ---------------------------------------------------------------------------
// adjoint links V^{ab} = 2 Tr(T_a U T_b U^dag), one thread per (site, mu)
// ---------------------------------------------------------------------------
template <int NC>
__global__ void __launch_bounds__(kAdjBlock) adjoint_links_kernel(int nd, int64_t V, int Lt, double bcr, double bci,
                                                                  const double2* __restrict__ U,
                                                                  double2* __restrict__ out) {
  constexpr int A = NC * NC - 1;
  __shared__ AdjTables<NC> tb;
  build_tables<NC>(tb);
  const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (x >= V) return;
  Mat<NC> u = load_link<NC>(U, mu, x, V);
  const bool boundary = mu == nd - 1 && (x % Lt) == Lt - 1;
  const cx<double> f = boundary ? cx<double>{bcr, bci} : cx<double>{1.0, 0.0};
  for (int b = 0; b < A; ++b) {
    Mat<NC> tbm;
#pragma unroll
    for (int p = 0; p < NC; ++p)
#pragma unroll
      for (int q = 0; q < NC; ++q) tbm.m[p][q] = tb.T[b][p][q];
    const Mat<NC> w = mul_nd(mul(u, tbm), u);  // U T_b U^dag
    for (int a = 0; a < A; ++a) {
      cx<double> t = czero<double>();
#pragma unroll
      for (int p = 0; p < NC; ++p)
#pragma unroll
        for (int q = 0; q < NC; ++q) t += tb.T[a][p][q] * w.m[q][p];
      st(out + ((size_t)(mu * A + a) * A + b) * V + x, f * (2.0 * t));
    }
  }
}

// ---------------------------------------------------------------------------
// fermion force: one thread per (site, mu)
// ---------------------------------------------------------------------------
constexpr int kMaxAdjForceTerms = 32;
struct AdjForceTerms {
  double alpha[kMaxAdjForceTerms];
};

// c_k += w * sum_ij TA[k][i][j] M_ij for L(P, Q) at this link, M_ij =
// sum_m [conj(Pv_m)_i (P+ Z)_{m j} - conj(Z_m)_i (P- Pv)_{m j}], Z_n = V Qv_n
// (the two einsums of dirac.py:547-560 with the adjoint components).
template <int ND, int NC, bool HERM>
LYM_D void adjoint_lie_term(const AdjTables<NC>& tb, int mu, const cx<double> (&Vm)[NC * NC - 1][NC * NC - 1],
                            const cx<double> (&Pv)[Gamma<ND>::NS][NC * NC - 1],
                            const cx<double> (&Qv)[Gamma<ND>::NS][NC * NC - 1], double w, cx<double> (&c)[NC * NC - 1]) {
  constexpr int NS = Gamma<ND>::NS, A = NC * NC - 1;
  cx<double> Z[NS][A], PZ[NS][A], PP[NS][A];
  for (int n = 0; n < NS; ++n)
    for (int a = 0; a < A; ++a) {
      cx<double> t = czero<double>();
      for (int b = 0; b < A; ++b) t += Vm[a][b] * Qv[n][b];
      Z[n][a] = t;
    }
  for (int m = 0; m < NS; ++m)
    for (int a = 0; a < A; ++a) {
      cx<double> zp = czero<double>(), pm = czero<double>();
      for (int n = 0; n < NS; ++n) {
        zp += projector<ND, HERM>(mu, 1.0, m, n) * Z[n][a];
        pm += projector<ND, HERM>(mu, -1.0, m, n) * Pv[n][a];
      }
      PZ[m][a] = zp;
      PP[m][a] = pm;
    }
  for (int i = 0; i < A; ++i)
    for (int j = 0; j < A; ++j) {
      cx<double> mij = czero<double>();
      for (int m = 0; m < NS; ++m) mij += cmul_cj(Pv[m][i], PZ[m][j]) - cmul_cj(Z[m][i], PP[m][j]);
      for (int k = 0; k < A; ++k) c[k] += w * (tb.TA[k][i][j] * mij);
    }
}

template <int ND, int NC, bool HERM>
__global__ void __launch_bounds__(kAdjBlock) adjoint_force_kernel(
    const int32_t* __restrict__ tab, int64_t V, int Lt, double kappa, double bcr, double bci,
    const double2* __restrict__ U, int nterms, AdjForceTerms terms, const double2* __restrict__ X,
    const double2* __restrict__ Y, int symmetric, double scale, double2* __restrict__ force) {
  constexpr int NS = Gamma<ND>::NS, A = NC * NC - 1;
  __shared__ AdjTables<NC> tb;
  build_tables<NC>(tb);
  const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (x >= V) return;
  const int64_t y = tab[mu * V + x];
  // adjoint link of this link, boundary factor on the last time slice
  Mat<NC> u = load_link<NC>(U, mu, x, V);
  const bool boundary = mu == ND - 1 && (x % Lt) == Lt - 1;
  const cx<double> f = boundary ? cx<double>{bcr, bci} : cx<double>{1.0, 0.0};
  cx<double> Vm[A][A];
  for (int b = 0; b < A; ++b) {
    Mat<NC> tbm;
    for (int p = 0; p < NC; ++p)
      for (int q = 0; q < NC; ++q) tbm.m[p][q] = tb.T[b][p][q];
    const Mat<NC> w = mul_nd(mul(u, tbm), u);
    for (int a = 0; a < A; ++a) {
      cx<double> t = czero<double>();
      for (int p = 0; p < NC; ++p)
        for (int q = 0; q < NC; ++q) t += tb.T[a][p][q] * w.m[q][p];
      Vm[a][b] = f * (2.0 * t);
    }
  }
  cx<double> c[A];
  for (int k = 0; k < A; ++k) c[k] = czero<double>();
  const size_t vec = (size_t)NS * NC * NC * V;
  for (int term = 0; term < nterms; ++term) {
    const double2* Xk = X + term * vec;
    const double2* Yk = Y + term * vec;
    // adjoint components 2 Tr(T_a M) of X, Y at x and at x + mu
    cx<double> xv[NS][A], yv[NS][A];
    for (int side = 0; side < (symmetric ? 2 : 1); ++side) {
      const double2* P = side == 0 ? Xk : Yk;  // L(P, Q): P at x, Q at x + mu
      const double2* Q = side == 0 ? Yk : Xk;
      for (int s = 0; s < NS; ++s)
        for (int a = 0; a < A; ++a) {
          cx<double> tp = czero<double>(), tq = czero<double>();
          for (int p = 0; p < NC; ++p)
            for (int q = 0; q < NC; ++q) {
              tp += tb.T[a][p][q] * ld(P + adj_index(s, q, p, NC, V, x));
              tq += tb.T[a][p][q] * ld(Q + adj_index(s, q, p, NC, V, y));
            }
          xv[s][a] = 2.0 * tp;
          yv[s][a] = 2.0 * tq;
        }
      adjoint_lie_term<ND, NC, HERM>(tb, mu, Vm, xv, yv, kappa * terms.alpha[term], c);
    }
  }
  Mat<NC> out = load_link<NC>(force, mu, x, V);
  for (int p = 0; p < NC; ++p)
    for (int q = 0; q < NC; ++q) {
      cx<double> t = czero<double>();
      for (int k = 0; k < A; ++k) t += c[k] * tb.T[k][p][q];
      out.m[p][q] += scale * t;
    }
  store_link<NC>(force, mu, x, V, out);
}

}  // namespace lym

using namespace lym;

extern "C" {

int lym_wilson_apply_adjoint(const lym_lattice* lat, int nc, double kappa, int hermitian, double bc_re,
                             double bc_im, const void* gauge_left, const void* gauge, int nvec, const void* in,
                             void* out, void* stream) {
  LYM_REQUIRE(lat && gauge_left && gauge && in && out, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(in != out, LYM_ERR_BAD_ARG, "in and out must not alias");
  LYM_REQUIRE(nvec >= 1 && nvec <= 65535, LYM_ERR_BAD_ARG, "nvec out of range");
  if (lat->nd != 2 && lat->nd != 4) {
    set_error("Number of dimensions %d not supported for fermions!", lat->nd);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N=%d not supported (2 or 3)", nc);
  dim3 grid(grid_for(lat->V, kAdjBlock), nc, nvec);
  cudaStream_t st = (cudaStream_t)stream;
  const int Lt = lat->dims[lat->nd - 1];
#define LYM_ADJ(ND_, NC_, H_)                                                                              \
  wilson_adjoint_kernel<ND_, NC_, H_><<<grid, kAdjBlock, 0, st>>>(lat->d_tab, (int)lat->V, Lt, kappa, bc_re, \
                                                                  bc_im, (const double2*)gauge_left,       \
                                                                  (const double2*)gauge, (const double2*)in, \
                                                                  (double2*)out)
  if (lat->nd == 2 && nc == 2) { if (hermitian) LYM_ADJ(2, 2, true); else LYM_ADJ(2, 2, false); }
  else if (lat->nd == 2 && nc == 3) { if (hermitian) LYM_ADJ(2, 3, true); else LYM_ADJ(2, 3, false); }
  else if (lat->nd == 4 && nc == 2) { if (hermitian) LYM_ADJ(4, 2, true); else LYM_ADJ(4, 2, false); }
  else { if (hermitian) LYM_ADJ(4, 3, true); else LYM_ADJ(4, 3, false); }
#undef LYM_ADJ
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_adjoint_links(const lym_lattice* lat, int nc, double bc_re, double bc_im, const void* gauge, void* out,
                      void* stream) {
  LYM_REQUIRE(lat && gauge && out, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N=%d not supported (2 or 3)", nc);
  dim3 grid(grid_for(lat->V, kAdjBlock), lat->nd);
  cudaStream_t st = (cudaStream_t)stream;
  const int Lt = lat->dims[lat->nd - 1];
  if (nc == 2)
    adjoint_links_kernel<2><<<grid, kAdjBlock, 0, st>>>(lat->nd, lat->V, Lt, bc_re, bc_im, (const double2*)gauge,
                                                        (double2*)out);
  else
    adjoint_links_kernel<3><<<grid, kAdjBlock, 0, st>>>(lat->nd, lat->V, Lt, bc_re, bc_im, (const double2*)gauge,
                                                        (double2*)out);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_fermion_force_adjoint(const lym_lattice* lat, int nc, double kappa, int hermitian, double bc_re,
                              double bc_im, const void* gauge, int nterms, const double* alphas, const void* X,
                              const void* Y, int symmetric, double scale, void* force, void* stream) {
  LYM_REQUIRE(lat && gauge && alphas && X && Y && force, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nterms >= 1 && nterms <= kMaxAdjForceTerms, LYM_ERR_BAD_ARG, "nterms must be in [1, %d]",
              kMaxAdjForceTerms);
  if (lat->nd != 2 && lat->nd != 4) {
    set_error("Number of dimensions %d not supported for fermions!", lat->nd);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N=%d not supported (2 or 3)", nc);
  AdjForceTerms t;
  for (int i = 0; i < kMaxAdjForceTerms; ++i) t.alpha[i] = i < nterms ? alphas[i] : 0.0;
  dim3 grid(grid_for(lat->V, kAdjBlock), lat->nd);
  cudaStream_t st = (cudaStream_t)stream;
  const int Lt = lat->dims[lat->nd - 1];
#define LYM_AF(ND_, NC_, H_)                                                                            \
  adjoint_force_kernel<ND_, NC_, H_><<<grid, kAdjBlock, 0, st>>>(lat->d_tab, lat->V, Lt, kappa, bc_re,    \
                                                                 bc_im, (const double2*)gauge, nterms, t, \
                                                                 (const double2*)X, (const double2*)Y,    \
                                                                 symmetric, scale, (double2*)force)
  if (lat->nd == 2 && nc == 2) { if (hermitian) LYM_AF(2, 2, true); else LYM_AF(2, 2, false); }
  else if (lat->nd == 2 && nc == 3) { if (hermitian) LYM_AF(2, 3, true); else LYM_AF(2, 3, false); }
  else if (lat->nd == 4 && nc == 2) { if (hermitian) LYM_AF(4, 2, true); else LYM_AF(4, 2, false); }
  else { if (hermitian) LYM_AF(4, 3, true); else LYM_AF(4, 3, false); }
#undef LYM_AF
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// slice sums of the pion correlator (fermion_measurements.py:76-90)
// ---------------------------------------------------------------------------
namespace lym {

// out[2z], out[2z+1] = sum over the vectors and the sites with x_dir = z of
// sum_{spin,colour} conj(S) S (fundamental, (ns, N, V) per vector) or
// sum_{spin,c,d} conj(S_cd) S_dc (adjoint, (ns, N, N, V)); one block per slice,
// fixed-order block reduction (deterministic).
__global__ void __launch_bounds__(256) timeslice_sums_kernel(int64_t V, int64_t stride, int L, int nvec, int ns,
                                                             int nc, int adjoint, const double2* __restrict__ in,
                                                             double* __restrict__ out) {
  __shared__ double sh[2 * 32];
  const int z = blockIdx.x;
  const int64_t per = V / L;
  const int ncomp = adjoint ? nc * nc : nc;
  const int64_t vec = (int64_t)ns * ncomp * V;
  double re = 0.0, im = 0.0;
  for (int64_t j = threadIdx.x; j < per; j += blockDim.x) {
    const int64_t x = (j / stride) * (L * stride) + (int64_t)z * stride + (j % stride);
    for (int v = 0; v < nvec; ++v)
      for (int s = 0; s < ns; ++s) {
        const double2* base = in + v * vec + (int64_t)s * ncomp * V;
        if (!adjoint) {
          for (int c = 0; c < nc; ++c) {
            const cx<double> a = ld(base + (int64_t)c * V + x);
            re += a.re * a.re + a.im * a.im;
          }
        } else {
          for (int c = 0; c < nc; ++c)
            for (int d = 0; d < nc; ++d) {
              const cx<double> a = ld(base + (int64_t)(c * nc + d) * V + x);
              const cx<double> b = ld(base + (int64_t)(d * nc + c) * V + x);
              const cx<double> t = cmul_cj(a, b);
              re += t.re;
              im += t.im;
            }
        }
      }
  }
  double v2[2] = {re, im};
  block_sum<2>(v2, sh);
  if (threadIdx.x == 0) {
    out[2 * z] = v2[0];
    out[2 * z + 1] = v2[1];
  }
}

}  // namespace lym

extern "C" int lym_timeslice_sums(const lym_lattice* lat, int direction, int nvec, int ns, int nc, int adjoint,
                                  const void* in, double* out, void* stream) {
  using namespace lym;
  LYM_REQUIRE(lat && in && out, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(direction >= 0 && direction < lat->nd, LYM_ERR_BAD_ARG, "direction %d out of range", direction);
  LYM_REQUIRE(nvec >= 1 && ns >= 1 && nc >= 1, LYM_ERR_BAD_ARG, "bad sizes");
  int64_t stride = 1;
  for (int d = direction + 1; d < lat->nd; ++d) stride *= lat->dims[d];
  const int L = lat->dims[direction];
  timeslice_sums_kernel<<<L, 256, 0, (cudaStream_t)stream>>>(lat->V, stride, L, nvec, ns, nc, adjoint != 0,
                                                            (const double2*)in, out);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}
