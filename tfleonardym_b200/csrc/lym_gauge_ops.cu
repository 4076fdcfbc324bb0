// Gauge-side kernels in the reference layout (FP64): staples and gauge force
// (fused with the momentum update), plaquette and momenta energy reductions,
// the link update exp(eps P) U, polar reunitarisation and the fused per-link
// fermion force.  One thread per link (site, direction); every neighbour link
// is read straight from the gauge field through the reference's sup/sdn
// tables -- no shifted copies are materialised (gauge_action.py:56-91 builds
// five gathered copies per plane instead).
#include "lym_internal.cuh"
#include "lym_kernels.cuh"
#include "lym_su.cuh"

#include <mutex>

namespace lym {

// ---------------------------------------------------------------------------
// staples: S_mu(x) = sum_{nu != mu} U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
//                               + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
// (gauge_action.py:56-101, staples.py:13-58)
// ---------------------------------------------------------------------------
template <int ND, int NC>
LYM_D Mat<NC> staple_sum(const int32_t* __restrict__ tab, int64_t V, const double2* __restrict__ U, int mu,
                         int64_t s, int no_dir) {
  Mat<NC> S = mzero<NC>();
#pragma unroll
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == mu || nu == no_dir) continue;
    const int64_t xmu = tab[mu * V + s];
    const int64_t xnu = tab[nu * V + s];
    const int64_t xmnu = tab[ND * V + nu * V + s];
    const int64_t xmnu_pmu = tab[mu * V + xmnu];
    Mat<NC> a = mul(load_link<NC>(U, nu, s, V), load_link<NC>(U, mu, xnu, V));
    madd(S, mul_nd(a, load_link<NC>(U, nu, xmu, V)));
    Mat<NC> b = mul_dn(load_link<NC>(U, nu, xmnu, V), load_link<NC>(U, mu, xmnu, V));
    madd(S, mul(b, load_link<NC>(U, nu, xmnu_pmu, V)));
  }
  return S;
}

template <int ND, int NC>
__global__ void __launch_bounds__(128) staples_kernel(const int32_t* __restrict__ tab, int64_t V,
                                                      const double2* __restrict__ U, int no_dir,
                                                      double2* __restrict__ out) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= V) return;
  Mat<NC> S = (mu == no_dir) ? mzero<NC>() : staple_sum<ND, NC>(tab, V, U, mu, s, no_dir);
  store_link<NC>(out, mu, s, V, S);
}

// The per-plane staple terms themselves, in the reference's list order
// (staples.py:23-58): for direction mu, the planes (mu, nu) with nu != mu,
// no_dir in increasing nu, each giving the "up" term U_nu(x) U_mu(x+nu)
// U_nu(x+mu)^dag (sup_staple_trace) then the "down" term U_nu(x-nu)^dag
// U_mu(x-nu) U_nu(x-nu+mu) (sdn_staple_trace).  out is (nd, 2(nd-1), N, N, V);
// slot 2k / 2k+1 holds plane k's terms; the slots of an excluded direction and
// the last two slots of the others when no_dir is a direction are left as they are.
template <int ND, int NC>
__global__ void __launch_bounds__(128) staple_terms_kernel(const int32_t* __restrict__ tab, int64_t V,
                                                           const double2* __restrict__ U, int no_dir,
                                                           double2* __restrict__ out) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= V || mu == no_dir) return;
  constexpr int NT = 2 * (ND - 1);
  const int64_t xmu = tab[mu * V + s];
  int k = 0;
#pragma unroll
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == mu || nu == no_dir) continue;
    const int64_t xnu = tab[nu * V + s];
    const int64_t xmnu = tab[ND * V + nu * V + s];
    const int64_t xmnu_pmu = tab[mu * V + xmnu];
    const Mat<NC> up = mul_nd(mul(load_link<NC>(U, nu, s, V), load_link<NC>(U, mu, xnu, V)),
                              load_link<NC>(U, nu, xmu, V));
    const Mat<NC> dn = mul(mul_dn(load_link<NC>(U, nu, xmnu, V), load_link<NC>(U, mu, xmnu, V)),
                           load_link<NC>(U, nu, xmnu_pmu, V));
    store_link<NC>(out, mu * NT + 2 * k, s, V, up);
    store_link<NC>(out, mu * NT + 2 * k + 1, s, V, dn);
    ++k;
  }
}

// F = -beta/(4N) (W^dag - W) - trace/N, W = U S^dag at one link (gauge_action.py:42-53)
template <int ND, int NC>
LYM_D Mat<NC> gauge_force_link(const int32_t* __restrict__ tab, int64_t V, const double2* __restrict__ U,
                               double beta, int mu, int64_t s) {
  Mat<NC> S = staple_sum<ND, NC>(tab, V, U, mu, s, -1);
  Mat<NC> W = mul_nd(load_link<NC>(U, mu, s, V), S);
  const double c = -0.25 * beta / NC;
  Mat<NC> F;
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) F.m[i][j] = c * (conj(W.m[j][i]) - W.m[i][j]);
  cx<double> tr = trace(F);
  tr = (1.0 / NC) * tr;
#pragma unroll
  for (int i = 0; i < NC; ++i) F.m[i][i] -= tr;
  return F;
}

// F = -beta/(4N) (W^dag - W) - trace/N, W = U S^dag (gauge_action.py:42-53).
// With mom != null: mom += eps F instead of storing F (hmc.py:59-61).
template <int ND, int NC>
__global__ void __launch_bounds__(128) gauge_force_kernel(const int32_t* __restrict__ tab, int64_t V,
                                                          const double2* __restrict__ U, double beta,
                                                          double2* __restrict__ force, double2* __restrict__ mom,
                                                          double eps) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= V) return;
  Mat<NC> S = staple_sum<ND, NC>(tab, V, U, mu, s, -1);
  Mat<NC> W = mul_nd(load_link<NC>(U, mu, s, V), S);
  const double c = -0.25 * beta / NC;
  Mat<NC> F;
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) F.m[i][j] = c * (conj(W.m[j][i]) - W.m[i][j]);
  cx<double> tr = trace(F);
  tr = (1.0 / NC) * tr;
#pragma unroll
  for (int i = 0; i < NC; ++i) F.m[i][i] -= tr;
  if (mom) {
    Mat<NC> P = load_link<NC>(mom, mu, s, V);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) P.m[i][j] += eps * F.m[i][j];
    store_link<NC>(mom, mu, s, V, P);
  } else {
    store_link<NC>(force, mu, s, V, F);
  }
}

// sum_{x, mu<nu} Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag (gauge_action.py:110-113)
template <int ND, int NC>
__global__ void __launch_bounds__(256) plaquette_kernel(const int32_t* __restrict__ tab, int64_t V,
                                                        const double2* __restrict__ U, double* partials,
                                                        unsigned* counter, double* result) {
  __shared__ double sh[2 * 32];
  double v[2] = {0.0, 0.0};
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < V; s += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int mu = 0; mu < ND; ++mu)
#pragma unroll
      for (int nu = mu + 1; nu < ND; ++nu) {
        Mat<NC> a = mul(load_link<NC>(U, mu, s, V), load_link<NC>(U, nu, tab[mu * V + s], V));
        Mat<NC> b = mul(load_link<NC>(U, nu, s, V), load_link<NC>(U, mu, tab[nu * V + s], V));
        // Tr(a b^dag)
        cx<double> t = czero<double>();
#pragma unroll
        for (int i = 0; i < NC; ++i)
#pragma unroll
          for (int k = 0; k < NC; ++k) t += a.m[i][k] * conj(b.m[i][k]);
        v[0] += t.re;
        v[1] += t.im;
      }
  }
  if (grid_sum<2>(v, partials, counter, sh) && threadIdx.x == 0) {
    result[0] = v[0];
    result[1] = v[1];
  }
}

// Momenta from unit normals, one thread per link, built as hmc.py:69-96 builds
// them from its draws: normals (nd, N^2-1, V) hold per direction the (re, im)
// pairs of the entries above the diagonal in row order, then the N-1 Cartan
// values; each is halved; P_ij = (re, im), P_ji = (-re, im); the diagonal is
// i times sum_i c_i H_i with the reference's diagonal generators.
template <int NC>
__global__ void __launch_bounds__(256) momenta_from_normals_kernel(int nd, int64_t V, const double* __restrict__ nrm,
                                                                   double2* __restrict__ P) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= V) return;
  constexpr int NG = NC * NC - 1;
  const double* n = nrm + (int64_t)mu * NG * V + s;
  Mat<NC> m;
  int k = 0;
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = i + 1; j < NC; ++j) {
      const double re = 0.5 * n[(int64_t)k * V], im = 0.5 * n[(int64_t)(k + 1) * V];
      k += 2;
      m.m[i][j] = {re, im};
      m.m[j][i] = {-re, im};
    }
  double diag[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) diag[i] = 0.0;
#pragma unroll
  for (int i = 1; i < NC; ++i) {
    const double r = 0.5 * n[(int64_t)k * V];
    ++k;
    const double di = (double)i;
#pragma unroll
    for (int j = 0; j < i; ++j) diag[j] += r / sqrt(di * (di + 1.0) / 2.0);
    diag[i] += -r * (di * sqrt(2.0 / (di * (di + 1.0))));
  }
#pragma unroll
  for (int i = 0; i < NC; ++i) m.m[i][i] = {0.0, diag[i]};
  store_link<NC>(P, mu, s, V, m);
}

// -Re sum Tr P^2 (hmc.py:170-176)
template <int NC>
__global__ void __launch_bounds__(256) momenta_energy_kernel(int64_t nlinks, int64_t V,
                                                             const double2* __restrict__ P, double* partials,
                                                             unsigned* counter, double* result) {
  __shared__ double sh[32];
  double v[1] = {0.0};
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < nlinks; l += (int64_t)gridDim.x * blockDim.x) {
    const int mu = (int)(l / V);
    const int64_t s = l - mu * V;
    Mat<NC> p = load_link<NC>(P, mu, s, V);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) v[0] -= (p.m[i][j] * p.m[j][i]).re;
  }
  if (grid_sum<1>(v, partials, counter, sh) && threadIdx.x == 0) result[0] = v[0];
}

__global__ void axpy_real_kernel(int64_t n, double2* __restrict__ y, const double2* __restrict__ x, double a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 yv = y[i], xv = x[i];
    y[i] = make_double2(yv.x + a * xv.x, yv.y + a * xv.y);
  }
}

// ---------------------------------------------------------------------------
// exp of an anti-Hermitian matrix (the HMC momenta, hmc.py:69-96)
// ---------------------------------------------------------------------------

// sin(w)/w with its series near zero
LYM_D double sinc(double w) {
  if (fabs(w) < 0.05) {
    double w2 = w * w;
    return 1.0 - w2 / 6.0 * (1.0 - w2 / 20.0 * (1.0 - w2 / 42.0 * (1.0 - w2 / 72.0)));
  }
  return sin(w) / w;
}

// exp(X) for 2x2 X = t 1 + X0, X0 traceless: X0^2 = -det(X0) 1 (Cayley-Hamilton),
// so exp(X0) = cos(a) 1 + sinc(a) X0 with a^2 = det(X0) (>= 0 for anti-Hermitian X0).
LYM_D Mat<2> expm(const Mat<2>& X) {
  cx<double> t = 0.5 * trace(X);
  Mat<2> X0 = X;
  X0.m[0][0] -= t;
  X0.m[1][1] -= t;
  double a2 = det(X0).re;
  double a = sqrt(fmax(a2, 0.0));
  double c = cos(a), sc = sinc(a);
  Mat<2> R;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) R.m[i][j] = sc * X0.m[i][j];
  R.m[0][0].re += c;
  R.m[1][1].re += c;
  // exp(t) with t = i phi for anti-Hermitian X (real part kept for generality)
  double e = exp(t.re), sn, cs;
  sincos(t.im, &sn, &cs);
  return mscale(cx<double>{e * cs, e * sn}, R);
}

// exp(X) for 3x3 anti-Hermitian X: X = t 1 + i Q with Q Hermitian traceless,
// exp(i Q) = f0 + f1 Q + f2 Q^2 with the closed-form coefficients of
// Morningstar & Peardon, Phys. Rev. D 69 (2004) 054501, eqs. (23)-(34).
LYM_D Mat<3> expm(const Mat<3>& X) {
  cx<double> t = (1.0 / 3.0) * trace(X);
  Mat<3> Q;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<double> x = X.m[i][j];
      if (i == j) x -= t;
      Q.m[i][j] = {x.im, -x.re};  // -i x
    }
  Mat<3> Q2 = mul(Q, Q);
  const double c1 = 0.5 * trace(Q2).re;
  cx<double> f0, f1, f2;
  if (c1 < 1e-12) {
    // exp(iQ) = 1 + iQ - Q^2/2 + O(|Q|^3) with |Q| < 1e-6
    f0 = {1.0, 0.0};
    f1 = {0.0, 1.0};
    f2 = {-0.5, 0.0};
  } else {
    double c0 = det(Q).re;
    const bool neg = c0 < 0;
    if (neg) c0 = -c0;
    const double c0max = 2.0 * pow(c1 / 3.0, 1.5);
    double ratio = c0 / c0max;
    ratio = fmin(1.0, fmax(-1.0, ratio));
    const double theta = acos(ratio);
    double st3, ct3;
    sincos(theta / 3.0, &st3, &ct3);
    const double u = sqrt(c1 / 3.0) * ct3;
    const double w = sqrt(c1) * st3;
    const double u2 = u * u, w2 = w * w;
    double s2u, c2u, su, cu;
    sincos(2.0 * u, &s2u, &c2u);
    sincos(u, &su, &cu);
    const cx<double> e2iu{c2u, s2u}, emiu{cu, -su};
    const double cw = cos(w), xi0 = sinc(w);
    cx<double> h0 = (u2 - w2) * e2iu + emiu * cx<double>{8.0 * u2 * cw, 2.0 * u * (3.0 * u2 + w2) * xi0};
    cx<double> h1 = (2.0 * u) * e2iu - emiu * cx<double>{2.0 * u * cw, -(3.0 * u2 - w2) * xi0};
    cx<double> h2 = e2iu - emiu * cx<double>{cw, 3.0 * u * xi0};
    const double d = 1.0 / (9.0 * u2 - w2);
    f0 = d * h0;
    f1 = d * h1;
    f2 = d * h2;
    if (neg) {  // f_j(-c0) = (-1)^j conj(f_j(c0))
      f0 = conj(f0);
      f1 = -conj(f1);
      f2 = conj(f2);
    }
  }
  Mat<3> R;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) R.m[i][j] = f1 * Q.m[i][j] + f2 * Q2.m[i][j];
#pragma unroll
  for (int i = 0; i < 3; ++i) R.m[i][i] += f0;
  double e = exp(t.re), sn, cs;
  sincos(t.im, &sn, &cs);
  return mscale(cx<double>{e * cs, e * sn}, R);
}

// Unitary polar factor by the scaled Newton iteration
// U <- (g U + U^{-dag} / g) / 2, g = |det U|^{-1/N} (Higham, "Functions of
// Matrices", sec. 8.6), then division by the principal det^{1/N}
// (smearing.py:17-31 computes X (X^dag X)^{-1/2} / det^{1/N} via sqrtm).
template <int NC>
LYM_D Mat<NC> polar_su(const Mat<NC>& X) {
  Mat<NC> Uk = X;
  for (int it = 0; it < 40; ++it) {
    cx<double> d = det(Uk);
    double g = pow(sqrt(norm2(d)), -1.0 / NC);
    Mat<NC> Z = mdag(inverse(Uk));
    Mat<NC> Un;
    double diff = 0.0;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        Un.m[i][j] = 0.5 * (g * Uk.m[i][j] + (1.0 / g) * Z.m[i][j]);
        diff += norm2(Un.m[i][j] - Uk.m[i][j]);
      }
    Uk = Un;
    if (diff < 1e-30) break;
  }
  cx<double> r = principal_root(det(Uk), NC);
  cx<double> ir = cdiv(cx<double>{1.0, 0.0}, r);
  return mscale(ir, Uk);
}

template <int NC>
__global__ void __launch_bounds__(128) update_links_kernel(int64_t nlinks, int64_t V, double2* __restrict__ U,
                                                           const double2* __restrict__ P, double eps, int reunit) {
  const int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  const int mu = (int)(l / V);
  const int64_t s = l - mu * V;
  Mat<NC> p = load_link<NC>(P, mu, s, V);
  Mat<NC> e = expm(mscale(cx<double>{eps, 0.0}, p));
  Mat<NC> r = mul(e, load_link<NC>(U, mu, s, V));
  if (reunit) r = polar_su<NC>(r);
  store_link<NC>(U, mu, s, V, r);
}

template <int NC>
__global__ void __launch_bounds__(128) unitary_projection_kernel(int64_t nlinks, int64_t V,
                                                                 const double2* __restrict__ in,
                                                                 double2* __restrict__ out) {
  const int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  const int mu = (int)(l / V);
  const int64_t s = l - mu * V;
  store_link<NC>(out, mu, s, V, polar_su<NC>(load_link<NC>(in, mu, s, V)));
}

// ---------------------------------------------------------------------------
// fermion force (dirac.py:525-565, fermion_action.py:64-93)
//
// For link (mu, x), with V_m = U_mu(x) Y_m(x+mu) (colour matvec per spin row m):
//   A = sum_m conj(X_m(x)) (x) (P+ V)_m ,  B = sum_m conj(V_m) (x) (P- X(x))_m
//   L(X, Y)_{ut} = kappa/2 [A_{tu} - B_{tu} - delta_{ut} (Tr A - Tr B)/N]
// which is the reference's sum over generators T^k_{ij} T^k_{ut} written with
// the SU(N) completeness relation sum_k T^k_ij T^k_ut = (d_it d_ju - d_ij d_ut/N)/2.
// P+- = (1 -+ gamma_mu), multiplied by gamma_d when hermitian.
// ---------------------------------------------------------------------------
constexpr int kMaxForceTerms = 64;
struct ForceTerms {
  double alpha[kMaxForceTerms];
};

// (1 - s gamma_mu) v, optionally times gamma_d, for the reference basis
template <int ND, int NC, bool HERM>
LYM_D void project_full(int mu, double sgn, const cx<double> (&v)[Gamma<ND>::NS][NC],
                        cx<double> (&o)[Gamma<ND>::NS][NC]) {
  constexpr int NS = Gamma<ND>::NS;
#pragma unroll
  for (int a = 0; a < NS / 2; ++a) {
    const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      cx<double> up = v[a][c] - sgn * mul_phase(ph, v[jb][c]);
      cx<double> lo = v[jb][c] - sgn * mul_phase(phase_conj(ph), v[a][c]);
      o[a][c] = up;
      o[jb][c] = HERM ? -lo : lo;
    }
  }
}

template <int ND, int NC, bool HERM>
LYM_D void lie_term(int mu, const Mat<NC>& U, const cx<double> (&X)[Gamma<ND>::NS][NC],
                    const cx<double> (&Ysup)[Gamma<ND>::NS][NC], Mat<NC>& A, Mat<NC>& B) {
  constexpr int NS = Gamma<ND>::NS;
  cx<double> Vv[NS][NC], PV[NS][NC], PX[NS][NC];
#pragma unroll
  for (int m = 0; m < NS; ++m)
#pragma unroll
    for (int i = 0; i < NC; ++i) {
      cx<double> t = czero<double>();
#pragma unroll
      for (int l = 0; l < NC; ++l) t += U.m[i][l] * Ysup[m][l];
      Vv[m][i] = t;
    }
  project_full<ND, NC, HERM>(mu, 1.0, Vv, PV);
  project_full<ND, NC, HERM>(mu, -1.0, X, PX);
#pragma unroll
  for (int m = 0; m < NS; ++m)
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        A.m[i][j] += cmul_cj(X[m][i], PV[m][j]);
        B.m[i][j] += cmul_cj(Vv[m][i], PX[m][j]);
      }
}

template <int ND, int NC, bool HERM>
__global__ void __launch_bounds__(128) fermion_force_kernel(
    const int32_t* __restrict__ tab, int64_t V, int Lt, double kappa, double bcr, double bci,
    const double2* __restrict__ U, int nterms, ForceTerms terms, const double2* __restrict__ X,
    const double2* __restrict__ Y, int symmetric, double scale, double2* __restrict__ force) {
  constexpr int NS = Gamma<ND>::NS;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= V) return;
  const int64_t y = tab[mu * V + s];
  Mat<NC> u = load_link<NC>(U, mu, s, V);
  if (mu == ND - 1 && (s % Lt) == Lt - 1) u = mscale(cx<double>{bcr, bci}, u);
  Mat<NC> F = mzero<NC>();
  const int64_t vec = (int64_t)NS * NC * V;
  for (int k = 0; k < nterms; ++k) {
    const double2* Xk = X + k * vec;
    const double2* Yk = Y + k * vec;
    cx<double> xs[NS][NC], ysup[NS][NC];
#pragma unroll
    for (int m = 0; m < NS; ++m)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        xs[m][c] = ld(Xk + (m * NC + c) * V + s);
        ysup[m][c] = ld(Yk + (m * NC + c) * V + y);
      }
    Mat<NC> A = mzero<NC>(), B = mzero<NC>();
    lie_term<ND, NC, HERM>(mu, u, xs, ysup, A, B);
    if (symmetric) {
#pragma unroll
      for (int m = 0; m < NS; ++m)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          xs[m][c] = ld(Yk + (m * NC + c) * V + s);
          ysup[m][c] = ld(Xk + (m * NC + c) * V + y);
        }
      lie_term<ND, NC, HERM>(mu, u, xs, ysup, A, B);
    }
    const double w = 0.5 * kappa * terms.alpha[k];
    cx<double> tr = (1.0 / NC) * (trace(A) - trace(B));
#pragma unroll
    for (int uu = 0; uu < NC; ++uu)
#pragma unroll
      for (int tt = 0; tt < NC; ++tt) {
        cx<double> v = A.m[tt][uu] - B.m[tt][uu];
        if (uu == tt) v -= tr;
        F.m[uu][tt] += w * v;
      }
  }
  Mat<NC> out = load_link<NC>(force, mu, s, V);
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) out.m[i][j] += scale * F.m[i][j];
  store_link<NC>(force, mu, s, V, out);
}

// ---------------------------------------------------------------------------
// The gauge part of an HMC step on many lattices at once (builder-defined: the
// reference runs one lattice per process, hmc.py:218-246): momenta P += eps_p F(U)
// for every link of every lattice in one launch, then U <- exp(eps_u P) U in a
// second (the force reads neighbouring links, so all forces come first).  The
// lattices' descriptors travel as the kernel parameter; every lattice owns a
// contiguous range of blocks (nd x its site blocks) and a block finds its lattice
// by binary search over the range starts.  Any mix of (nd, N) in one launch.
// ---------------------------------------------------------------------------
struct HmcLat {
  const int32_t* tab;
  double2* U;
  double2* P;
  int64_t V;
  double beta;
  int nd, nc;
  int b0;  // first block of this lattice
};
constexpr int kHmcMaxLat = 256;
struct HmcTable {
  int n;
  double eps;
  HmcLat l[kHmcMaxLat];
};

LYM_D int hmc_lat_of(const HmcTable& t, int b) {
  int lo = 0, hi = t.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.l[mid].b0 <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int ND, int NC>
LYM_D void hmc_kick_link(const HmcLat& L, double eps, int mu, int64_t s) {
  const Mat<NC> F = gauge_force_link<ND, NC>(L.tab, L.V, L.U, L.beta, mu, s);
  Mat<NC> P = load_link<NC>(L.P, mu, s, L.V);
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) P.m[i][j] += eps * F.m[i][j];
  store_link<NC>(L.P, mu, s, L.V, P);
}

template <int NC>
LYM_D void hmc_drift_link(const HmcLat& L, double eps, int mu, int64_t s) {
  const Mat<NC> e = expm(mscale(cx<double>{eps, 0.0}, load_link<NC>(L.P, mu, s, L.V)));
  store_link<NC>(L.U, mu, s, L.V, mul(e, load_link<NC>(L.U, mu, s, L.V)));
}

// kick = 1: momenta from the force; 0: links from the momenta
__global__ void __launch_bounds__(128) hmc_multi_kernel(const __grid_constant__ HmcTable t, int kick) {
  const HmcLat& L = t.l[hmc_lat_of(t, blockIdx.x)];
  const int64_t nb = (L.V + 127) / 128;
  const int64_t lb = blockIdx.x - L.b0;
  const int mu = (int)(lb / nb);
  const int64_t s = (lb - mu * nb) * 128 + threadIdx.x;
  if (s >= L.V) return;
  if (kick) {
    switch (L.nd * 10 + L.nc) {
      case 22: hmc_kick_link<2, 2>(L, t.eps, mu, s); break;
      case 23: hmc_kick_link<2, 3>(L, t.eps, mu, s); break;
      case 32: hmc_kick_link<3, 2>(L, t.eps, mu, s); break;
      case 33: hmc_kick_link<3, 3>(L, t.eps, mu, s); break;
      case 42: hmc_kick_link<4, 2>(L, t.eps, mu, s); break;
      default: hmc_kick_link<4, 3>(L, t.eps, mu, s); break;
    }
  } else if (L.nc == 2) {
    hmc_drift_link<2>(L, t.eps, mu, s);
  } else {
    hmc_drift_link<3>(L, t.eps, mu, s);
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
#define LYM_DISPATCH_ND_NC(nd, nc, CALL)                                              \
  do {                                                                                \
    if ((nd) == 2 && (nc) == 2) { constexpr int ND = 2, NC = 2; CALL; }               \
    else if ((nd) == 2 && (nc) == 3) { constexpr int ND = 2, NC = 3; CALL; }          \
    else if ((nd) == 3 && (nc) == 2) { constexpr int ND = 3, NC = 2; CALL; }          \
    else if ((nd) == 3 && (nc) == 3) { constexpr int ND = 3, NC = 3; CALL; }          \
    else if ((nd) == 4 && (nc) == 2) { constexpr int ND = 4, NC = 2; CALL; }          \
    else if ((nd) == 4 && (nc) == 3) { constexpr int ND = 4, NC = 3; CALL; }          \
    else { set_error("unsupported (nd=%d, N=%d)", (nd), (nc)); return LYM_ERR_UNSUPPORTED; } \
  } while (0)

}  // namespace lym

using namespace lym;

extern "C" {

int lym_staple_terms(const lym_lattice* lat, int nc, const void* gauge, int no_direction, void* terms,
                     void* stream) {
  LYM_REQUIRE(lat && gauge && terms, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(gauge != terms, LYM_ERR_BAD_ARG, "gauge and terms must not alias");
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid(grid_for(lat->V, 128), lat->nd);
  LYM_DISPATCH_ND_NC(lat->nd, nc, (staple_terms_kernel<ND, NC><<<grid, 128, 0, st>>>(
                                      lat->d_tab, lat->V, (const double2*)gauge, no_direction, (double2*)terms)));
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_staples(const lym_lattice* lat, int nc, const void* gauge, int no_direction, void* staples,
                void* stream) {
  LYM_REQUIRE(lat && gauge && staples, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(gauge != staples, LYM_ERR_BAD_ARG, "gauge and staples must not alias");
  dim3 grid(grid_for(lat->V, 128), lat->nd);
  cudaStream_t st = (cudaStream_t)stream;
  LYM_DISPATCH_ND_NC(lat->nd, nc, (staples_kernel<ND, NC><<<grid, 128, 0, st>>>(
                                      lat->d_tab, lat->V, (const double2*)gauge, no_direction, (double2*)staples)));
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_gauge_force(const lym_lattice* lat, int nc, double beta, const void* gauge, void* force, void* momenta,
                    double eps, void* stream) {
  LYM_REQUIRE(lat && gauge && (force || momenta), LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(gauge != force && gauge != momenta, LYM_ERR_BAD_ARG, "outputs must not alias the gauge field");
  dim3 grid(grid_for(lat->V, 128), lat->nd);
  cudaStream_t st = (cudaStream_t)stream;
  LYM_DISPATCH_ND_NC(lat->nd, nc, (gauge_force_kernel<ND, NC><<<grid, 128, 0, st>>>(
                                      lat->d_tab, lat->V, (const double2*)gauge, beta, (double2*)force,
                                      (double2*)momenta, eps)));
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_plaquette_sum(const lym_lattice* lat, int nc, const void* gauge, double* out, void* stream) {
  LYM_REQUIRE(lat && gauge && out, LYM_ERR_BAD_ARG, "null argument");
  Scratch* s;
  int rc = scratch_get(&s);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(host_reduce_mutex());
  const int slot = 1;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned nb = reduction_blocks(lat->V, 256);
  double* part = s->partials + (size_t)slot * Scratch::kMaxBlocks * Scratch::kMaxVals;
  double* res = s->results + slot * Scratch::kMaxVals;
  LYM_DISPATCH_ND_NC(lat->nd, nc, (plaquette_kernel<ND, NC><<<nb, 256, 0, st>>>(
                                      lat->d_tab, lat->V, (const double2*)gauge, part, s->counters + slot, res)));
  LYM_CHECK_LAUNCH();
  LYM_CUDA(cudaMemcpyAsync(s->host + slot * Scratch::kMaxVals, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  out[0] = s->host[slot * Scratch::kMaxVals];
  out[1] = s->host[slot * Scratch::kMaxVals + 1];
  return LYM_OK;
}

int lym_momenta_from_normals(int nd, int nc, int64_t volume, const double* normals, void* momenta, void* stream) {
  LYM_REQUIRE(normals && momenta && nd >= 1 && nd <= LYM_MAX_ND && volume >= 0, LYM_ERR_BAD_ARG, "bad argument");
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N must be 2 or 3");
  if (volume == 0) return LYM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid(grid_for(volume, 256), nd);
  if (nc == 2)
    momenta_from_normals_kernel<2><<<grid, 256, 0, st>>>(nd, volume, normals, (double2*)momenta);
  else
    momenta_from_normals_kernel<3><<<grid, 256, 0, st>>>(nd, volume, normals, (double2*)momenta);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_momenta_energy(int nd, int nc, int64_t volume, const void* momenta, double* out, void* stream) {
  LYM_REQUIRE(momenta && out && nd >= 1 && nd <= LYM_MAX_ND && volume >= 0, LYM_ERR_BAD_ARG, "bad argument");
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N must be 2 or 3");
  Scratch* s;
  int rc = scratch_get(&s);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(host_reduce_mutex());
  const int slot = 1;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nl = (int64_t)nd * volume;
  unsigned nb = reduction_blocks(nl, 256);
  double* part = s->partials + (size_t)slot * Scratch::kMaxBlocks * Scratch::kMaxVals;
  double* res = s->results + slot * Scratch::kMaxVals;
  if (nc == 2)
    momenta_energy_kernel<2><<<nb, 256, 0, st>>>(nl, volume, (const double2*)momenta, part, s->counters + slot, res);
  else
    momenta_energy_kernel<3><<<nb, 256, 0, st>>>(nl, volume, (const double2*)momenta, part, s->counters + slot, res);
  LYM_CHECK_LAUNCH();
  LYM_CUDA(cudaMemcpyAsync(s->host + slot * Scratch::kMaxVals, res, sizeof(double), cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  out[0] = s->host[slot * Scratch::kMaxVals];
  return LYM_OK;
}

int lym_update_momenta(int64_t n, void* momenta, const void* force, double eps, void* stream) {
  LYM_REQUIRE(n >= 0 && momenta && force, LYM_ERR_BAD_ARG, "null argument");
  if (n == 0) return LYM_OK;
  axpy_real_kernel<<<reduction_blocks(n, 256) * 4, 256, 0, (cudaStream_t)stream>>>(n, (double2*)momenta,
                                                                                     (const double2*)force, eps);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_gauge_hmc_step_multi(int nlat, const lym_lattice* const* lats, const int* nc, const double* betas,
                             void* const* gauges, void* const* momenta, double eps_p, double eps_u, void* stream) {
  LYM_REQUIRE(nlat >= 1 && nlat <= kHmcMaxLat, LYM_ERR_BAD_ARG, "nlat must be in [1, %d]", kHmcMaxLat);
  LYM_REQUIRE(lats && nc && betas && gauges && momenta, LYM_ERR_BAD_ARG, "null argument");
  HmcTable t;
  t.n = nlat;
  int64_t blocks = 0;
  for (int l = 0; l < nlat; ++l) {
    LYM_REQUIRE(lats[l] && gauges[l] && momenta[l], LYM_ERR_BAD_ARG, "null argument (lattice %d)", l);
    LYM_REQUIRE(nc[l] == 2 || nc[l] == 3, LYM_ERR_UNSUPPORTED, "N must be 2 or 3 (lattice %d)", l);
    LYM_REQUIRE(lats[l]->nd >= 2 && lats[l]->nd <= 4, LYM_ERR_UNSUPPORTED, "nd must be 2, 3 or 4 (lattice %d)", l);
    LYM_REQUIRE(lats[l]->V >= 1, LYM_ERR_BAD_ARG, "empty lattice %d", l);
    LYM_REQUIRE(gauges[l] != momenta[l], LYM_ERR_BAD_ARG, "gauge and momenta alias (lattice %d)", l);
    for (int k = 0; k < l; ++k)  // two lattices on one buffer would race in the same launch
      LYM_REQUIRE(gauges[k] != gauges[l] && momenta[k] != momenta[l] && gauges[k] != momenta[l] &&
                      momenta[k] != gauges[l],
                  LYM_ERR_BAD_ARG, "lattices %d and %d share a buffer", k, l);
    t.l[l] = HmcLat{lats[l]->d_tab, (double2*)gauges[l], (double2*)momenta[l], lats[l]->V, betas[l], lats[l]->nd,
                    nc[l], (int)blocks};
    blocks += (int64_t)lats[l]->nd * ((lats[l]->V + 127) / 128);
  }
  LYM_REQUIRE(blocks < (int64_t(1) << 31), LYM_ERR_UNSUPPORTED, "too many links for one launch");
  cudaStream_t st = (cudaStream_t)stream;
  t.eps = eps_p;
  hmc_multi_kernel<<<(unsigned)blocks, 128, 0, st>>>(t, 1);
  LYM_CHECK_LAUNCH();
  t.eps = eps_u;
  hmc_multi_kernel<<<(unsigned)blocks, 128, 0, st>>>(t, 0);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_update_links(int nd, int nc, int64_t volume, void* gauge, const void* momenta, double eps, int reunitarize,
                     void* stream) {
  LYM_REQUIRE(gauge && momenta && nd >= 1 && nd <= LYM_MAX_ND && volume >= 0, LYM_ERR_BAD_ARG, "bad argument");
  if (volume == 0) return LYM_OK;
  const int64_t nl = (int64_t)nd * volume;
  cudaStream_t st = (cudaStream_t)stream;
  if (nc == 2)
    update_links_kernel<2><<<grid_for(nl, 128), 128, 0, st>>>(nl, volume, (double2*)gauge,
                                                              (const double2*)momenta, eps, reunitarize);
  else if (nc == 3)
    update_links_kernel<3><<<grid_for(nl, 128), 128, 0, st>>>(nl, volume, (double2*)gauge,
                                                              (const double2*)momenta, eps, reunitarize);
  else {
    set_error("N=%d not supported", nc);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_unitary_projection(int nd, int nc, int64_t volume, const void* in, void* out, void* stream) {
  LYM_REQUIRE(in && out && nd >= 1 && nd <= LYM_MAX_ND && volume >= 0, LYM_ERR_BAD_ARG, "bad argument");
  if (volume == 0) return LYM_OK;
  const int64_t nl = (int64_t)nd * volume;
  cudaStream_t st = (cudaStream_t)stream;
  if (nc == 2)
    unitary_projection_kernel<2><<<grid_for(nl, 128), 128, 0, st>>>(nl, volume, (const double2*)in, (double2*)out);
  else if (nc == 3)
    unitary_projection_kernel<3><<<grid_for(nl, 128), 128, 0, st>>>(nl, volume, (const double2*)in, (double2*)out);
  else {
    set_error("N=%d not supported", nc);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int lym_fermion_force(const lym_lattice* lat, int nc, double kappa, int hermitian, double bc_re, double bc_im,
                      const void* gauge, int nterms, const double* alphas, const void* X, const void* Y,
                      int symmetric, double scale, void* force, void* stream) {
  LYM_REQUIRE(lat && gauge && alphas && X && Y && force, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nterms >= 1 && nterms <= kMaxForceTerms, LYM_ERR_BAD_ARG, "nterms must be in [1, %d]",
              kMaxForceTerms);
  if (lat->nd != 2 && lat->nd != 4) {
    set_error("Number of dimensions %d not supported for fermions!", lat->nd);
    return LYM_ERR_UNSUPPORTED;
  }
  ForceTerms t;
  for (int i = 0; i < kMaxForceTerms; ++i) t.alpha[i] = i < nterms ? alphas[i] : 0.0;
  dim3 grid(grid_for(lat->V, 128), lat->nd);
  cudaStream_t st = (cudaStream_t)stream;
  const int Lt = lat->dims[lat->nd - 1];
#define LYM_FF(ND_, NC_, H_)                                                                        \
  fermion_force_kernel<ND_, NC_, H_><<<grid, 128, 0, st>>>(lat->d_tab, lat->V, Lt, kappa, bc_re, bc_im, \
                                                           (const double2*)gauge, nterms, t,          \
                                                           (const double2*)X, (const double2*)Y,      \
                                                           symmetric, scale, (double2*)force)
  if (lat->nd == 2 && nc == 2) { if (hermitian) LYM_FF(2, 2, true); else LYM_FF(2, 2, false); }
  else if (lat->nd == 2 && nc == 3) { if (hermitian) LYM_FF(2, 3, true); else LYM_FF(2, 3, false); }
  else if (lat->nd == 4 && nc == 2) { if (hermitian) LYM_FF(4, 2, true); else LYM_FF(4, 2, false); }
  else if (lat->nd == 4 && nc == 3) { if (hermitian) LYM_FF(4, 3, true); else LYM_FF(4, 3, false); }
  else {
    set_error("N=%d not supported", nc);
    return LYM_ERR_UNSUPPORTED;
  }
#undef LYM_FF
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// gauge observables (measurements.py:46-290): link products along paths, slice sums
// ---------------------------------------------------------------------------
namespace lym {

constexpr int kMaxPathSteps = 256;
struct PathSteps {
  signed char step[kMaxPathSteps];  // +(mu+1): U_mu(y), y += mu;  -(mu+1): y -= mu, U_mu(y)^dag
};

// One thread per starting site: M = product of the links along the path; writes
// Tr M (trace = 1, out (V) complex) or M (out (N, N, V)).
template <int NC>
__global__ void __launch_bounds__(128) path_kernel(const int32_t* __restrict__ tab, int nd, int64_t V,
                                                   const double2* __restrict__ U, int nsteps, PathSteps path,
                                                   int want_trace, double2* __restrict__ out) {
  const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (x >= V) return;
  Mat<NC> m = mident<NC>();
  int64_t y = x;
  for (int k = 0; k < nsteps; ++k) {
    const int s = path.step[k];
    const int mu = (s > 0 ? s : -s) - 1;
    if (s > 0) {
      m = mul(m, load_link<NC>(U, mu, y, V));
      y = tab[mu * V + y];
    } else {
      y = tab[(nd + mu) * V + y];
      m = mul_nd(m, load_link<NC>(U, mu, y, V));
    }
  }
  if (want_trace) {
    st(out + x, trace(m));
  } else {
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) st(out + ((int64_t)i * NC + j) * V + x, m.m[i][j]);
  }
}

// out[2z], out[2z+1] = sum of f(x) over the sites with x_dir = z (and, when
// mask_len > 0, x_mask = 0); x_d = (x / stride_d) mod L_d for the lexicographic
// index with the last coordinate fastest.  One block per slice, fixed-order
// reduction (deterministic).
__global__ void __launch_bounds__(256) slice_sum_kernel(int64_t V, int64_t stride, int L, int64_t mask_stride,
                                                        int mask_len, const double2* __restrict__ f,
                                                        double* __restrict__ out) {
  __shared__ double sh[2 * 32];
  const int z = blockIdx.x;
  double re = 0.0, im = 0.0;
  for (int64_t x = threadIdx.x; x < V; x += blockDim.x) {
    if ((x / stride) % L != z) continue;
    if (mask_len > 0 && (x / mask_stride) % mask_len != 0) continue;
    const double2 v = f[x];
    re += v.x;
    im += v.y;
  }
  double v2[2] = {re, im};
  block_sum<2>(v2, sh);
  if (threadIdx.x == 0) {
    out[2 * z] = v2[0];
    out[2 * z + 1] = v2[1];
  }
}

}  // namespace lym

extern "C" int lym_path_product(const lym_lattice* lat, int nc, const void* gauge, int nsteps, const int* steps,
                                int trace, void* out, void* stream) {
  using namespace lym;
  LYM_REQUIRE(lat && gauge && out && (steps || nsteps == 0), LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nsteps >= 0 && nsteps <= kMaxPathSteps, LYM_ERR_BAD_ARG, "at most %d steps", kMaxPathSteps);
  PathSteps p{};
  for (int k = 0; k < nsteps; ++k) {
    const int s = steps[k];
    LYM_REQUIRE(s != 0 && (s > 0 ? s : -s) <= lat->nd, LYM_ERR_BAD_ARG, "step %d out of range", s);
    p.step[k] = (signed char)s;
  }
  dim3 grid(grid_for(lat->V, 128));
  cudaStream_t st = (cudaStream_t)stream;
  if (nc == 2)
    path_kernel<2><<<grid, 128, 0, st>>>(lat->d_tab, lat->nd, lat->V, (const double2*)gauge, nsteps, p, trace != 0,
                                         (double2*)out);
  else if (nc == 3)
    path_kernel<3><<<grid, 128, 0, st>>>(lat->d_tab, lat->nd, lat->V, (const double2*)gauge, nsteps, p, trace != 0,
                                         (double2*)out);
  else {
    set_error("N=%d not supported", nc);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

extern "C" int lym_slice_sums(const lym_lattice* lat, int direction, int mask_direction, const void* field,
                              double* out, void* stream) {
  using namespace lym;
  LYM_REQUIRE(lat && field && out, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(direction >= 0 && direction < lat->nd && mask_direction < lat->nd, LYM_ERR_BAD_ARG,
              "direction out of range");
  auto stride_of = [&](int d) {
    int64_t s = 1;
    for (int e = d + 1; e < lat->nd; ++e) s *= lat->dims[e];
    return s;
  };
  const int L = lat->dims[direction];
  const int mask_len = mask_direction >= 0 ? lat->dims[mask_direction] : 0;
  slice_sum_kernel<<<L, 256, 0, (cudaStream_t)stream>>>(lat->V, stride_of(direction), L,
                                                        mask_direction >= 0 ? stride_of(mask_direction) : 1,
                                                        mask_len, (const double2*)field, out);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}
