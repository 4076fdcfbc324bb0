// Full-lattice shifted solvers on Q^2 = D^dag D in the reference layout (FP64):
//  * multishift CG (builder-defined, Jegerlehner's recurrences, hep-lat/9612014)
//  * the reference's multishift MMMR (dirac_solver.py:19-53), same arithmetic
//    order, so its iteration count matches the reference's.
// Scalars are computed on the host from fused device reductions (two
// synchronisations per iteration); the operator is two launches of the
// reference-layout Wilson kernel.
#include <cmath>
#include <complex>
#include <vector>

#include "lym_internal.cuh"
#include "lym_kernels.cuh"

namespace lym {

constexpr int kMaxShifts = 32;

struct ShiftVecs {
  double2* x[kMaxShifts];
  double2* p[kMaxShifts];
  double ar[kMaxShifts], ai[kMaxShifts];   // x_s += a_s * (r or p_s)
  double zr[kMaxShifts], zi[kMaxShifts];   // p_s = z_s r + b_s p_s
  double br[kMaxShifts], bi[kMaxShifts];
  int active[kMaxShifts];
};

// out = a + sigma * b; d[0..1] = <out, b>, d[2] = <out, out>
__global__ void __launch_bounds__(256) shift_dots_kernel(int64_t n, const double2* a,
                                                         const double2* __restrict__ b, double sigma,
                                                         double2* out, double* partials,
                                                         unsigned* counter, double* result) {
  __shared__ double sh[3 * 32];
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 x = a[i], y = b[i];
    double2 o = make_double2(x.x + sigma * y.x, x.y + sigma * y.y);
    out[i] = o;
    v[0] += o.x * y.x + o.y * y.y;
    v[1] += o.x * y.y - o.y * y.x;
    v[2] += o.x * o.x + o.y * o.y;
  }
  if (grid_sum<3>(v, partials, counter, sh) && threadIdx.x == 0) {
    result[0] = v[0];
    result[1] = v[1];
    result[2] = v[2];
  }
}

// x_s += a_s * src_s for active shifts (src_s = r if use_r else p_s);
// r -= (cr + i ci) * q ; result[0] = |r|^2
__global__ void __launch_bounds__(256) shift_update_kernel(int64_t n, int nshift, ShiftVecs sv, int use_r,
                                                           double2* __restrict__ r, const double2* __restrict__ q,
                                                           double cr, double ci, double* partials, unsigned* counter,
                                                           double* result) {
  __shared__ double sh[32];
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 rv = r[i];
    for (int s = 0; s < nshift; ++s) {
      if (!sv.active[s]) continue;
      const double2 src = use_r ? rv : sv.p[s][i];
      double2 xv = sv.x[s][i];
      xv.x += sv.ar[s] * src.x - sv.ai[s] * src.y;
      xv.y += sv.ar[s] * src.y + sv.ai[s] * src.x;
      sv.x[s][i] = xv;
    }
    const double2 qv = q[i];
    double2 nr = make_double2(rv.x - (cr * qv.x - ci * qv.y), rv.y - (cr * qv.y + ci * qv.x));
    r[i] = nr;
    v[0] += nr.x * nr.x + nr.y * nr.y;
  }
  if (grid_sum<1>(v, partials, counter, sh) && threadIdx.x == 0) result[0] = v[0];
}

// p_s = z_s r + b_s p_s for active shifts
__global__ void __launch_bounds__(256) shift_p_kernel(int64_t n, int nshift, ShiftVecs sv,
                                                      const double2* __restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 rv = r[i];
    for (int s = 0; s < nshift; ++s) {
      if (!sv.active[s]) continue;
      double2 pv = sv.p[s][i];
      double2 o;
      o.x = sv.zr[s] * rv.x - sv.zi[s] * rv.y + sv.br[s] * pv.x - sv.bi[s] * pv.y;
      o.y = sv.zr[s] * rv.y + sv.zi[s] * rv.x + sv.br[s] * pv.y + sv.bi[s] * pv.x;
      sv.p[s][i] = o;
    }
  }
}

__global__ void copy_kernel(int64_t n, const double2* __restrict__ a, double2* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

struct MsWork {
  double2* pool = nullptr;
  size_t nvec = 0;
  int64_t n = 0;
  cudaStream_t stream = nullptr;
};

// Reduction slots for these host-driven solvers: they hold the host mutex for
// the whole solve, so slot 1 of the shared scratch is theirs.
struct Reducer {
  Scratch* s;
  double* part;
  unsigned* cnt;
  double* res;
  double* host;
};

static int get_reducer(Reducer* r) {
  int rc = scratch_get(&r->s);
  if (rc) return rc;
  const int slot = 1;
  r->part = r->s->partials + (size_t)slot * Scratch::kMaxBlocks * Scratch::kMaxVals;
  r->cnt = r->s->counters + slot;
  r->res = r->s->results + slot * Scratch::kMaxVals;
  r->host = r->s->host + slot * Scratch::kMaxVals;
  return LYM_OK;
}

static int read_back(Reducer& r, int n, cudaStream_t st) {
  LYM_CUDA(cudaMemcpyAsync(r.host, r.res, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  return LYM_OK;
}

// tmp2 = Q(Q v): hermitian Wilson operator applied twice
static int apply_q2(const GaugeView& gv, double kappa, const double2* v, double2* tmp, double2* out, cudaStream_t st) {
  int rc = wilson_full(gv.lat, gv.nc, kappa, 1, gv.bcr, gv.bci, gv.uref, 1, v, tmp, st);
  if (rc) return rc;
  return wilson_full(gv.lat, gv.nc, kappa, 1, gv.bcr, gv.bci, gv.uref, 1, tmp, out, st);
}

}  // namespace lym

using namespace lym;

extern "C" {

int lym_multishift_solve(lym_gauge* g, double kappa, int nshift, const double* shifts, const void* b, void* xs,
                         double tol, int max_iter, int* iterations, void* stream) {
  LYM_REQUIRE(g && shifts && b && xs && iterations, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nshift >= 1 && nshift <= kMaxShifts, LYM_ERR_BAD_ARG, "nshift must be in [1, %d]", kMaxShifts);
  LYM_REQUIRE(tol > 0 && max_iter > 0, LYM_ERR_BAD_ARG, "tol and max_iter must be positive");
  GaugeView gv;
  int rc = gauge_view(g, &gv);
  if (rc) return rc;
  LYM_REQUIRE(gv.lat->nd != 3, LYM_ERR_UNSUPPORTED,
              "Q^2 + sigma needs the hermitian Q = gamma_d D, which three dimensions do not have");
  int base = 0;
  for (int s = 0; s < nshift; ++s) {
    LYM_REQUIRE(shifts[s] >= 0, LYM_ERR_BAD_ARG, "negative shifts need BiCGStab (dirac_solver.py:26-30)");
    if (shifts[s] < shifts[base]) base = s;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = gv.V * gv.ncomp;
  std::lock_guard<std::mutex> lk(host_reduce_mutex());
  Reducer red;
  rc = get_reducer(&red);
  if (rc) return rc;
  // workspace: r, ap, tmp, and p_s per shift
  double2* pool = nullptr;
  if (cudaMalloc(&pool, sizeof(double2) * n * (3 + nshift)) != cudaSuccess) {
    cudaGetLastError();
    set_error("multishift workspace does not fit");
    return LYM_ERR_OOM;
  }
  double2* r = pool;
  double2* ap = pool + n;
  double2* tmp = pool + 2 * n;
  double2* x = (double2*)xs;
  const unsigned nb = reduction_blocks(n, 256);
  ShiftVecs sv{};
  for (int s = 0; s < nshift; ++s) {
    sv.x[s] = x + s * n;
    sv.p[s] = pool + (3 + s) * n;
    sv.active[s] = 1;
  }
  int status = LYM_OK;
  auto fail = [&](int code) {
    cudaStreamSynchronize(st);
    cudaFree(pool);
    return code;
  };
  if (cudaMemsetAsync(x, 0, sizeof(double2) * n * nshift, st) != cudaSuccess) return fail(LYM_ERR_CUDA);
  copy_kernel<<<nb * 2, 256, 0, st>>>(n, (const double2*)b, r);
  for (int s = 0; s < nshift; ++s) copy_kernel<<<nb * 2, 256, 0, st>>>(n, (const double2*)b, sv.p[s]);
  rc = cdot_device(n, b, b, red.res, 1, st);
  if (rc) return fail(rc);
  if (read_back(red, 1, st)) return fail(LYM_ERR_CUDA);
  double rr = red.host[0];
  const double stop2 = tol * tol * rr;
  std::vector<double> zprev(nshift, 1.0), z(nshift, 1.0), znext(nshift, 1.0);
  double a_prev = 1.0, b_prev = 0.0;
  int it = 0;
  bool converged = rr == 0.0;
  const double s0 = shifts[base];
  while (!converged && it < max_iter) {
    rc = apply_q2(gv, kappa, sv.p[base], tmp, ap, st);
    if (rc) return fail(rc);
    shift_dots_kernel<<<nb, 256, 0, st>>>(n, ap, sv.p[base], s0, ap, red.part, red.cnt, red.res);
    if (read_back(red, 3, st)) return fail(LYM_ERR_CUDA);
    const double pap = red.host[0];  // <ap, p> real for Hermitian positive A
    const double a = rr / pap;
    for (int s = 0; s < nshift; ++s) {
      if (!sv.active[s]) continue;
      if (s == base) {
        znext[s] = 1.0;
        sv.ar[s] = a;
      } else {
        const double d = shifts[s] - s0;
        znext[s] = z[s] * zprev[s] * a_prev / (a * b_prev * (zprev[s] - z[s]) + zprev[s] * a_prev * (1.0 + d * a));
        sv.ar[s] = a * znext[s] / z[s];
      }
      sv.ai[s] = 0.0;
    }
    shift_update_kernel<<<nb, 256, 0, st>>>(n, nshift, sv, 0, r, ap, a, 0.0, red.part, red.cnt, red.res);
    if (read_back(red, 1, st)) return fail(LYM_ERR_CUDA);
    const double rr_new = red.host[0];
    const double bet = rr_new / rr;
    for (int s = 0; s < nshift; ++s) {
      if (!sv.active[s]) continue;
      if (s == base) {
        sv.zr[s] = 1.0;
        sv.br[s] = bet;
      } else {
        sv.zr[s] = znext[s];
        const double q = znext[s] / z[s];
        sv.br[s] = bet * q * q;
      }
      sv.zi[s] = 0.0;
      sv.bi[s] = 0.0;
    }
    shift_p_kernel<<<nb, 256, 0, st>>>(n, nshift, sv, r);
    ++it;
    for (int s = 0; s < nshift; ++s) {
      zprev[s] = z[s];
      z[s] = znext[s];
      if (s != base && sv.active[s] && z[s] * z[s] * rr_new < stop2) sv.active[s] = 0;
    }
    a_prev = a;
    b_prev = bet;
    rr = rr_new;
    converged = rr_new < stop2;
    if (cudaGetLastError() != cudaSuccess) return fail(LYM_ERR_CUDA);
  }
  *iterations = it;
  if (!converged) {
    set_error("multishift CG: no convergence after %d iterations", it);
    status = LYM_ERR_NOT_CONVERGED;
  }
  cudaStreamSynchronize(st);
  cudaFree(pool);
  return status;
}

int lym_mmmr_solve(lym_gauge* g, double kappa, int nshift, const double* shifts, const void* b, void* xs,
                   int max_steps, double precision, double omega, int* steps, void* stream) {
  LYM_REQUIRE(g && shifts && b && xs && steps, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(nshift >= 1 && nshift <= kMaxShifts, LYM_ERR_BAD_ARG, "nshift must be in [1, %d]", kMaxShifts);
  LYM_REQUIRE(max_steps > 0, LYM_ERR_BAD_ARG, "max_steps must be positive");
  for (int s = 0; s < nshift; ++s)
    LYM_REQUIRE(shifts[s] >= 0, LYM_ERR_UNSUPPORTED, "negative shifts go to BiCGStab (dirac_solver.py:26-30)");
  GaugeView gv;
  int rc = gauge_view(g, &gv);
  if (rc) return rc;
  LYM_REQUIRE(gv.lat->nd != 3, LYM_ERR_UNSUPPORTED,
              "Q^2 + sigma needs the hermitian Q = gamma_d D, which three dimensions do not have");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = gv.V * gv.ncomp;
  std::lock_guard<std::mutex> lk(host_reduce_mutex());
  Reducer red;
  rc = get_reducer(&red);
  if (rc) return rc;
  double2* pool = nullptr;
  if (cudaMalloc(&pool, sizeof(double2) * n * 3) != cudaSuccess) {
    cudaGetLastError();
    set_error("MMMR workspace does not fit");
    return LYM_ERR_OOM;
  }
  double2* r = pool;
  double2* p = pool + n;
  double2* tmp = pool + 2 * n;
  double2* x = (double2*)xs;
  const unsigned nb = reduction_blocks(n, 256);
  auto fail = [&](int code) {
    cudaStreamSynchronize(st);
    cudaFree(pool);
    return code;
  };
  if (cudaMemsetAsync(x, 0, sizeof(double2) * n * nshift, st) != cudaSuccess) return fail(LYM_ERR_CUDA);
  copy_kernel<<<nb * 2, 256, 0, st>>>(n, (const double2*)b, r);
  ShiftVecs sv{};
  for (int s = 0; s < nshift; ++s) {
    sv.x[s] = x + s * n;
    sv.p[s] = nullptr;
    sv.active[s] = 1;
  }
  std::vector<std::complex<double>> f(nshift, 1.0);
  const double sl = shifts[nshift - 1];
  int step = 0;
  bool converged = false;
  for (step = 0; step < max_steps; ++step) {
    // p = A r + shift_last r  (dirac_solver.py:33)
    rc = apply_q2(gv, kappa, r, tmp, p, st);
    if (rc) return fail(rc);
    shift_dots_kernel<<<nb, 256, 0, st>>>(n, p, r, sl, p, red.part, red.cnt, red.res);
    if (read_back(red, 3, st)) return fail(LYM_ERR_CUDA);
    // alpha = omega <p, r> / <p, p>   (dirac_solver.py:35)
    const std::complex<double> alpha = omega * std::complex<double>(red.host[0], red.host[1]) / red.host[2];
    sv.ar[nshift - 1] = alpha.real();
    sv.ai[nshift - 1] = alpha.imag();
    for (int s = 0; s < nshift - 1; ++s) {  // dirac_solver.py:39-43
      f[s] = f[s] / (1.0 + (shifts[s] - sl) * alpha);
      const std::complex<double> c = alpha * f[s];
      sv.ar[s] = c.real();
      sv.ai[s] = c.imag();
    }
    // x_s += alpha f_s r ; r -= alpha p ; |<r, r>|   (dirac_solver.py:37-47)
    shift_update_kernel<<<nb, 256, 0, st>>>(n, nshift, sv, 1, r, p, alpha.real(), alpha.imag(), red.part, red.cnt,
                                            red.res);
    if (read_back(red, 1, st)) return fail(LYM_ERR_CUDA);
    if (std::fabs(red.host[0]) < precision) {
      converged = true;
      break;
    }
    if (cudaGetLastError() != cudaSuccess) return fail(LYM_ERR_CUDA);
  }
  *steps = converged ? step : max_steps - 1;
  cudaStreamSynchronize(st);
  cudaFree(pool);
  if (!converged) {
    set_error("MMMR: no convergence after %d steps", max_steps);
    return LYM_ERR_NOT_CONVERGED;
  }
  return LYM_OK;
}

}  // extern "C"
