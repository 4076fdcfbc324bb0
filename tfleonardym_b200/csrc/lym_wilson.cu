// Wilson Dirac operator in the reference layout (FP64, full lattice) and the
// vector algebra the reference-compatible solvers need.
//
// One thread per (site, vector).  Each spinor component plane (ns, N, V) is
// contiguous over sites, so every load of a complex128 is one coalesced
// 16-byte access; neighbour indices come from the int32 copies of the
// reference's own sup/sdn tables (lattice.py:86-120).
#include <mutex>

#include "lym_internal.cuh"
#include "lym_kernels.cuh"

namespace lym {

// ---------------------------------------------------------------------------
// library-owned reduction scratch, one per device
// ---------------------------------------------------------------------------
static std::mutex g_scratch_mu;
static std::mutex g_host_reduce_mu;
std::mutex& host_reduce_mutex() { return g_host_reduce_mu; }
static Scratch g_scratch[64];
static bool g_scratch_ok[64];

int scratch_get(Scratch** out) {
  int dev = 0;
  LYM_CUDA(cudaGetDevice(&dev));
  LYM_REQUIRE(dev >= 0 && dev < 64, LYM_ERR_BAD_ARG, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  Scratch& s = g_scratch[dev];
  if (!g_scratch_ok[dev]) {
    size_t np = (size_t)Scratch::kSlots * Scratch::kMaxBlocks * Scratch::kMaxVals;
    if (cudaMalloc(&s.partials, np * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&s.counters, Scratch::kSlots * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&s.results, Scratch::kSlots * Scratch::kMaxVals * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&s.host, Scratch::kSlots * Scratch::kMaxVals * sizeof(double)) != cudaSuccess) {
      set_error("scratch allocation failed");
      return LYM_ERR_OOM;
    }
    LYM_CUDA(cudaMemset(s.counters, 0, Scratch::kSlots * sizeof(unsigned)));
    LYM_CUDA(cudaDeviceSynchronize());
    g_scratch_ok[dev] = true;
  }
  *out = &s;
  return LYM_OK;
}

// ---------------------------------------------------------------------------
// full-lattice hop, reference layout
// ---------------------------------------------------------------------------
// One hop of the full-lattice operator for R vectors at one site: acc[r] +=
// W (1 - s g_mu) psi_r(y), W = U (s = +1, forward) or U^dag (s = -1, backward);
// the link is loaded once by the caller and applied to the R vectors.
template <int ND, int NC, int R>
LYM_D void full_hop(int mu, int s, const cx<double> (&u)[NC][NC], const double2* const (&psi)[R], int V, int y,
                    cx<double> (&acc)[R][Gamma<ND>::NS][NC]) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if constexpr (ND == 3) {
      cx<double> p0[NC], p1[NC], h[NC], t[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        p0[c] = ld(psi[r] + (size_t)c * V + y);
        p1[c] = ld(psi[r] + (size_t)(NC + c) * V + y);
      }
      proj3<double, NC>(mu, s, p0, p1, h);
#pragma unroll
      for (int i = 0; i < NC; ++i) {
        if (s > 0) {
          t[i] = u[i][0] * h[0];
#pragma unroll
          for (int j = 1; j < NC; ++j) cmac(t[i], u[i][j], h[j]);
        } else {
          t[i] = cmul_cj(u[0][i], h[0]);
#pragma unroll
          for (int j = 1; j < NC; ++j) cmac_cj(t[i], u[j][i], h[j]);
        }
      }
      recon3<double, NC>(mu, s, t, acc[r][0], acc[r][1]);
    } else {
#pragma unroll
      for (int a = 0; a < Gamma<ND>::NS / 2; ++a) {
        const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
        cx<double> h[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const cx<double> pb = mul_phase(ph, ld(psi[r] + (size_t)(jb * NC + c) * V + y));
          const cx<double> pa = ld(psi[r] + (size_t)(a * NC + c) * V + y);
          h[c] = s > 0 ? pa - pb : pa + pb;
        }
        // lower row: -s conj(g_a)
        const int lph = s > 0 ? phase_neg(phase_conj(ph)) : phase_conj(ph);
#pragma unroll
        for (int i = 0; i < NC; ++i) {
          cx<double> t;
          if (s > 0) {
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

// One thread per site and R vectors.  The grid is one-dimensional with the vector
// group fastest (block b: group b % ngroups, site block b / ngroups), so the blocks
// that read one site block's links run back to back and all but the first find the
// links in L2: each link crosses HBM about once per launch, not once per vector.
// One resident block per SM is declared enough, so ptxas keeps every neighbour's
// loads in flight at once (memory-bound FP64 stencil).
template <int ND, int NC, bool HERM, int R>
__global__ void __launch_bounds__(128, 1) wilson_full_kernel(
    const int32_t* __restrict__ tab, int V, int Lt, double kappa, double bcr, double bci,
    const double2* __restrict__ U, const double2* __restrict__ in, double2* __restrict__ out, int ngroups) {
  constexpr int NS = Gamma<ND>::NS;
  const int group = (int)(blockIdx.x % (unsigned)ngroups);
  const int s = (int)(blockIdx.x / (unsigned)ngroups) * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const size_t vec = (size_t)NS * NC * V;
  const double2* psi[R];
#pragma unroll
  for (int r = 0; r < R; ++r) psi[r] = in + ((size_t)group * R + r) * vec;
  const cx<double> bc{bcr, bci};

  cx<double> acc[R][NS][NC];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[r][a][c] = czero<double>();

#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      // forward: U_mu(x) (1 - g_mu) psi(x + mu); backward: U_mu(x - mu)^dag (1 + g_mu) psi(x - mu)
      const bool fwd = dir == 0;
      const int y = fwd ? tab[mu * V + s] : tab[ND * V + mu * V + s];
      const int ls = fwd ? s : y;  // the link lives on x (forward) or x - mu (backward)
      cx<double> u[NC][NC];
#pragma unroll
      for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) u[i][j] = ld(U + ((size_t)(mu * NC + i) * NC + j) * V + ls);
      if (mu == ND - 1 && (s % Lt) == (fwd ? Lt - 1 : 0)) {
#pragma unroll
        for (int i = 0; i < NC; ++i)
#pragma unroll
          for (int j = 0; j < NC; ++j) u[i][j] = bc * u[i][j];
      }
      full_hop<ND, NC, R>(mu, fwd ? 1 : -1, u, psi, V, y, acc);
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    double2* res = out + ((size_t)group * R + r) * vec;
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        cx<double> v = ld(psi[r] + (size_t)(a * NC + c) * V + s) + kappa * acc[r][a][c];
        if (HERM && a >= NS / 2) v = -v;
        st(res + (size_t)(a * NC + c) * V + s, v);
      }
  }
}

template <int ND, int NC, int R>
static void launch_full_r(const lym_lattice* lat, double kappa, int herm, double bcr, double bci, const void* gauge,
                          int ngroups, const void* in, void* out, cudaStream_t st) {
  const unsigned grid = grid_for(lat->V, 128) * (unsigned)ngroups;
  const int Lt = lat->dims[ND - 1];
  if (herm)
    wilson_full_kernel<ND, NC, true, R><<<grid, 128, 0, st>>>(lat->d_tab, (int)lat->V, Lt, kappa, bcr, bci,
                                                             (const double2*)gauge, (const double2*)in,
                                                             (double2*)out, ngroups);
  else
    wilson_full_kernel<ND, NC, false, R><<<grid, 128, 0, st>>>(lat->d_tab, (int)lat->V, Lt, kappa, bcr, bci,
                                                              (const double2*)gauge, (const double2*)in,
                                                              (double2*)out, ngroups);
}

// nvec vectors: groups of R = 2 (4D, four-component spinors) or 4 (2D, 3D) vectors
// per thread share each link load (sized to the 255-register budget), the groups of
// a site block in consecutive blocks; a remainder runs one vector per thread.
// Measured at 32^4 SU(3), 4 vectors: 0.43 of the HBM peak with R = 2, 0.39 with
// R = 1 (one vector alone: 0.66-0.69) -- the kernel is latency-bound at 8 warps per SM.
template <int ND, int NC>
static int launch_full(const lym_lattice* lat, double kappa, int herm, double bcr, double bci,
                       const void* gauge, int nvec, const void* in, void* out, cudaStream_t st) {
  constexpr int R = ND == 4 ? 2 : 4;
  const size_t vec = (size_t)Gamma<ND>::NS * NC * lat->V * sizeof(double2);
  const int ng = nvec / R;
  if (ng > 0) launch_full_r<ND, NC, R>(lat, kappa, herm, bcr, bci, gauge, ng, in, out, st);
  const int rest = nvec - ng * R;
  if (rest > 0)
    launch_full_r<ND, NC, 1>(lat, kappa, herm, bcr, bci, gauge, rest, (const char*)in + (size_t)ng * R * vec,
                             (char*)out + (size_t)ng * R * vec, st);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

int wilson_full(const lym_lattice* lat, int nc, double kappa, int herm, double bcr, double bci,
                const void* gauge, int nvec, const void* in, void* out, cudaStream_t st) {
  LYM_REQUIRE(lat && gauge && in && out, LYM_ERR_BAD_ARG, "null argument");
  LYM_REQUIRE(in != out, LYM_ERR_BAD_ARG, "in and out must not alias");
  LYM_REQUIRE(nvec >= 1 && nvec <= 65535, LYM_ERR_BAD_ARG, "nvec out of range");
  if (lat->nd < 2 || lat->nd > 4) {
    set_error("Number of dimensions %d not supported for fermions!", lat->nd);
    return LYM_ERR_UNSUPPORTED;
  }
  LYM_REQUIRE(lat->nd != 3 || !herm, LYM_ERR_UNSUPPORTED,
              "three dimensions have no hermitian form gamma_d D (two-component spinors, no gamma_5)");
  LYM_REQUIRE(nc == 2 || nc == 3, LYM_ERR_UNSUPPORTED, "N=%d not supported (2 or 3)", nc);
  if (lat->nd == 3 && nc == 2) return launch_full<3, 2>(lat, kappa, 0, bcr, bci, gauge, nvec, in, out, st);
  if (lat->nd == 3 && nc == 3) return launch_full<3, 3>(lat, kappa, 0, bcr, bci, gauge, nvec, in, out, st);
  if (lat->nd == 2 && nc == 2) return launch_full<2, 2>(lat, kappa, herm, bcr, bci, gauge, nvec, in, out, st);
  if (lat->nd == 2 && nc == 3) return launch_full<2, 3>(lat, kappa, herm, bcr, bci, gauge, nvec, in, out, st);
  if (lat->nd == 4 && nc == 2) return launch_full<4, 2>(lat, kappa, herm, bcr, bci, gauge, nvec, in, out, st);
  return launch_full<4, 3>(lat, kappa, herm, bcr, bci, gauge, nvec, in, out, st);
}

// ---------------------------------------------------------------------------
// vector algebra, complex128
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) cdot_kernel(int64_t n, const double2* __restrict__ a,
                                                   const double2* __restrict__ b, double* partials,
                                                   unsigned* counter, double* result) {
  __shared__ double sh[2 * 32];
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 x = a[i], y = b[i];
    v[0] += x.x * y.x + x.y * y.y;
    v[1] += x.x * y.y - x.y * y.x;
  }
  if (grid_sum<2>(v, partials, counter, sh) && threadIdx.x == 0) {
    result[0] = v[0];
    result[1] = v[1];
  }
}

__global__ void caxpby_kernel(int64_t n, double ar, double ai, const double2* __restrict__ x, double br,
                              double bi, double2* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 xv = x[i], yv = y[i];
    y[i] = make_double2(ar * xv.x - ai * xv.y + br * yv.x - bi * yv.y,
                        ar * xv.y + ai * xv.x + br * yv.y + bi * yv.x);
  }
}

unsigned reduction_blocks(int64_t n, int block) {
  int64_t b = (n + block - 1) / block;
  if (b > Scratch::kMaxBlocks) b = Scratch::kMaxBlocks;
  if (b < 1) b = 1;
  return (unsigned)b;
}

int cdot_device(int64_t n, const void* a, const void* b, double* result_dev, int slot, cudaStream_t st) {
  Scratch* s;
  int rc = scratch_get(&s);
  if (rc) return rc;
  unsigned nb = reduction_blocks(n, 256);
  cdot_kernel<<<nb, 256, 0, st>>>(n, (const double2*)a, (const double2*)b,
                                   s->partials + (size_t)slot * Scratch::kMaxBlocks * Scratch::kMaxVals,
                                   s->counters + slot, result_dev);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

}  // namespace lym

using namespace lym;

extern "C" {

int lym_wilson_apply(const lym_lattice* lat, int nc, double kappa, int hermitian, double bc_re, double bc_im,
                     const void* gauge, const void* in, void* out, void* stream) {
  return wilson_full(lat, nc, kappa, hermitian, bc_re, bc_im, gauge, 1, in, out, (cudaStream_t)stream);
}

int lym_wilson_apply_batch(const lym_lattice* lat, int nc, double kappa, int hermitian, double bc_re,
                           double bc_im, const void* gauge, int nvec, const void* in, void* out, void* stream) {
  return wilson_full(lat, nc, kappa, hermitian, bc_re, bc_im, gauge, nvec, in, out, (cudaStream_t)stream);
}

int lym_cdot(int64_t n, const void* a, const void* b, double* result, void* stream) {
  LYM_REQUIRE(n >= 0 && a && b && result, LYM_ERR_BAD_ARG, "null argument");
  Scratch* s;
  int rc = scratch_get(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lk(host_reduce_mutex());
  const int slot = 1;
  rc = cdot_device(n, a, b, s->results + slot * Scratch::kMaxVals, slot, st);
  if (rc) return rc;
  LYM_CUDA(cudaMemcpyAsync(s->host + slot * Scratch::kMaxVals, s->results + slot * Scratch::kMaxVals,
                           2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  result[0] = s->host[slot * Scratch::kMaxVals];
  result[1] = s->host[slot * Scratch::kMaxVals + 1];
  return LYM_OK;
}

int lym_caxpby(int64_t n, const double* a, const void* x, const double* b, void* y, void* stream) {
  LYM_REQUIRE(n >= 0 && a && b && x && y, LYM_ERR_BAD_ARG, "null argument");
  if (n == 0) return LYM_OK;
  unsigned nb = reduction_blocks(n, 256) * 4;
  caxpby_kernel<<<nb, 256, 0, (cudaStream_t)stream>>>(n, a[0], a[1], (const double2*)x, b[0], b[1],
                                                      (double2*)y);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

}  // extern "C"
