// Lattice runtime: neighbour tables, boundary field, device lattice object.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "lym_internal.cuh"

namespace lym {

thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int check_dims(int nd, const int64_t* dims, int64_t* volume) {
  LYM_REQUIRE(nd >= 1 && nd <= LYM_MAX_ND && dims != nullptr, LYM_ERR_BAD_ARG,
              "nd must be in [1, %d] and dims non-null", LYM_MAX_ND);
  int64_t v = 1;
  for (int i = 0; i < nd; ++i) {
    LYM_REQUIRE(dims[i] >= 1 && dims[i] < (1 << 20), LYM_ERR_BAD_ARG, "bad extent %lld",
                (long long)dims[i]);
    v *= dims[i];
  }
  LYM_REQUIRE(v < (int64_t(1) << 31), LYM_ERR_BAD_ARG, "volume %lld too large", (long long)v);
  *volume = v;
  return LYM_OK;
}

// Tables of lattice.py:86-120: site index s = Horner(x_0, ..., x_{nd-1}) with
// the last coordinate fastest; sup[mu][s] / sdn[mu][s] = index of x +- mu-hat
// with periodic wrap.  Written out here as a direct odometer over the sites.
void build_tables(int nd, const int64_t* dims, int64_t V, int64_t* sup, int64_t* sdn,
                  int64_t* coords) {
  std::vector<int64_t> stride(nd);
  int64_t st = 1;
  for (int mu = nd - 1; mu >= 0; --mu) {
    stride[mu] = st;
    st *= dims[mu];
  }
  std::vector<int64_t> x(nd, 0);
  for (int64_t s = 0; s < V; ++s) {
    for (int mu = 0; mu < nd; ++mu) {
      if (coords) coords[mu * V + s] = x[mu];
      int64_t up = (x[mu] + 1 == dims[mu]) ? s - (dims[mu] - 1) * stride[mu] : s + stride[mu];
      int64_t dn = (x[mu] == 0) ? s + (dims[mu] - 1) * stride[mu] : s - stride[mu];
      if (sup) sup[mu * V + s] = up;
      if (sdn) sdn[mu * V + s] = dn;
    }
    for (int mu = nd - 1; mu >= 0; --mu) {  // odometer increment, last fastest
      if (++x[mu] < dims[mu]) break;
      x[mu] = 0;
    }
  }
}

}  // namespace lym

using namespace lym;

extern "C" {

int lym_version(void) { return 10000; }

const char* lym_last_error(void) { return g_last_error; }

const char* lym_status_string(int s) {
  switch (s) {
    case LYM_OK: return "ok";
    case LYM_ERR_BAD_ARG: return "bad argument";
    case LYM_ERR_BAD_SHAPE: return "incompatible shapes";
    case LYM_ERR_UNSUPPORTED: return "unsupported";
    case LYM_ERR_NOT_CONVERGED: return "not converged";
    case LYM_ERR_CUDA: return "cuda error";
    case LYM_ERR_OOM: return "out of device memory";
    case LYM_ERR_REJECTED: return "rejected";
    case LYM_ERR_TIMEOUT: return "timeout";
    default: return "unknown status";
  }
}

int lym_lookup_tables(int nd, const int64_t* dims, int64_t* sup, int64_t* sdn, int64_t* coords) {
  int64_t V;
  int st = check_dims(nd, dims, &V);
  if (st) return st;
  LYM_REQUIRE(sup || sdn || coords, LYM_ERR_BAD_ARG, "no output requested");
  build_tables(nd, dims, V, sup, sdn, coords);
  return LYM_OK;
}

int lym_antiperiodic_field(int nd, const int64_t* dims, double fre, double fim, double* field) {
  int64_t V;
  int st = check_dims(nd, dims, &V);
  if (st) return st;
  LYM_REQUIRE(field != nullptr, LYM_ERR_BAD_ARG, "field is null");
  const int64_t L = dims[nd - 1];
  for (int64_t s = 0; s < V; ++s) {
    bool last = (s % L) == L - 1;  // last coordinate is the fastest index
    field[2 * s] = last ? fre : 1.0;
    field[2 * s + 1] = last ? fim : 0.0;
  }
  return LYM_OK;
}

int lym_lattice_create(int nd, const int64_t* dims, lym_lattice** out) {
  LYM_REQUIRE(out != nullptr, LYM_ERR_BAD_ARG, "out is null");
  int64_t V;
  int st = check_dims(nd, dims, &V);
  if (st) return st;
  std::vector<int64_t> sup(nd * V), sdn(nd * V);
  build_tables(nd, dims, V, sup.data(), sdn.data(), nullptr);
  std::vector<int32_t> tab(2 * nd * V);
  for (int64_t i = 0; i < nd * V; ++i) {
    tab[i] = (int32_t)sup[i];
    tab[nd * V + i] = (int32_t)sdn[i];
  }
  lym_lattice* lat = new lym_lattice();
  lat->nd = nd;
  lat->V = V;
  lat->even = true;
  for (int i = 0; i < LYM_MAX_ND; ++i) lat->dims[i] = i < nd ? (int)dims[i] : 1;
  for (int i = 0; i < nd; ++i) lat->even = lat->even && (dims[i] % 2 == 0);
  cudaGetDevice(&lat->device);
  cudaError_t e = cudaMalloc(&lat->d_tab, sizeof(int32_t) * tab.size());
  if (e != cudaSuccess) {
    delete lat;
    set_error("cudaMalloc tables: %s", cudaGetErrorString(e));
    return LYM_ERR_OOM;
  }
  e = cudaMemcpy(lat->d_tab, tab.data(), sizeof(int32_t) * tab.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(lat->d_tab);
    delete lat;
    set_error("cudaMemcpy tables: %s", cudaGetErrorString(e));
    return LYM_ERR_CUDA;
  }
  *out = lat;
  return LYM_OK;
}

int lym_lattice_destroy(lym_lattice* lat) {
  if (!lat) return LYM_OK;
  if (lat->d_tab) cudaFree(lat->d_tab);
  delete lat;
  return LYM_OK;
}

}  // extern "C"

namespace {
__global__ void widen_tables(const int32_t* __restrict__ t, int64_t n, int64_t* __restrict__ sup,
                             int64_t* __restrict__ sdn) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) {
    sup[i] = t[i];
    sdn[i] = t[n + i];
  }
}
}  // namespace

extern "C" int lym_lattice_tables_device(const lym_lattice* lat, int64_t* sup_dev, int64_t* sdn_dev,
                                         void* stream) {
  LYM_REQUIRE(lat && sup_dev && sdn_dev, LYM_ERR_BAD_ARG, "null argument");
  int64_t n = (int64_t)lat->nd * lat->V;
  widen_tables<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(lat->d_tab, n, sup_dev, sdn_dev);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}

// ---------------------------------------------------------------------------
// on-disk gauge format (lattice.py:10-70): decode on the device
// ---------------------------------------------------------------------------
namespace lym {

// One thread per (site, mu): 12 big-endian float32 words (the first two
// columns of conj(U), re/im) -> U in the reference layout (nd, 3, 3, V).  Column
// 0 is normalised, column 1 orthogonalised against it and normalised, column 2 =
// conj(col0 x col1): the reference's steps in its order, FP64, |z|^2 as
// hypot(re, im)^2 like the reference's abs(z)**2.
__global__ void __launch_bounds__(128) xdr_su3_kernel(int nd, int64_t V, const unsigned* __restrict__ raw,
                                                      double2* __restrict__ out) {
  const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (x >= V) return;
  // the link's 48-byte record as three 16-byte loads (records start 16-byte aligned)
  const uint4* w4 = reinterpret_cast<const uint4*>(raw + (x * nd + mu) * 12);
  unsigned w[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint4 t = __ldg(w4 + k);
    w[4 * k] = t.x;
    w[4 * k + 1] = t.y;
    w[4 * k + 2] = t.z;
    w[4 * k + 3] = t.w;
  }
  cx<double> c[3][2];  // c[row][col] of conj-stored values, conjugated back
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float re = __uint_as_float(__byte_perm(w[2 * k], 0, 0x0123));
    const float im = __uint_as_float(__byte_perm(w[2 * k + 1], 0, 0x0123));
    c[k / 2][k % 2] = {(double)re, -(double)im};  // word order: row, column, re/im
  }
  auto a2 = [](cx<double> z) {
    const double h = hypot(z.re, z.im);
    return h * h;
  };
  cx<double> u[3][3];
  double t = 1.0 / sqrt(a2(c[0][0]) + a2(c[1][0]) + a2(c[2][0]));
#pragma unroll
  for (int i = 0; i < 3; ++i) u[i][0] = t * c[i][0];
  cx<double> p = c[0][1] * conj(u[0][0]) + c[1][1] * conj(u[1][0]) + c[2][1] * conj(u[2][0]);
#pragma unroll
  for (int i = 0; i < 3; ++i) u[i][1] = c[i][1] - p * u[i][0];
  t = 1.0 / sqrt(a2(u[0][1]) + a2(u[1][1]) + a2(u[2][1]));
#pragma unroll
  for (int i = 0; i < 3; ++i) u[i][1] = t * u[i][1];
  u[0][2] = conj(u[1][0]) * conj(u[2][1]) - conj(u[2][0]) * conj(u[1][1]);
  u[1][2] = conj(u[2][0]) * conj(u[0][1]) - conj(u[0][0]) * conj(u[2][1]);
  u[2][2] = conj(u[0][0]) * conj(u[1][1]) - conj(u[1][0]) * conj(u[0][1]);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) out[((int64_t)(mu * 3 + i) * 3 + j) * V + x] = make_double2(u[i][j].re, u[i][j].im);
}

}  // namespace lym

extern "C" int lym_decode_xdr_gauge(int nd, int nc, int64_t volume, const void* raw, void* gauge, void* stream) {
  using namespace lym;
  LYM_REQUIRE(raw && gauge && nd >= 1 && nd <= LYM_MAX_ND && volume >= 0, LYM_ERR_BAD_ARG, "bad argument");
  LYM_REQUIRE(nc == 3, LYM_ERR_UNSUPPORTED, "the XDR format holds SU(3) links (N=%d given)", nc);
  LYM_REQUIRE(((uintptr_t)raw & 15) == 0, LYM_ERR_BAD_ARG, "raw words must be 16-byte aligned");
  if (volume == 0) return LYM_OK;
  dim3 grid(grid_for(volume, 128), nd);
  xdr_su3_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(nd, volume, (const unsigned*)raw, (double2*)gauge);
  LYM_CHECK_LAUNCH();
  return LYM_OK;
}
