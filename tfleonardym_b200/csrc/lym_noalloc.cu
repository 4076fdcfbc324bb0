// Batched dot products that allocate nothing: the reduction scratch lives in
// a fixed file-scope device array instead of library-allocated memory.
//
// Who needs this: code that runs where another allocator owns the device
// memory -- a deep-learning framework's pooling allocator (TensorFlow's, for
// the reference's own host) or a service with a fixed device-memory budget --
// cannot call cudaMalloc: the allocation would bypass the owner's accounting,
// can fail once the pool has taken the free memory, and costs a device
// synchronisation.  The caller passes inputs and outputs; everything else this
// entry point touches is the static array below.
#include <mutex>

#include "lym_internal.cuh"
#include "lym_kernels.cuh"

namespace lym {

constexpr int kNoAllocMaxVec = 64;   // vectors per call
constexpr int kNoAllocBlocks = 256;  // partial sums per vector

struct NoAllocScratch {
  double partials[kNoAllocMaxVec][kNoAllocBlocks][2];
  unsigned counters[kNoAllocMaxVec];
  double results[kNoAllocMaxVec][2];
};

// Every GPU that loads the library holds this (about 263 KB) until the process exits.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// The batched form of cdot_kernel (lym_wilson.cu): blockIdx.y selects the vector pair.
__global__ void __launch_bounds__(256) cdot_batch_kernel(int64_t n, const double2* __restrict__ a,
                                                         const double2* __restrict__ b, NoAllocScratch* s) {
  __shared__ double sh[2 * 32];
  const int v = blockIdx.y;
  const double2* av = a + (int64_t)v * n;
  const double2* bv = b + (int64_t)v * n;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 x = av[i], y = bv[i];
    acc[0] += x.x * y.x + x.y * y.y;
    acc[1] += x.x * y.y - x.y * y.x;
  }
  if (grid_sum<2>(acc, &s->partials[v][0][0], &s->counters[v], sh) && threadIdx.x == 0) {
    s->results[v][0] = acc[0];
    s->results[v][1] = acc[1];
  }
}

static std::mutex g_noalloc_mu;
static NoAllocScratch* g_noalloc_ptr[64];

// Device address of the static scratch for the current device, looked up once
// per device with that device current (host code cannot use the symbol itself).
static int noalloc_scratch(NoAllocScratch** out) {
  int dev = 0;
  LYM_CUDA(cudaGetDevice(&dev));
  LYM_REQUIRE(dev >= 0 && dev < 64, LYM_ERR_BAD_ARG, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    NoAllocScratch* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("cudaGetSymbolAddress of the static dot-product scratch: %s", cudaGetErrorString(e));
      return LYM_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return LYM_OK;
}

}  // namespace lym

using namespace lym;

extern "C" int lym_cdot_batch_noalloc(int nvec, int64_t n, const void* a, const void* b, double* results,
                                      void* stream) {
  LYM_REQUIRE(a && b && results && n >= 0, LYM_ERR_BAD_ARG, "null argument or negative length");
  LYM_REQUIRE(nvec >= 1 && nvec <= kNoAllocMaxVec, LYM_ERR_BAD_ARG,
              "nvec=%d is outside [1, %d]: the static scratch of lym_cdot_batch_noalloc holds %d vectors",
              nvec, kNoAllocMaxVec, kNoAllocMaxVec);
  NoAllocScratch* s;
  int rc = noalloc_scratch(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // the completion counters must start at zero; a call that failed mid-way may have left one set
  LYM_CUDA(cudaMemsetAsync(s->counters, 0, sizeof(s->counters), st));
  int64_t nb = (n + 255) / 256;
  if (nb > kNoAllocBlocks) nb = kNoAllocBlocks;
  if (nb < 1) nb = 1;
  cdot_batch_kernel<<<dim3((unsigned)nb, (unsigned)nvec), 256, 0, st>>>(n, (const double2*)a, (const double2*)b, s);
  LYM_CHECK_LAUNCH();
  LYM_CUDA(cudaMemcpyAsync(results, s->results, sizeof(double) * 2 * nvec, cudaMemcpyDeviceToHost, st));
  LYM_CUDA(cudaStreamSynchronize(st));
  return LYM_OK;
}
