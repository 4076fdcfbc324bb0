// Internal structures and device utilities shared by the lym translation units.
#pragma once

#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "lym_common.cuh"

#define LYM_MAX_ND 4

struct lym_lattice {
  int nd = 0;
  int dims[LYM_MAX_ND] = {1, 1, 1, 1};
  int64_t V = 0;
  bool even = false;    // every extent even: even-odd ordering available
  int device = 0;
  int32_t* d_tab = nullptr;  // [sup (nd, V) | sdn (nd, V)]
};

namespace lym {

int check_dims(int nd, const int64_t* dims, int64_t* volume);
void build_tables(int nd, const int64_t* dims, int64_t V, int64_t* sup, int64_t* sdn, int64_t* coords);

// Per-device scratch owned by the library (reduction partials and counters).
struct Scratch {
  double* partials = nullptr;   // kMaxBlocks * kMaxVals doubles per slot
  unsigned* counters = nullptr; // one counter per slot, kept at zero between uses
  double* results = nullptr;    // kMaxVals doubles per slot
  double* host = nullptr;       // pinned mirror of results
  static constexpr int kMaxBlocks = 1184;  // 8 x 148 SMs
  static constexpr int kMaxVals = 4;
  static constexpr int kSlots = 256;
};
int scratch_get(Scratch** out);

// ---------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------
LYM_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum NV values over the block; result valid in thread 0.  `sh` must hold
// NV * 32 doubles.  Fixed reduction tree: bit-reproducible for a fixed block size.
template <int NV>
LYM_D void block_sum(double (&v)[NV], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double w = warp_sum(v[k]);
    if (lane == 0) sh[k * 32 + warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double w = lane < nwarps ? sh[k * 32 + lane] : 0.0;
      v[k] = warp_sum(w);
    }
  }
  __syncthreads();
}

// Two-stage grid reduction with the "last block finishes" pattern.  Each block
// of a grid (gridDim.x blocks along x, one slot per blockIdx.y) stores its
// partial; the block that arrives last sums all partials in block order and
// returns true in every thread of that block, with the totals in `v`
// (thread 0) -- the caller then writes results.  No block ever waits for
// another, so there is no spin loop.
// grid_sum_n: the same for a slot of nb blocks numbered blk (several slots
// may share one launch, e.g. the lattices of a multi-lattice launch).
template <int NV>
LYM_D bool grid_sum_n(double (&v)[NV], double* partials, unsigned* counter, double* sh, int blk, int nb) {
  __shared__ bool last;
  block_sum<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[blk * NV + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    last = (t == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += ((volatile double*)partials)[b * NV + k];
  }
  block_sum<NV>(acc, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = acc[k];
    *counter = 0u;  // ready for the next use of this slot
  }
  return true;
}

template <int NV>
LYM_D bool grid_sum(double (&v)[NV], double* partials, unsigned* counter, double* sh) {
  return grid_sum_n<NV>(v, partials, counter, sh, blockIdx.x, gridDim.x);
}

LYM_D cx<double> ld(const double2* p) {
  double2 t = __ldg(p);
  return {t.x, t.y};
}
LYM_D void st(double2* p, cx<double> v) { *p = make_double2(v.re, v.im); }

}  // namespace lym
