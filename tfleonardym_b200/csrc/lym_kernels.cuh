// Internal entry points shared between the lym translation units.
#pragma once

#include <mutex>

#include "lym_internal.cuh"

namespace lym {

// Reference-layout FP64 Wilson operator on nvec spinors (lym_wilson.cu).
int wilson_full(const lym_lattice* lat, int nc, double kappa, int herm, double bcr, double bci,
                const void* gauge, int nvec, const void* in, void* out, cudaStream_t st);

// Blocks for a grid reduction over n items (capped at Scratch::kMaxBlocks).
unsigned reduction_blocks(int64_t n, int block);

// sum conj(a) b into result_dev[0..1] using scratch slot `slot`.
int cdot_device(int64_t n, const void* a, const void* b, double* result_dev, int slot, cudaStream_t st);

// Serialises the entry points that return host scalars through scratch slot 1.
std::mutex& host_reduce_mutex();

// Read-only view of a lym_gauge's reference-layout copy (lym_solver.cu).
struct GaugeView {
  const lym_lattice* lat;
  int nc, ncomp;
  int64_t V;
  double bcr, bci;
  const double2* uref;
};
int gauge_view(const lym_gauge* g, GaugeView* v);


}  // namespace lym
