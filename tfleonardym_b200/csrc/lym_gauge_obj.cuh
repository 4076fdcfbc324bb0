// The lym_gauge object (links packed for the even-odd solvers) and the CUDA
// graph recorder, shared by the even-odd CG (lym_solver.cu) and the
// even-odd multishift CG (lym_mshift.cu).
#pragma once

#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "lym_eo.cuh"

namespace lym {
struct Work;
struct MsWork;
}  // namespace lym

struct lym_gauge {
  const lym_lattice* lat = nullptr;
  int nc = 0, nd = 0, ns = 0, ncomp = 0;
  int64_t V = 0, Vh = 0;
  double bcr = 1, bci = 0;
  unsigned prec_mask = 0;
  bool comp = false;  // sloppy links compressed (links are SU(N))
  lym::EoGeom geom{};
  double2* uref = nullptr;  // reference-layout FP64 copy (boundary factor NOT applied)
  double2* u64 = nullptr;
  // sloppy links: compressed to N-1 rows (only when every link is SU(N)) and full N x N
  float4* u32 = nullptr;   // compressed
  int n32 = 0;
  uint2* u16 = nullptr;    // compressed
  int n16 = 0;
  float4* u32f = nullptr;  // full, boundary factor folded in
  int n32f = 0;
  uint2* u16f = nullptr;   // full, boundary factor folded in
  int n16f = 0;
  int* nbr = nullptr;      // even-odd neighbour table (EoGeom::nbr)
  std::vector<lym::Work*> works;      // CG workspaces, most recently used first
  std::vector<lym::MsWork*> ms_works; // multishift workspaces, most recently used first
  // Held for the whole of every call that uses or changes the workspaces or the
  // packed links (solves, lym_dslash_eo, lym_gauge_update): two host threads that
  // share a gauge object take turns instead of sharing one workspace's stream,
  // pinned state buffers and graphs.
  std::recursive_mutex mu;
};

namespace lym {

// Frees the multishift workspaces of a gauge object (lym_mshift.cu); called
// when its links are repacked and when it is destroyed.
void free_ms_works(lym_gauge* g);

// Records kernel launches as the nodes of a CUDA graph, each after the
// previous one, instead of stream capture: nothing is ever capturing, so
// another thread's first launch of a lazily loaded kernel (a library or a
// torch kernel) cannot collide with a capture in progress.
struct GraphRec {
  cudaGraph_t graph = nullptr;      // graph being recorded; null: launch directly
  cudaGraphNode_t last = nullptr;   // its last node
  cudaError_t err = cudaSuccess;    // first error while adding nodes
};

// smem: dynamic shared memory bytes of the launch
template <typename... KArgs, typename... Args>
inline void launch_rec_smem(GraphRec& rec, cudaStream_t st, void (*kernel)(KArgs...), dim3 grid, dim3 block,
                            size_t smem, Args&&... args) {
  if (!rec.graph) {
    kernel<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    return;
  }
  std::tuple<KArgs...> vals(std::forward<Args>(args)...);
  void* ptrs[sizeof...(KArgs)];
  std::apply([&](auto&... v) {
    int i = 0;
    ((ptrs[i++] = (void*)&v), ...);
  }, vals);
  cudaKernelNodeParams p{};
  p.func = (void*)kernel;
  p.gridDim = grid;
  p.blockDim = block;
  p.sharedMemBytes = (unsigned)smem;
  p.kernelParams = ptrs;
  cudaGraphNode_t node = nullptr;
  const cudaError_t e = cudaGraphAddKernelNode(&node, rec.graph, rec.last ? &rec.last : nullptr,
                                               rec.last ? 1 : 0, &p);
  if (e != cudaSuccess && rec.err == cudaSuccess) rec.err = e;
  if (e == cudaSuccess) rec.last = node;
}

template <typename... KArgs, typename... Args>
inline void launch_rec(GraphRec& rec, cudaStream_t st, void (*kernel)(KArgs...), dim3 grid, dim3 block,
                       Args&&... args) {
  launch_rec_smem(rec, st, kernel, grid, block, 0, std::forward<Args>(args)...);
}

}  // namespace lym
