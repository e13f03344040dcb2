// Hot scatter targets: the successors that receive a large share of all arcs.  With preferential
// in-degrees a few vertices are the successor of several percent of the arcs (on the 2M/40M graph
// one vertex receives 6.6% of them, 2.6M per pass), and a sweep that scatters one atomic add per
// arc sends millions of them to one L2 slice per pass.  Each block of a scatter sweep keeps
// block-local partial sums for the hot targets in shared memory and adds them to the global vector
// once per block at its end; every other target takes the global atomic directly.
//
// The set is chosen once at load (build_hot, engine.cu): the kHotMax vertices with the largest
// in-degree (counted over all arcs by k_in_degree), those with at least kHotMinShare of the arcs,
// placed in a direct-mapped table of kHotSlots ids indexed by a multiplicative hash (a vertex whose
// slot is taken by a hotter one stays on the global path).
#pragma once
#include "lean.cuh"

namespace tga {

constexpr int kHotSlots = 512;      // table size (power of two)
constexpr int kHotMax = 64;         // hot targets at most
constexpr int kHotMinShare = 4096;  // a hot target receives at least arcs / kHotMinShare arcs

__host__ __device__ __forceinline__ int hot_slot(int32_t y) { return (int)(((uint32_t)y * 0x9E3779B1u) >> 23); }

// Block-local partial sums of the hot targets (T: the type of the per-block partials; Out: the
// type of the global vector they are added to).  init() and flush() are block-wide and must be
// reached by every thread of the block.
template <class T>
struct HotAcc {
  int32_t* ids;  // shared: kHotSlots ids (-1 empty)
  T* acc;        // shared: kHotSlots partials

  __device__ __forceinline__ void init(const GraphView& g) {
    for (int s = threadIdx.x; s < kHotSlots; s += blockDim.x) {
      ids[s] = g.hot ? __ldg(g.hot + s) : -1;
      acc[s] = T(0);
    }
    __syncthreads();
  }
  // Adds v to y's partial if y is hot; false if y takes the global path.
  __device__ __forceinline__ bool add(int32_t y, T v) {
    const int s = hot_slot(y);
    if (ids[s] != y) return false;
    atomicAdd(&acc[s], v);
    return true;
  }
  template <class Out>
  __device__ __forceinline__ void flush(Out* out) {
    __syncthreads();
    for (int s = threadIdx.x; s < kHotSlots; s += blockDim.x)
      if (acc[s] != T(0)) atomicAdd(&out[ids[s]], (Out)acc[s]);
  }
};

#define TGA_HOT_SHARED(T, name)                         \
  __shared__ int32_t name##_ids[kHotSlots];              \
  __shared__ T name##_acc[kHotSlots];                    \
  HotAcc<T> name{name##_ids, name##_acc};

// In-degree of every vertex, counted over all arcs (one pass over the lean schedule at load).
static __global__ void TGA_LEAN_BOUNDS k_in_degree(GraphView g, LeanWork lw, int32_t* indeg) {
  run_lean<false, false>(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int) { return true; }, [&](int, int, int) { return true; },
      [&](int, int y, int64_t) {
        atomicAdd(&indeg[y], 1);
        return true;
      },
      [&](int) {});
}

}  // namespace tga
