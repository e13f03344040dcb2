// Hot scatter targets: the successors that receive a large share of all arcs.  With preferential
// in-degrees a few vertices are the successor of several percent of the arcs (on the 2M/40M graph
// one vertex receives 6.6% of them, 2.6M per pass), and a sweep that scatters one atomic add per
// arc sends millions of them to one L2 slice per pass.  Each block of a scatter sweep keeps
// block-local partial sums for the hot targets in shared memory and adds them to the global vector
// once per block at its end; every other target takes the global atomic directly.  Traversals
// read the arrival (and frontier bits) of a hot successor before relaxing it: after its first
// levels its arrival is rarely lowered, and the atomic that would change nothing is not sent.
//
// The set is chosen once at load (build_hot, algos.cu): the kHotMax vertices with the largest
// in-degree (counted over all arcs by k_in_degree), those with at least kHotMinShare of the arcs,
// placed in a direct-mapped table of kHotSlots ids indexed by a multiplicative hash (a vertex whose
// slot is taken by a hotter one stays on the global path).  The device table holds the ids
// (kHotSlots int32, -1 empty) followed by each slot's compact index (kHotSlots int32, 0..kHotMax-1),
// which numbers the partials.
#pragma once
#include "lean.cuh"

namespace tga {

constexpr int kHotSlots = 512;      // table size (power of two)
constexpr int kHotMax = 64;         // hot targets at most
constexpr int kHotMinShare = 4096;  // a hot target receives at least arcs / kHotMinShare arcs

__host__ __device__ __forceinline__ int hot_slot(int32_t y) { return (int)(((uint32_t)y * 0x9E3779B1u) >> 23); }

// The hot ids into shared memory (ids[kHotSlots]), and with idx their compact indexes
// (idx[kHotSlots]); the caller synchronises the block.
__device__ __forceinline__ void hot_load(const GraphView& g, int32_t* ids, int32_t* idx = nullptr) {
  for (int s = threadIdx.x; s < kHotSlots; s += blockDim.x) {
    ids[s] = g.hot ? __ldg(g.hot + s) : -1;
    if (idx) idx[s] = g.hot ? __ldg(g.hot + kHotSlots + s) : 0;
  }
}
__device__ __forceinline__ bool hot_is(const int32_t* ids, int32_t y) { return ids[hot_slot(y)] == y; }
// Compact index of y if y is hot, else -1.
__device__ __forceinline__ int hot_index(const int32_t* ids, const int32_t* idx, int32_t y) {
  const int s = hot_slot(y);
  return ids[s] == y ? idx[s] : -1;
}

// Block-local partial sums of the hot targets (T: the type of the per-block partials; Out: the
// type of the global vector they are added to).  init() and flush() are block-wide and must be
// reached by every thread of the block.
template <class T>
struct HotAcc {
  int32_t* ids;  // shared: kHotSlots ids (-1 empty)
  int32_t* idx;  // shared: kHotSlots compact indexes
  T* acc;        // shared: kHotMax partials

  __device__ __forceinline__ void init(const GraphView& g) {
    hot_load(g, ids, idx);
    for (int s = threadIdx.x; s < kHotMax; s += blockDim.x) acc[s] = T(0);
    __syncthreads();
  }
  // Adds v to y's partial if y is hot; false if y takes the global path.
  __device__ __forceinline__ bool add(int32_t y, T v) {
    const int k = hot_index(ids, idx, y);
    if (k < 0) return false;
    atomicAdd(&acc[k], v);
    return true;
  }
  template <class Out>
  __device__ __forceinline__ void flush(Out* out) {
    __syncthreads();
    for (int s = threadIdx.x; s < kHotSlots; s += blockDim.x)
      if (ids[s] >= 0 && acc[idx[s]] != T(0)) atomicAdd(&out[ids[s]], (Out)acc[idx[s]]);
  }
};

#define TGA_HOT_SHARED(T, name)                         \
  __shared__ int32_t name##_ids[kHotSlots];              \
  __shared__ int32_t name##_idx[kHotSlots];              \
  __shared__ T name##_acc[kHotMax];                      \
  HotAcc<T> name{name##_ids, name##_idx, name##_acc};

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
