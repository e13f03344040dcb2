// Pieces shared by the kernels that run many levels in one cooperative launch (traversals and
// batched traversals): the launch control block, a time-bounded grid barrier, and warp-aggregated
// queue appends.
#pragma once
#include "sweep.cuh"

namespace tga {

constexpr uint64_t kBarrierNs = 10ull * 1000 * 1000 * 1000;  // longest wait at a grid barrier

// Control block of one launch (zeroed by the host before the launch, best = INT32_MAX).
struct TravCtl {
  int32_t cnt[3];        // queue lengths (rotating, see above)
  int32_t next[3];       // work counters of the levels (same rotation)
  uint32_t bar_count;    // grid barrier: blocks arrived
  uint32_t bar_gen;      // grid barrier: generation
  int32_t status;        // nonzero: a barrier wait ran out
  int32_t levels;        // levels executed
  int32_t tcnt;          // CC: vertices whose arrival became finite for the current seed
  int32_t best;          // CC: seed search minimum
  int32_t comps;         // CC: components
  int32_t dcnt[3];       // multi-source: wide queue lengths (same rotation as cnt)
  int32_t dnext[3];      // multi-source: wide queue work counters
  int32_t yield;         // batched CC: the launch's time budget ran out (stop at this batch)
  int32_t batches;       // batched CC: batches run by the launch
};
// The host reads the block back into a 128-byte slot of its pinned area.
static_assert(sizeof(TravCtl) <= 128, "TravCtl outgrew its pinned readback slot");

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier over all blocks of the cooperative launch; false if the launch has failed (this block
// must return at once).  A wait longer than limit_ns sets ctl->status and the kErrTimeout bit of
// *err, and every block leaves at its next barrier.
static __device__ bool grid_sync_limit(TravCtl* ctl, uint32_t* err, uint64_t limit_ns) {
  __shared__ int failed;
  __syncthreads();
  if (threadIdx.x == 0) {
    failed = 0;
    volatile uint32_t* gen = &ctl->bar_gen;
    volatile int32_t* status = &ctl->status;
    const uint32_t mine = *gen;
    __threadfence();
    if (atomicAdd(&ctl->bar_count, 1u) == gridDim.x - 1) {
      ctl->bar_count = 0;
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    } else {
      const uint64_t t0 = global_ns();
      for (uint32_t spin = 0; *gen == mine; ++spin) {
        if (*status) {
          failed = 1;
          break;
        }
        if ((spin & 255u) == 255u && global_ns() - t0 > limit_ns) {
          atomicExch(&ctl->status, 1);
          atomicOr(err, kErrTimeout);
          failed = 1;
          break;
        }
        __nanosleep(100);
      }
    }
    if (*status) failed = 1;
    __threadfence();
  }
  __syncthreads();
  return !failed;
}

static __device__ __forceinline__ bool grid_sync(TravCtl* ctl, const GraphView& g) {
  return grid_sync_limit(ctl, g.err, kBarrierNs);
}

// Reserves n slots per lane with one atomic per warp (all 32 lanes must call it together); returns
// this lane's first slot.
__device__ __forceinline__ int warp_reserve(int32_t* cnt, int n) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int incl = n;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(full, incl, 31);
  int base = 0;
  if (lane == 31 && total) base = atomicAdd(cnt, total);
  base = __shfl_sync(full, base, 31);
  return base + incl - n;
}

// Entries of vertex v in a queue: v itself or all its slices.
// Deals the vertices marked in 32 words of a dirty bitmap (lane l holds word base + l, already
// loaded into `bits`) one per lane, in rounds of 32, so that a word with many marked vertices does
// not leave one lane to process them all while the others wait: fn(v) is called by every lane of
// the warp in every round (all 32 lanes must call deal_dirty together), with v = -1 for a lane
// that has no vertex in that round.  Marked vertex idx (in word order) belongs to the first lane
// whose inclusive count exceeds idx, at rank idx - (that lane's exclusive count) among its bits.
template <class Fn>
__device__ __forceinline__ void deal_dirty(uint32_t bits, int base, Fn fn) {
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int cnt = __popc(bits);
  int incl = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += u;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  for (int j0 = 0; j0 < total; j0 += 32) {
    const int idx = j0 + lane;
    int owner = 0;  // lanes whose inclusive count is <= idx
    for (int step = 16; step; step >>= 1) {
      const int probe = __shfl_sync(kFull, incl, owner + step - 1);
      if (probe <= idx) owner += step;
    }
    owner = min(owner, 31);
    uint32_t w = __shfl_sync(kFull, bits, owner);
    int r = idx - (__shfl_sync(kFull, incl, owner) - __shfl_sync(kFull, cnt, owner));
    int pos = 0;  // the r-th (0-based) set bit of w
    for (int width = 16; width; width >>= 1) {
      const int c = __popc(w & ((1u << width) - 1));
      if (r >= c) {
        r -= c;
        w >>= width;
        pos += width;
      }
    }
    fn(idx < total ? (base + owner) * 32 + pos : -1);
  }
}

__device__ __forceinline__ int entry_count(const Work& w, int v) {
  const int n = __ldg(w.slice_first + v + 1) - __ldg(w.slice_first + v);
  return n ? n : 1;
}
__device__ __forceinline__ void write_entries(const Work& w, int v, int32_t* q, int at) {
  const int s0 = __ldg(w.slice_first + v), s1 = __ldg(w.slice_first + v + 1);
  if (s0 == s1) q[at] = v;
  else
    for (int j = s0; j < s1; ++j) q[at++] = -(j + 1);
}

}  // namespace tga
