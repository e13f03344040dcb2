// Edge-balanced work decomposition of the successor lists.
//
// Power-law outdegrees make one-thread-per-vertex kernels wait for their largest list (a 163K-edge
// list decoded by one thread takes longer than the rest of the graph together).  At load time every
// list longer than the slice length is cut into slices: a slice holds the complete decoder state at
// its first edge (reference-chain levels, timestamp cursor, previous timestamp), so any thread can
// resume decoding there.  A slice may start inside a run of equal successors (lists are sorted, so
// equal successors are adjacent); the "first in-window occurrence of equal consecutive successors"
// rule then needs the position of the run's first in-window edge, which each call computes for
// its window (k_run_first in sweep.cuh) for the few runs that slices cut.
// The remaining (short) lists are grouped into work items of consecutive vertices holding about the
// same number of edges as a slice.
#pragma once
#include "decoder.cuh"

namespace tga {

// SliceState (decoder.cuh) holds the complete decoder state at the first edge of a slice.

// slice >= 0: one slice; slice < 0: every vertex of [v0, v1) whole.
struct WorkItem {
  int32_t v0, v1, slice;
};

__device__ __forceinline__ void cursor_restore(const GraphView& g, EdgeCursor& c, const SliceState& s) {
  c.top = s.top;
  c.chain = s.chain;
  if (s.chain) *c.deep = g.slice_deep[s.deep];
  c.ts.init(g.t, s.tpos);
  c.prev = s.prev;
  c.remaining = s.count;
  c.x = s.v;
}

// Writes the cursor's state at edge `first` of v; the chain levels go to *deep (kept only for
// lists that copy from a chain; the host moves them to the compact slice_deep array).
__device__ __forceinline__ void cursor_save(const EdgeCursor& c, SliceState& s, DeepState& deep, int v, int first) {
  s.top = c.top;
  s.chain = c.chain;
  s.deep = -1;
  if (c.chain) deep = *c.deep;
  s.tpos = c.ts.pos();
  s.prev = c.prev;
  s.v = v;
  s.first = first;
  s.count = 0;
  s.run = -1;
}

// One thread per long list: walks the list once and records a slice every `len` edges.  A slice
// that starts inside a run of equal successors gets run = the list index where that run starts
// (the host turns it into a run index).  cap[b] slots are reserved per list.
// Chain levels go to deep_out + deep_base[b] (deep_base[b + 1] - deep_base[b] is the list's slot count when it
// copies from a chain, 0 otherwise: cursor_save writes them only for such lists).
static __global__ void k_build_slices(GraphView g, const int32_t* big_v, const int64_t* slot_base,
                                      const int64_t* deep_base, int32_t nbig, int32_t len, SliceState* out,
                                      DeepState* deep_out, int32_t* nslices) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbig) return;
  const int v = big_v[b];
  SliceState* dst = out + slot_base[b];
  DeepState* ddst = deep_out + deep_base[b];
  const int cap = (int)(slot_base[b + 1] - slot_base[b]);
  DeepState deep, saved_deep;
  EdgeCursor c(&deep);
  const int d = c.open(g, v);
  cursor_save(c, dst[0], ddst[0], v, 0);
  int k = 1, last = 0, prev_y = -1, run_start = 0;
  for (int i = 0; i < d; ++i) {
    const bool cand = (i - last >= len) && k < cap;
    EdgeCursor saved(&saved_deep);
    if (cand) {
      saved = c;
      saved.deep = &saved_deep;
      if (c.chain) saved_deep = deep;
    }
    int y;
    int64_t t;
    if (!c.next(g, y, t)) break;
    if (cand) {
      dst[k - 1].count = i - last;
      cursor_save(saved, dst[k], ddst[k], v, i);
      if (y == prev_y) dst[k].run = run_start;
      last = i;
      ++k;
    }
    if (y != prev_y) run_start = i;
    prev_y = y;
  }
  dst[k - 1].count = d - last;
  nslices[b] = k;
}

}  // namespace tga
