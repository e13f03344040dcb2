// Lean schedule of the full sweeps (neighbour access, PageRank, HITS, window counts, degree
// centrality, full decode): the sweep order with each entry carrying what opening it needs, so a
// whole (short) list is opened from one coalesced 16-byte load -- the bit positions of its record
// and of its timestamps (LeanEntry) -- instead of two Elias-Fano selects of several dependent
// loads each.  Entries are decoded by LeanCursor (leancursor.cuh).
#pragma once
#include "sweep.cuh"

namespace tga {

// Lean sweeps: 4 blocks of 256 per SM (up to 64 registers, no local memory).  The HITS sweeps and
// the colouring check run with 5 (51 registers and a few spilled words): measured on the 2M/40M
// graph, HITS x30 29.1 -> 27.5 ms and colouring 4.13 -> 3.99 ms, while PageRank and neighbour
// access were slower that way (23.4 -> 25.8 ms, 0.58 -> 0.62 ms) and keep 4.
#define TGA_LEAN_BOUNDS __launch_bounds__(kBlock, 4)
#define TGA_LEAN_BOUNDS5 __launch_bounds__(kBlock, 5)

// Schedule entry of a lean sweep: v >= 0 a whole list whose record starts at bit gbit of the
// graph stream and whose timestamps start at bit tbit; v < 0 the slice -(v+1) (positions unused).
// Positions are 48-bit: hi16 = (gbit >> 32) << 16 | (tbit >> 32).
struct LeanEntry {
  int32_t v;
  uint32_t hi16;
  uint32_t glo, tlo;
};

__host__ __device__ inline LeanEntry lean_entry(int32_t v, uint64_t gbit, uint64_t tbit) {
  LeanEntry e;
  e.v = v;
  e.hi16 = (uint32_t)(((gbit >> 32) & 0xFFFF) << 16 | ((tbit >> 32) & 0xFFFF));
  e.glo = (uint32_t)gbit;
  e.tlo = (uint32_t)tbit;
  return e;
}

// A lean schedule as kernels take it.
struct LeanWork {
  const LeanEntry* e;
  int32_t count;
  const SliceState* slices;
  const int32_t* run_first;
};

// Sweep driver over a lean schedule: thread i decodes entry i (the schedule groups entries of equal
// length, so the lanes of a warp finish together).  (Measured against a grid of one to two waves in
// which each thread walks the schedule with the grid's stride and prefetches its next entry: that
// hid more load latency but its lanes fell out of step, and the PageRank pass took 1.26-1.41 ms
// against 1.17 ms.)
// Hooks and kRuns / kTimes / kRunArg as in run_order (sweep.cuh).  kSkip (with kTimes = false):
// edge() returns an int -- 0 stop the list, 1 go on, 2 go on and the edges that repeat this
// successor right after it do not matter to the hook: they are consumed without a merge step or a
// hook call, and count as decoded edges.  (With timestamps the repeats' deltas still have to be
// decoded one by one, and a per-lane skip loop only makes the warp diverge.)
template <bool kRuns = false, bool kTimes = true, bool kRunArg = false, bool kSkip = false, class Want, class Begin,
          class Edge, class End>
__device__ __forceinline__ unsigned long long lean_one(const GraphView& g, const LeanEntry* entries, int i,
                                                       const SliceState* slices, const int32_t* run_first, Want& want,
                                                       Begin& begin, Edge& edge, End& end) {
  static_assert(!(kSkip && kTimes), "repeats carry their own timestamps");
  unsigned long long edges = 0;
  const LeanEntry e = entries[i];
  LeanCursor c;
  RunFilter rf;
  int x, first = 0, cnt, lead = kNoRunFilter, run = -1;
  if (e.v >= 0) {
    x = e.v;
    if (!want(x)) return 0;
    const uint64_t gbit = ((uint64_t)(e.hi16 >> 16) << 32) | e.glo;
    const uint64_t tbit = ((uint64_t)(e.hi16 & 0xFFFF) << 32) | e.tlo;
    cnt = c.open(g, x, gbit, tbit);
  } else {
    const SliceState& s = slices[-e.v - 1];
    x = s.v;
    if (!want(x)) return 0;
    cnt = c.restore(g, s);
    first = s.first;
    if (kRuns && s.run >= 0) lead = __ldg(run_first + s.run);
    run = s.run;
  }
  bool go;
  if constexpr (kRunArg) go = cnt > 0 && begin(x, first, cnt, run);
  else go = cnt > 0 && begin(x, first, cnt);
  if (!go) return 0;
  if (kRuns) rf.start(lead, first);
  int y;
  int64_t t;
  while (c.template next<kTimes>(g, y, t)) {
    const bool pass = !kRuns || rf.pass(y);
    if constexpr (kSkip) {
      if (!pass) continue;
      const int r = edge(x, y, t);
      if (r == 0) break;
      // (a slice inside a run whose kept edge is still ahead goes on edge by edge)
      if (r == 2 && (!kRuns || rf.lead == kNoRunFilter || rf.lead < rf.idx)) {
        const int k = c.skip_repeats(g, y);
        if (kRuns) rf.idx += k;
      }
    } else {
      if (pass && !edge(x, y, t)) break;
    }
  }
  end(x);
  // decoded edges (repeats consumed by skip_repeats included): what the cursor no longer holds
  edges = (unsigned long long)(cnt - max(c.remaining, 0));
  return edges;
}

template <bool kRuns = false, bool kTimes = true, bool kRunArg = false, bool kSkip = false, class Want, class Begin,
          class Edge, class End>
__device__ __forceinline__ unsigned long long run_lean(const GraphView& g, const LeanEntry* entries, int count,
                                                       const SliceState* slices, const int32_t* run_first, Want want,
                                                       Begin begin, Edge edge, End end) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= count) return 0;
  return lean_one<kRuns, kTimes, kRunArg, kSkip>(g, entries, i, slices, run_first, want, begin, edge, end);
}

// The same over a fixed grid (a cooperative launch, for the dense levels of the traversals, which
// sweep the whole schedule with a frontier test in want): chunks of 32 entries are dealt by
// spread_warp_rank(), so that the slices of one long list, which sit together in the schedule,
// land on different SMs.
template <bool kRuns = false, bool kTimes = true, bool kRunArg = false, class Want, class Begin, class Edge, class End>
__device__ __forceinline__ unsigned long long run_lean_grid(const GraphView& g, const LeanWork& lw, Want want, Begin begin,
                                                            Edge edge, End end) {
  unsigned long long edges = 0;
  const int nthreads = (int)(gridDim.x * blockDim.x);
  for (int i = spread_warp_rank() * 32 + (int)(threadIdx.x & 31); i < lw.count; i += nthreads)
    edges += lean_one<kRuns, kTimes, kRunArg, false>(g, lw.e, i, lw.slices, lw.run_first, want, begin, edge, end);
  return edges;
}

// Resolution of the copy masks at load: one thread per list x of `ids` (lists with a reference),
// its copy mask run over the referenced chain with the general decoder.  Pass 1 (out == nullptr)
// stores the count in count[i]; pass 2 writes the values at out + base[x].
static __global__ void k_resolve_copies(GraphView g, const int32_t* ids, int32_t n, uint32_t* count,
                                        const uint32_t* base, int32_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = ids[i];
  DeepState deep;
  EdgeCursor c(&deep);
  if (c.open(g, x) <= 0 || !c.chain) {
    if (!out) count[i] = 0;
    return;
  }
  int h = c.top.hc;
  uint32_t k = 0;
  int32_t* dst = out ? out + base[x] : nullptr;
#pragma unroll 1
  while (h != kInf && k <= (uint32_t)g.max_list) {
    if (dst) dst[k] = h;
    ++k;
    h = deep_copy_next(*g.self, deep);
  }
  if (!out) count[i] = k;
}

// Builds the whole-list entries of a lean schedule: entry i of `ids` (a vertex, or -(slice+1))
// becomes a LeanEntry, with the record and timestamp positions of a vertex looked up in the
// Elias-Fano indexes.
static __global__ void k_lean_entries(GraphView g, const int32_t* ids, int32_t n, LeanEntry* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = ids[i];
  if (v < 0) {
    out[i] = lean_entry(v, 0, 0);
    return;
  }
  out[i] = lean_entry(v, ef_get(g, g.gef, (uint64_t)v), ef_get(g, g.tef, (uint64_t)v));
}

}  // namespace tga
