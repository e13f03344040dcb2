// Batched queries: many temporal BFS sources in one traversal, many windowed PageRanks in one
// strided vector.  Each frontier (or every) list is decoded once per level (iteration) and its
// edges are applied to all the queries that need them.
//
// Multi-source BFS.  Up to kMaxSources sources run in one cooperative launch, each with its own
// time window.  Per vertex, a frontier mask of kMaxSources bits (kWords 64-bit words) says for
// which sources its arrival dropped in the last level; a level decodes each such list once and,
// per edge, relaxes it for every source of the mask whose window holds the edge's time, keeping
// each source's "first in-window occurrence of equal consecutive successors" rule with a per-run
// mask of the sources that have already seen an in-window edge.  Relaxations are reductions
// without a return value (RED.MIN on the source's arrival, RED.OR on the successor's next mask)
// plus a dirty bit; after a grid barrier a scan keeps only the sources whose arrival really
// dropped, clears the finished level's masks and builds the next queues.  Same queue rotation,
// dense-level sweep and bounded barrier as the single-source traversal (traverse.cu).
//
// Arrivals are vertex-major (row v holds the arrivals of all sources at v), so the sources of one
// list touch a few adjacent sectors.  The scan splits the frontier by the number of sources in a
// vertex's mask: lists with fewer than kWarpSources go to the sparse queue, one thread per entry;
// the others to the wide queue, one warp per entry, where lane 0 decodes and each lane handles the
// sources lane, lane + 32, ... with their arrivals at the list's vertex held in registers, so an
// edge costs a lane at most kSlots checks instead of one thread walking every source.
#include <algorithm>
#include <memory>
#include <cstring>
#include <vector>

#include "gridsync.cuh"
#include "hot.cuh"
#include "trace.cuh"

namespace tga {

constexpr int kMaxSources = 256;
constexpr int kWords = kMaxSources / 64;
constexpr int kSlots = kMaxSources / 32;   // sources per lane in the wide relax
constexpr int kWarpSources = 8;            // masks with at least this many sources take the wide queue
constexpr uint32_t kNoArrival = 0xFFFFFFFFu;
constexpr int kKeepSeen = -3;  // the first successor continues a run begun in an earlier slice

struct MultiArgs {
  Work w;
  TravCtl* ctl;
  int32_t* q[2];             // sparse queues (rotating with the levels)
  int32_t* dq[2];            // wide queues
  uint32_t* arr;             // [nv][stride] arrival of v for source s (kNoArrival: unreached)
  uint32_t* prev;            // [nv][stride] arrival at which v was last enqueued for s
  uint64_t* F[2];            // [nv][kWords] frontier masks: level L reads F[L & 1], fills F[(L+1) & 1]
  uint32_t* dirty;           // bit per vertex: relaxed in the current level
  int32_t ndirty;
  const int64_t* lo;         // [nsrc] windows [lo, hi)
  const int64_t* hi;
  const int32_t* run_first;  // [nruns][run_stride] list index of a cut run's first in-window edge
  int32_t run_stride;        // columns of run_first (a source s reads column scol[s])
  uint32_t* stamp;           // [nv] epoch of the traversal that last touched the vertex
  int32_t* touched;          // vertices touched by this traversal (arrival set for some source)
  int32_t* ntouched;
  uint32_t epoch;
  int32_t nsrc, nv;
  int32_t stride;            // sources per arrival row (the state's capacity)
  int32_t nv_lists;          // vertices with an out-list (graph n)
  int32_t dense_min, level_cap;
  unsigned long long* edges;
};

__device__ __forceinline__ size_t arr_at(const MultiArgs& a, int v, int s) { return (size_t)v * a.stride + s; }

__device__ __forceinline__ int mask_sources(const uint64_t* F, int v) {
  int n = 0;
#pragma unroll
  for (int k = 0; k < kWords; ++k) n += __popcll(__ldcg(F + (size_t)v * kWords + k));
  return n;
}

// Sparse part of a level: one thread per list whose mask has fewer than kWarpSources sources
// (the queue, or with `dense` every such list in schedule order).  The list's sources and their
// arrivals at the list's vertex sit in kSparseSlots register slots, loaded once per list, so an
// edge costs one window test (and a fire-and-forget RED.MIN) per source, not a dependent load.
constexpr int kSparseSlots = kWarpSources - 1;

__device__ __forceinline__ unsigned long long multi_relax_sparse(const GraphView& g, MultiArgs& a, const Work& w,
                                                                 const int64_t* slo, const int64_t* shi,
                                                                 const int32_t* scol, const int32_t* q, int qn, int L,
                                                                 bool dense) {
  const uint64_t* Fc = a.F[L & 1];
  uint64_t* Fn = a.F[(L + 1) & 1];
  int src[kSparseSlots];     // source of slot i (-1: empty)
  uint32_t ax[kSparseSlots];  // its arrival at the list's vertex
  uint32_t seen = 0;          // bit i: slot i took an edge of the current run of equal successors
  int yprev = -1;
  auto begin = [&](int x, int first, int, int run) {
    if (x < g.active_begin || x > g.max_label) return false;
    uint64_t m0 = __ldcg(Fc + (size_t)x * kWords + 0), m1 = __ldcg(Fc + (size_t)x * kWords + 1);
    uint64_t m2 = __ldcg(Fc + (size_t)x * kWords + 2), m3 = __ldcg(Fc + (size_t)x * kWords + 3);
    if (!(m0 | m1 | m2 | m3)) return false;
#pragma unroll
    for (int i = 0; i < kSparseSlots; ++i) {
      int s = -1;
      if (m0) {
        s = __ffsll((long long)m0) - 1;
        m0 &= m0 - 1;
      } else if (m1) {
        s = 64 + __ffsll((long long)m1) - 1;
        m1 &= m1 - 1;
      } else if (m2) {
        s = 128 + __ffsll((long long)m2) - 1;
        m2 &= m2 - 1;
      } else if (m3) {
        s = 192 + __ffsll((long long)m3) - 1;
        m3 &= m3 - 1;
      }
      src[i] = s;
      ax[i] = s >= 0 ? __ldcg(a.arr + arr_at(a, x, s)) : kNoArrival;
    }
    // The scan sends lists with kWarpSources or more sources to the wide queue; more here is a bug.
    if (m0 | m1 | m2 | m3) set_err(g, kErrCode);
    seen = 0;
    yprev = -1;
    if (run >= 0) {
      // Sources whose first in-window edge of this run lies before the slice saw the run already.
      const int32_t* rf = a.run_first + (size_t)run * a.run_stride;
#pragma unroll
      for (int i = 0; i < kSparseSlots; ++i)
        if (src[i] >= 0 && __ldg(rf + scol[src[i]]) < first) seen |= 1u << i;
      yprev = kKeepSeen;
    }
    return true;
  };
  auto edge = [&](int, int y, int64_t t) {
    if (yprev == kKeepSeen) {
      yprev = y;
    } else if (y != yprev) {
      seen = 0;
      yprev = y;
    }
    const bool usable = y >= g.active_begin && y < g.max_vertex && t >= 0 && t < 0xFFFFFFFFll;
    uint64_t add0 = 0, add1 = 0, add2 = 0, add3 = 0;
#pragma unroll
    for (int i = 0; i < kSparseSlots; ++i) {
      const int s = src[i];
      if (s < 0 || ((seen >> i) & 1u)) continue;
      if (t < slo[s] || t >= shi[s]) continue;
      seen |= 1u << i;
      if (!usable || (int64_t)ax[i] > t) continue;
      // An arrival already at t or earlier needs no atomic (measured on the CC of 2M/40M: checking
      // every successor, not only the hot ones, 36.3 -> 34.8 ms).
      if (__ldcg(a.arr + arr_at(a, y, s)) <= (uint32_t)t) continue;
      atomicMin(a.arr + arr_at(a, y, s), (uint32_t)t);
      const uint64_t bit = 1ull << (s & 63);
      const int wd = s >> 6;
      add0 |= wd == 0 ? bit : 0;
      add1 |= wd == 1 ? bit : 0;
      add2 |= wd == 2 ? bit : 0;
      add3 |= wd == 3 ? bit : 0;
    }
    if (add0 | add1 | add2 | add3) {
      unsigned long long* f = (unsigned long long*)(Fn + (size_t)y * kWords);
      {  // bits another relaxation of this level has set already need no atomic
        if (add0 && (__ldcg(f + 0) & add0) == add0) add0 = 0;
        if (add1 && (__ldcg(f + 1) & add1) == add1) add1 = 0;
        if (add2 && (__ldcg(f + 2) & add2) == add2) add2 = 0;
        if (add3 && (__ldcg(f + 3) & add3) == add3) add3 = 0;
      }
      if (add0) atomicOr(f + 0, (unsigned long long)add0);
      if (add1) atomicOr(f + 1, (unsigned long long)add1);
      if (add2) atomicOr(f + 2, (unsigned long long)add2);
      if (add3) atomicOr(f + 3, (unsigned long long)add3);
      if (!((__ldcg(&a.dirty[y >> 5]) >> (y & 31)) & 1u)) atomicOr(&a.dirty[y >> 5], 1u << (y & 31));
    }
    return true;
  };
  if (dense) {
    // (measured: this order-based sweep runs the CC of the 2M/40M graph in 39.0 ms, the lean
    // schedule's grid walk in 45.2 ms)
    return run_order<false, true, false, true, true>(
        g, w,
        [&](int x) {
          const int n = mask_sources(Fc, x);
          return n > 0 && n < kWarpSources;
        },
        begin, edge, [](int) {});
  }
  return drive_queue<false, true, true>(g, w, q, qn, begin, edge, [](int) {});
}

// Wide part of a level: one warp per entry of the wide queue (entries taken from *counter).
__device__ unsigned long long multi_relax_wide(const GraphView& g, MultiArgs& a, const int64_t* slo,
                                               const int64_t* shi, const int32_t* scol, const int32_t* dq, int dn,
                                               int32_t* counter, int L, const int32_t* hids) {
  constexpr unsigned kFull = 0xffffffffu;
  const uint64_t* Fc = a.F[L & 1];
  uint64_t* Fn = a.F[(L + 1) & 1];
  const int lane = threadIdx.x & 31;
  LeanCursor c;
  unsigned long long edges = 0;
  for (;;) {
    int i = 0;
    if (lane == 0) i = atomicAdd(counter, 1);
    i = __shfl_sync(kFull, i, 0);
    if (i >= dn) break;
    const int e = __ldcg(dq + i);
    int x = e, first = 0, run = -1;
    if (e < 0) {
      const SliceState& s = a.w.slices[-e - 1];
      x = s.v;
      first = s.first;
      run = s.run;
    }
    if (x < g.active_begin || x > g.max_label) continue;
    // Slot k of this lane is source k * 32 + lane (bit 32 * (k & 1) + lane of mask word k / 2).
    uint32_t mine = 0, seen = 0;
    uint32_t ax[kSlots];
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const int s = k * 32 + lane;
      ax[k] = kNoArrival;
      if ((__ldcg(Fc + (size_t)x * kWords + (k >> 1)) >> (s & 63)) & 1) {
        mine |= 1u << k;
        ax[k] = __ldcg(a.arr + arr_at(a, x, s));
        if (run >= 0 && __ldg(a.run_first + (size_t)run * a.run_stride + scol[s]) < first) seen |= 1u << k;
      }
    }
    // Every lane decodes the entry (the same words, loaded once for the warp, and the same code
    // path, so the warp does not diverge): no lane waits on a shuffle from a decoding lane, and the
    // next edge is decoded while the current one is relaxed.
    int count = 0;
    {
      int f, lead, r;
      open_entry(g, a.w, e, c, f, count, lead, r);
    }
    if (count <= 0) continue;
    int yprev = run >= 0 ? kKeepSeen : -1;
    int yn = 0;
    int64_t tn = 0;
    bool more = c.next(g, yn, tn);
    while (more) {
      const int y = yn;
      const int64_t t = tn;
      more = c.next(g, yn, tn);
      edges += lane == 0;
      if (yprev == kKeepSeen) {
        yprev = y;
      } else if (y != yprev) {
        seen = 0;
        yprev = y;
      }
      const bool usable = y >= g.active_begin && y < g.max_vertex && t >= 0 && t < 0xFFFFFFFFll;
      const bool hot = usable && hot_is(hids, y);
      uint32_t add = 0;
#pragma unroll
      for (int k = 0; k < kSlots; ++k) {
        if (!(((mine & ~seen) >> k) & 1)) continue;
        const int s = k * 32 + lane;
        if (t < slo[s] || t >= shi[s]) continue;
        seen |= 1u << k;
        if (!usable || (int64_t)ax[k] > t) continue;
        if (hot && __ldcg(a.arr + arr_at(a, y, s)) <= (uint32_t)t) continue;  // nothing to lower
        atomicMin(a.arr + arr_at(a, y, s), (uint32_t)t);
        add |= 1u << k;
      }
      if (__any_sync(kFull, add != 0)) {
#pragma unroll
        for (int wd = 0; wd < kWords; ++wd) {
          const uint32_t lo = __ballot_sync(kFull, (add >> (2 * wd)) & 1);
          const uint32_t hi = __ballot_sync(kFull, (add >> (2 * wd + 1)) & 1);
          const uint64_t bits = (uint64_t)lo | ((uint64_t)hi << 32);
          unsigned long long* f = (unsigned long long*)(Fn + (size_t)y * kWords + wd);
          if (lane == 0 && bits && !(hot && (__ldcg(f) & bits) == bits)) atomicOr(f, (unsigned long long)bits);
        }
        if (lane == 0 && (!hot || !((__ldcg(&a.dirty[y >> 5]) >> (y & 31)) & 1u)))
          atomicOr(&a.dirty[y >> 5], 1u << (y & 31));
      }
    }
  }
  return edges;
}

// After level L (targets F[(L+1) & 1]): clears the masks of level L's frontier (queues cq/cn and
// cdq/cdn), keeps per dirty vertex only the sources whose arrival dropped, and appends the
// vertices with any such source to the next sparse or wide queue by their number of sources.
__device__ __forceinline__ void multi_scan(MultiArgs& a, const int32_t* cq, int cn, const int32_t* cdq, int cdn,
                                           int32_t* nq, int32_t* ncnt, int32_t* ndq, int32_t* ndcnt, int L) {
  uint64_t* Fc = a.F[L & 1];
  uint64_t* Fn = a.F[(L + 1) & 1];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  for (int i = tid; i < cn + cdn; i += nthreads) {
    const int e = i < cn ? __ldcg(cq + i) : __ldcg(cdq + i - cn);
    const int x = e >= 0 ? e : a.w.slices[-e - 1].v;
#pragma unroll
    for (int k = 0; k < kWords; ++k) Fc[(size_t)x * kWords + k] = 0;
  }
  const int lane = threadIdx.x & 31;
  const int warp = tid >> 5, nwarps = nthreads >> 5;
  for (int base = warp * 32; base < a.ndirty; base += nwarps * 32) {
    const int i = base + lane;
    uint32_t bits = 0;
    if (i < a.ndirty) {
      bits = __ldcg(a.dirty + i);
      if (bits) a.dirty[i] = 0;
    }
    deal_dirty(bits, base, [&](int v) {
      int nkept = 0;
      if (v >= 0) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) {
          const uint64_t m = __ldcg(Fn + (size_t)v * kWords + k);
          uint64_t kept = 0;
          for (uint64_t c = m; c; c &= c - 1) {
            const int bb = __ffsll((long long)c) - 1;
            const size_t at = arr_at(a, v, k * 64 + bb);
            const uint32_t now = __ldcg(a.arr + at), before = __ldcg(a.prev + at);
            if (now < before) {
              a.prev[at] = now;
              kept |= 1ull << bb;
            }
          }
          if (kept != m) Fn[(size_t)v * kWords + k] = kept;
          nkept += __popcll(kept);
        }
      }
      const bool wide = nkept >= kWarpSources, sparse = nkept > 0 && !wide;
      const int ec = (wide || sparse) ? entry_count(a.w, v) : 0;
      const int at = warp_reserve(ncnt, sparse ? ec : 0);
      if (sparse) write_entries(a.w, v, nq, at);
      const int atw = warp_reserve(ndcnt, wide ? ec : 0);
      if (wide) write_entries(a.w, v, ndq, atw);
      // kept vertices this traversal has not touched before
      const bool fresh = (wide || sparse) && __ldcg(&a.stamp[v]) != a.epoch;
      const int tat = warp_reserve(a.ntouched, fresh ? 1 : 0);
      if (fresh) {
        a.stamp[v] = a.epoch;
        a.touched[tat] = v;
      }
    });
  }
}

// Levels 1.. of a multi-source traversal whose sources are seeded (level-0 relaxations in F[1]
// and the dirty bits); the control block's queue and work counters must be zero.  All blocks of
// the cooperative launch call it together; false if the launch has failed (return at once).
__device__ bool multi_levels(const GraphView& g, MultiArgs& a, const int64_t* slo, const int64_t* shi,
                             const int32_t* scol, unsigned long long& mine, int& levels, const int32_t* hids) {
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  TravCtl* ctl = a.ctl;
  // The sources were seeded as level 0's relaxations: the scan turns them into level 1's queues.
  multi_scan(a, a.q[0], 0, a.dq[0], 0, a.q[1], &ctl->cnt[1], a.dq[1], &ctl->dcnt[1], 0);
  if (!grid_sync(ctl, g)) return false;
  int L = 1;
  for (;;) {
    const int qn = __ldcg(&ctl->cnt[L % 3]), dn = __ldcg(&ctl->dcnt[L % 3]);
    if (qn == 0 && dn == 0) break;
    if (L >= a.level_cap) {
      if (lead) {
        set_err(g, kErrTimeout);
        ctl->status = 1;
      }
      return false;
    }
    if (lead) {
      ctl->cnt[(L + 2) % 3] = 0;
      ctl->next[(L + 1) % 3] = 0;
      ctl->dcnt[(L + 2) % 3] = 0;
      ctl->dnext[(L + 1) % 3] = 0;
    }
    if (dn > 0) mine += multi_relax_wide(g, a, slo, shi, scol, a.dq[L & 1], dn, &ctl->dnext[L % 3], L, hids);
    if (qn > 0) {
      Work w = a.w;
      w.next = &ctl->next[L % 3];
      mine += multi_relax_sparse(g, a, w, slo, shi, scol, a.q[L & 1], qn, L, qn >= a.dense_min);
    }
    if (!grid_sync(ctl, g)) return false;
    multi_scan(a, a.q[L & 1], qn, a.dq[L & 1], dn, a.q[(L + 1) & 1], &ctl->cnt[(L + 1) % 3], a.dq[(L + 1) & 1],
               &ctl->dcnt[(L + 1) % 3], L);
    if (!grid_sync(ctl, g)) return false;
    ++L;
  }
  levels = L;
  return true;
}

// Sources 0..nsrc-1 of a traversal (grid-stride over the calling threads): the arrival of each
// source vertex (max(lo, 0)) as its level-0 relaxation.
__device__ __forceinline__ void multi_seed(MultiArgs& a, const int32_t* src, int32_t nsrc, int32_t n) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsrc; s += gridDim.x * blockDim.x) {
    const int v = __ldcg(src + s);
    const int64_t lo = __ldcg(a.lo + s);
    a.arr[arr_at(a, v, s)] = (uint32_t)(lo > 0 ? lo : 0);
    if (atomicExch(&a.stamp[v], a.epoch) != a.epoch) a.touched[atomicAdd(a.ntouched, 1)] = v;
    if (v < n) {
      atomicOr((unsigned long long*)(a.F[1] + (size_t)v * kWords + s / 64), (unsigned long long)(1ull << (s & 63)));
      atomicOr(&a.dirty[v >> 5], 1u << (v & 31));
    }
  }
}

// Per-source windows and run-table columns in shared memory (source s: window s, column s).
__device__ __forceinline__ void load_windows(const MultiArgs& a, int64_t* slo, int64_t* shi, int32_t* scol) {
  for (int s = threadIdx.x; s < kMaxSources; s += blockDim.x) {
    slo[s] = s < a.nsrc ? a.lo[s] : 0;
    shi[s] = s < a.nsrc ? a.hi[s] : 0;
    scol[s] = s;
  }
  __syncthreads();
}

// 3 blocks per SM (80 registers): 8 sources on the 2M/40M graph 22.0 -> 21.3 ms against 2 blocks.
__global__ void TGA_TRAVERSE_BOUNDS k_bfs_multi(GraphView g, MultiArgs a) {
  __shared__ int64_t slo[kMaxSources], shi[kMaxSources];
  __shared__ int32_t scol[kMaxSources];
  __shared__ int32_t hids[kHotSlots];
  hot_load(g, hids);
  load_windows(a, slo, shi, scol);
  unsigned long long mine = 0;
  int levels = 0;
  if (!multi_levels(g, a, slo, shi, scol, mine, levels, hids)) return;
  add_edges(a.edges, mine);
  if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->levels = levels;
}

// Sources of the batch: arrival and level-0 relaxation of each source vertex.
__global__ void k_bfs_multi_seed(MultiArgs a, const int32_t* src) { multi_seed(a, src, a.nsrc, a.nv_lists); }

// Per-source first in-window edge of each run of equal successors cut by slices: one thread per
// (run, overlapping slice) decodes the run's part of the slice and lowers run_first[run][s] for
// every source s whose window holds one of those edges.
__global__ void TGA_DECODE_BOUNDS k_run_first_multi(GraphView g, const SliceState* slices, const RunInfo* runs,
                                                    const int2* pairs, int32_t npairs, const int64_t* lo,
                                                    const int64_t* hi, int32_t nsrc, int32_t* run_first,
                                                    int32_t stride) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const int2 pr = pairs[p];
  const RunInfo r = runs[pr.x];
  const SliceState& s = slices[pr.y];
  LeanCursor c;
  c.restore(g, s);
  uint64_t found[kWords] = {};
  int idx = s.first, y_run = -1, y;
  int64_t t;
  while (c.next(g, y, t)) {
    const int i = idx++;
    if (i < r.start) continue;
    if (y_run < 0) y_run = y;
    else if (y != y_run) break;
    for (int q = 0; q < nsrc; ++q) {
      const uint64_t bit = 1ull << (q & 63);
      if ((found[q >> 6] & bit) || t < lo[q] || t >= hi[q]) continue;
      found[q >> 6] |= bit;
      atomicMin(&run_first[(size_t)pr.x * stride + q], i);
    }
  }
}

// Back to "unreached" for every source at every vertex the traversal touched (all the entries it
// can have set), so the next traversal starts without clearing the whole [sources][vertices] state.
__global__ void k_multi_reset(uint32_t* arr, uint32_t* prev, int32_t stride, const int32_t* touched,
                              const int32_t* ntouched, int32_t nsrc) {
  const int64_t total = (int64_t)(*ntouched) * nsrc;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int u = touched[i / nsrc];
    const size_t at = (size_t)u * stride + i % nsrc;
    arr[at] = kNoArrival;
    prev[at] = kNoArrival;
  }
}

// Arrivals of sources 0..nsrc-1 to the source-major result layout (out[s][v], INT32_MAX for
// unreached): 32 x 32 tiles through shared memory, so both sides are read and written in rows.
__global__ void k_multi_unpack(const uint32_t* arr, int32_t stride, int32_t nsrc, int32_t nv, int32_t* out) {
  __shared__ uint32_t tile[32][33];
  const int v0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int v = v0 + r, s = s0 + threadIdx.x;
    tile[r][threadIdx.x] = (v < nv && s < nsrc) ? arr[(size_t)v * stride + s] : kNoArrival;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int s = s0 + r, v = v0 + threadIdx.x;
    if (s < nsrc && v < nv) {
      const uint32_t x = tile[threadIdx.x][r];
      out[(size_t)s * nv + v] = x == kNoArrival ? INT32_MAX : (int32_t)x;
    }
  }
}

// Scratch of a multi-source traversal of up to `cap` sources: the persistent state (m_*) and, in
// s_d, the windows, sources and per-source run table.  Growing the state (capacity rounded up to
// a power of two, at least 32) clears it; so does a traversal that ended early (m_clean false).
static int multi_buffers(GraphHandle& h, int32_t cap) {
  const size_t nv = (size_t)h.view.max_vertex;
  const size_t qcap = nv + (size_t)h.nslices + 1;
  int rc;
  const size_t run_bytes = (size_t)std::max(h.nruns, 1) * kMaxSources * 4;
  if ((rc = h.s_q0.ensure(qcap * 4)) || (rc = h.s_q1.ensure(qcap * 4)) || (rc = h.s_cnt.ensure(sizeof(TravCtl))) ||
      (rc = h.s_d.ensure(kMaxSources * 20 + run_bytes)) || (rc = h.m_dq.ensure(2 * qcap * 4)))
    return rc;
  if (cap > h.m_cap || !h.m_clean) {
    int32_t c = std::max(h.m_cap, 32);
    while (c < cap) c *= 2;
    c = std::min(c, kMaxSources);
    h.m_clean = false;
    if ((rc = h.m_state.ensure(2 * (size_t)c * nv * 4)) || (rc = h.m_mask.ensure(2 * nv * kWords * 8)) ||
        (rc = h.m_dirty.ensure(((nv + 31) / 32) * 4)) || (rc = h.m_stamp.ensure(nv * 4)) ||
        (rc = h.m_touched.ensure((nv + 1) * 4)))
      return rc;
    TGA_CUDA_TRY(cudaMemsetAsync(h.m_state.p, 0xFF, 2 * (size_t)c * nv * 4, h.stream));
    TGA_CUDA_TRY(cudaMemsetAsync(h.m_mask.p, 0, 2 * nv * kWords * 8, h.stream));
    TGA_CUDA_TRY(cudaMemsetAsync(h.m_dirty.p, 0, ((nv + 31) / 32) * 4, h.stream));
    TGA_CUDA_TRY(cudaMemsetAsync(h.m_stamp.p, 0, nv * 4, h.stream));
    TGA_CUDA_TRY(cudaMemsetAsync(h.m_touched.as<int32_t>() + nv, 0, 4, h.stream));
    h.m_cap = c;
    h.m_pending = 0;
    h.m_epoch = 0;
    h.m_clean = true;
  }
  return TGA_OK;
}

static int64_t* multi_lo(GraphHandle& h) { return h.s_d.as<int64_t>(); }
static int64_t* multi_hi(GraphHandle& h) { return h.s_d.as<int64_t>() + kMaxSources; }
static int32_t* multi_src(GraphHandle& h) { return reinterpret_cast<int32_t*>(h.s_d.as<int64_t>() + 2 * kMaxSources); }
static int32_t* multi_run_table(GraphHandle& h) { return multi_src(h) + kMaxSources; }

// Per-source run table of the windows in multi_lo/multi_hi (sources 0..nsrc-1).
static int multi_runs(GraphHandle& h, int32_t nsrc) {
  if (h.nruns <= 0) return TGA_OK;
  int32_t* drf = multi_run_table(h);
  KL(k_fill_i32, grid_for((int64_t)h.nruns * kMaxSources, kBlock))(drf, INT32_MAX, (int64_t)h.nruns * kMaxSources);
  KL(k_run_first_multi, grid_for(h.nrun_pairs, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_runs.as<RunInfo>(),
                                                       h.d_run_pairs.as<int2>(), h.nrun_pairs, multi_lo(h),
                                                       multi_hi(h), nsrc, drf, kMaxSources);
  return TGA_OK;
}

// Fills `a` for traversals of up to nsrc sources whose windows are in multi_lo/multi_hi and whose
// run table is built (multi_runs), after multi_buffers(h, >= nsrc), and prepares the state: the
// previous traversal's entries back to "unreached", an empty touched list, a fresh epoch (a.epoch;
// a launch running several traversals uses a.epoch, a.epoch + 1, ... and records the last in
// h.m_epoch) and a zero control block.
static int multi_prepare(GraphHandle& h, int32_t nsrc, unsigned long long* edges, MultiArgs& a) {
  const size_t nv = (size_t)h.view.max_vertex;
  if (nsrc > h.m_cap || !h.m_clean) return fail(TGA_E_ARG, "multi-source state not prepared");
  a = MultiArgs{};
  a.w = Work{h.d_items.as<WorkItem>(), h.d_slices.as<SliceState>(), h.d_slice_first.as<int32_t>(), nullptr, h.nitems,
             h.d_order.as<int32_t>(), h.norder, nullptr};
  a.ctl = h.s_cnt.as<TravCtl>();
  a.q[0] = h.s_q0.as<int32_t>();
  a.q[1] = h.s_q1.as<int32_t>();
  a.dq[0] = h.m_dq.as<int32_t>();
  a.dq[1] = a.dq[0] + nv + (size_t)h.nslices + 1;
  a.arr = h.m_state.as<uint32_t>();
  a.prev = a.arr + (size_t)h.m_cap * nv;
  a.F[0] = h.m_mask.as<uint64_t>();
  a.F[1] = a.F[0] + nv * kWords;
  a.dirty = h.m_dirty.as<uint32_t>();
  a.ndirty = (int32_t)((nv + 31) / 32);
  a.lo = multi_lo(h);
  a.hi = multi_hi(h);
  a.run_first = multi_run_table(h);
  a.run_stride = kMaxSources;
  a.stamp = h.m_stamp.as<uint32_t>();
  a.touched = h.m_touched.as<int32_t>();
  a.ntouched = a.touched + nv;  // the count follows the list; it outlives the shared control block
  a.nsrc = nsrc;
  a.nv = (int32_t)nv;
  a.stride = h.m_cap;
  a.nv_lists = h.view.n;
  a.dense_min = std::max<int32_t>(h.dense_min, 1);
  a.level_cap = 1 << 20;
  a.edges = edges;
  if (h.m_pending > 0) {
    KL(k_multi_reset, 4 * h.sm_count)(a.arr, a.prev, a.stride, a.touched, a.ntouched, h.m_pending);
    h.m_pending = 0;
  }
  TGA_CUDA_TRY(cudaMemsetAsync(a.ntouched, 0, 4, h.stream));
  if (h.m_epoch >= 0x7fffffffu) {  // far from wrapping: clear the stamps and start again
    TGA_CUDA_TRY(cudaMemsetAsync(a.stamp, 0, nv * 4, h.stream));
    h.m_epoch = 0;
  }
  a.epoch = ++h.m_epoch;
  TravCtl ctl{};
  std::memcpy(h.h_pinned + 32, &ctl, sizeof ctl);
  TGA_CUDA_TRY(cudaMemcpyAsync(a.ctl, h.h_pinned + 32, sizeof ctl, cudaMemcpyHostToDevice, h.stream));
  return TGA_OK;
}

// Cooperative launch of a multi-source kernel (one grid of all resident blocks), then the control
// block back to *ctl.  The state counts as cleared-or-pending only once the launch has finished
// without a barrier timeout.
static int multi_launch(GraphHandle& h, const void* kernel, void** args, TravCtl* ctl) {
  int per_sm = 0;
  TGA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
  if (per_sm < 1) return fail(TGA_E_CUDA, "batched traversal kernel cannot be resident");
  cudaEvent_t* ev = h.kernel_begin();
  ++h.timing.launches;
  h.m_clean = false;
  TGA_CUDA_TRY(cudaLaunchCooperativeKernel(kernel, dim3(per_sm * h.sm_count), dim3(kBlock), args, 0, h.stream));
  h.kernel_end(ev);
  TGA_CUDA_TRY(cudaMemcpyAsync(h.h_pinned + 32, h.s_cnt.p, sizeof(TravCtl), cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  std::memcpy(ctl, h.h_pinned + 32, sizeof *ctl);
  if (ctl->status) return fail(TGA_E_TIMEOUT, "a grid barrier wait ran out");
  h.m_clean = true;
  return TGA_OK;
}

// Runs one multi-source traversal of nsrc sources whose vertices and windows are already in
// multi_src/multi_lo/multi_hi and whose run table is built (multi_runs); multi_buffers(h, >= nsrc)
// must have run.  Leaves the arrivals in a.arr ([nsrc][max_vertex], kNoArrival: unreached) and the
// vertices with any finite arrival on a.touched (count in *a.ntouched) until the next call.
// *levels gets the levels run.
static int multi_run(GraphHandle& h, int32_t nsrc, unsigned long long* edges, MultiArgs& a, int32_t* levels) {
  TGA_TRY(multi_prepare(h, nsrc, edges, a));
  KL(k_bfs_multi_seed, grid_for(nsrc, kBlock))(a, multi_src(h));
  h.m_pending = nsrc;
  void* args[] = {&h.view, &a};
  TravCtl ctl;
  TGA_TRY(multi_launch(h, (const void*)k_bfs_multi, args, &ctl));
  *levels = ctl.levels;
  return TGA_OK;
}

// One batch of at most kMaxSources sources: arrivals to arrival_out (nsrc x max_vertex, host).
// rows (optional): per source a destination of max_vertex entries (NULL: not copied) instead of
// the contiguous arrival_out.
static int bfs_multi_batch(GraphHandle& h, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                           int32_t* arrival_out, int32_t* const* rows = nullptr) {
  const size_t nv = (size_t)h.view.max_vertex;
  const size_t state = (size_t)nsrc * nv * 4;
  TGA_TRY(multi_buffers(h, nsrc));
  TGA_TRY(h.s_e.ensure(state));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  TGA_CUDA_TRY(cudaMemcpyAsync(multi_lo(h), t_lo, (size_t)nsrc * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(multi_hi(h), t_hi, (size_t)nsrc * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(multi_src(h), src, (size_t)nsrc * 4, cudaMemcpyHostToDevice, h.stream));
  TGA_TRY(multi_runs(h, nsrc));
  MultiArgs a;
  int32_t levels = 0;
  TGA_TRY(multi_run(h, nsrc, edges, a, &levels));
  int32_t* out = h.s_e.as<int32_t>();
  k_multi_unpack<<<dim3(grid_for(nv, 32), grid_for(nsrc, 32)), dim3(32, 8), 0, h.stream>>>(a.arr, a.stride, nsrc, (int32_t)nv,
                                                                                         out);
  ++h.timing.launches;
  if (arrival_out) TGA_CUDA_TRY(cudaMemcpyAsync(arrival_out, out, state, cudaMemcpyDeviceToHost, h.stream));
  if (rows)
    for (int32_t i = 0; i < nsrc; ++i)
      if (rows[i]) TGA_CUDA_TRY(cudaMemcpyAsync(rows[i], out + (size_t)i * nv, nv * 4, cudaMemcpyDeviceToHost, h.stream));
  h.timing.iterations = levels;
  return finish(h, edges);
}

// ---------------------------------------------------------------------------------------------
// Connected components with seeds run as speculative batches.  The seed loop (traverse.cu,
// k_cc) takes the smallest unreached vertex with outdegree > 9 as the next seed and labels its
// temporal reach.  Here the next K such vertices become the sources of one multi-source traversal
// (each with its own fresh arrivals, as the sequential loop has); then, in seed order, a candidate
// is a real seed iff no earlier real seed of the batch reached it, the early-exit rules run on the
// exact reach counts, and every vertex takes the component number of the last real seed that
// reached it.  The labels equal the sequential loop's.
//
// The whole loop is one cooperative launch, for up to kMaxCcQueries queries (windows) at once:
// each batch splits the kMaxSources source slots among the queries still running (query q gets a
// contiguous range of min(K_q, kMaxSources / active) slots).  Per batch: block q picks query q's
// candidates; all blocks seed and traverse every query's sources together; all count the reach of
// each slot over the touched vertices and mark which candidates of a query reached which; block q
// validates query q in seed order and chooses its next K; all blocks label the touched vertices
// for every query and reset their arrivals.  Grid barriers separate the phases, so no batch waits
// for the host.  K_q doubles while the reach of the candidates that turned out not to be seeds
// (traversal work thrown away) stays below an eighth of the real seeds' reach plus a fixed
// allowance, and halves when it exceeds the real seeds' reach plus that allowance.

constexpr int kMaxCcQueries = 32;

struct CcBatchState {
  int64_t total;       // reach counts so far (early-exit rule)
  int32_t v;           // candidates start here
  int32_t comp;        // components so far
  int32_t small_run;   // consecutive components smaller than 5
  int32_t stop;        // the seed loop has ended (early exit)
  int32_t done;        // no candidates left below the end (read by the slot allotment)
  int32_t exhausted;   // this batch's scan reached the end (becomes `done` after validation)
  int32_t ncand;       // candidates of the current batch
  int32_t K;           // candidates wanted per batch
  int32_t pad;
};

struct CcArgs {
  CcBatchState* st;             // [nq]
  const int32_t* deg;
  uint8_t* reached;             // [nq][max_vertex] labelled already
  int32_t* label;               // [nq][max_vertex]
  const int64_t* q_lo;          // [nq] windows
  const int64_t* q_hi;
  int32_t* cand;                // [kMaxSources] source vertex of each slot
  unsigned long long* counts;   // [kMaxSources] finite arrivals per slot
  int32_t* comp_of;             // [kMaxSources] component of a real seed, -1 otherwise
  uint32_t* reach_bits;         // [kMaxSources][kMaxSources / 32] slot i reached slot j's vertex
  int32_t nq;
  int32_t end;                  // candidates lie below this vertex
  int32_t early;                // apply the early exits
  int32_t min_k;                // first and smallest number of candidates a batch takes
  int64_t limit;                // early exit: reach total above this
  int64_t budget_ns;            // stop at a batch boundary once the launch ran this long (0: never)
};

// Per-block view of the current batch's slot ranges.
struct CcSlots {
  int32_t base[kMaxCcQueries];  // first slot of query q
  int32_t k[kMaxCcQueries];     // slots offered to query q this batch
  int32_t n[kMaxCcQueries];     // candidates found (live slots from base)
  int32_t total;                // live slots of the batch
};

// Smallest (and first) number of candidates a batch takes, by the number of candidate vertices.
// Measured on the 2M/40M graph (full window / window over the middle half of the span): 4 -> 34.5
// / 38.7 ms, 16 -> 34.3 / 38.1, 64 -> 32.4 / 36.5, 128 -> 31.7 / 37.3, 256 -> 38.7 / 35.9 ms; the
// seeds before the giant component reach few vertices, so small first batches spend their levels
// on little work.  On the 6,000-vertex / 120,000-edge graph the first seed reaches most of the
// graph and the early exit stops after a few seeds: 4 -> 1.28 ms, 64 -> 9.8 ms (each extra seed
// of the first batch is a traversal of the whole graph that is thrown away).
constexpr int kCcMinKSmall = 4;
constexpr int kCcMinKLarge = 64;
constexpr int32_t kCcLargeGraph = 1 << 20;
constexpr int64_t kCcWasteAllowance = 4096;  // reach a batch may throw away and still grow K

// Every block: slot ranges of this batch from the queries' states (same result in every block).
__device__ void cc_allot(const CcArgs& c, CcSlots& sl) {
  if (threadIdx.x == 0) {
    int active = 0;
    for (int q = 0; q < c.nq; ++q) active += !__ldcg(&c.st[q].stop) && !__ldcg(&c.st[q].done);
    const int share = active ? kMaxSources / active : 0;
    int base = 0;
    for (int q = 0; q < c.nq; ++q) {
      const bool on = !__ldcg(&c.st[q].stop) && !__ldcg(&c.st[q].done);
      sl.base[q] = base;
      sl.k[q] = on ? min(__ldcg(&c.st[q].K), share) : 0;
      base += sl.k[q];
    }
  }
  __syncthreads();
}

// Block q: the first K vertices >= v below end that are unreached by query q and have outdegree
// > 9, in order, to cand[base..]; st->ncand = their number, st->exhausted once the scan reached
// the end (`done` itself changes only in the validation phase, never while blocks allot slots).
// Each thread tests 8 consecutive vertices per step.
__device__ void cc_candidates(const CcArgs& c, int q, int base, int K, int64_t nv, int32_t* s_wsum,
                              int32_t* s_count) {
  constexpr int kPer = 8;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  CcBatchState* st = c.st + q;
  const uint8_t* reached = c.reached + (size_t)q * nv;
  if (threadIdx.x == 0) *s_count = 0;
  __syncthreads();
  bool exhausted = true;
  if (K > 0) {
    for (int64_t b0 = __ldcg(&st->v); b0 < c.end; b0 += (int64_t)kBlock * kPer) {
      const int64_t u0 = b0 + (int64_t)threadIdx.x * kPer;
      uint32_t f = 0;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const int64_t u = u0 + k;
        if (u < c.end && !__ldcg(reached + u) && __ldg(c.deg + u) > 9) f |= 1u << k;
      }
      const int cnt = __popc(f);
      int incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane == 31) s_wsum[wid] = incl;
      __syncthreads();
      int before = 0, total = 0;
      for (int k = 0; k < kBlock / 32; ++k) {
        if (k < wid) before += s_wsum[k];
        total += s_wsum[k];
      }
      int pos = *s_count + before + incl - cnt;
      for (uint32_t bb = f; bb; bb &= bb - 1, ++pos)
        if (pos < K) c.cand[base + pos] = (int32_t)(u0 + __ffs(bb) - 1);
      __syncthreads();
      if (threadIdx.x == 0) *s_count += total;
      __syncthreads();
      if (*s_count >= K) {
        exhausted = false;
        break;
      }
    }
  }
  if (threadIdx.x == 0) {
    st->ncand = K > 0 ? min(*s_count, K) : 0;
    if (K > 0 && exhausted) st->exhausted = 1;
  }
}

// All blocks: finite arrivals per slot over the touched vertices (one warp per vertex, lane l
// reading slots l, l + 32, ...; block-local sums first), and the pair matrix of the batch: bit i
// of reach_bits[j] set when slot i < j of the same query reached slot j's vertex.
__device__ void cc_count(const MultiArgs& a, const CcArgs& c, const CcSlots& sl, const int32_t* scol,
                         uint32_t* s_cnt) {
  for (int s = threadIdx.x; s < kMaxSources; s += blockDim.x) s_cnt[s] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nslots = sl.base[c.nq - 1] + sl.n[c.nq - 1];
  const int nt = __ldcg(a.ntouched);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < nt; i += nwarps) {
    const int u = __ldcg(a.touched + i);
    uint32_t hit[kSlots];
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const int j = k * 32 + lane;
      hit[k] = j < nslots && __ldcg(a.arr + arr_at(a, u, j)) != kNoArrival;
    }
#pragma unroll
    for (int k = 0; k < kSlots; ++k)
      if (hit[k]) atomicAdd(&s_cnt[k * 32 + lane], 1u);
  }
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  for (int e = tid; e < nslots * nslots; e += nthreads) {
    const int j = e / nslots, i = e % nslots;
    const int q = scol[j];
    if (i < j && scol[i] == q && i >= sl.base[q] && j < sl.base[q] + sl.n[q] &&
        __ldcg(a.arr + arr_at(a, __ldcg(c.cand + j), i)) != kNoArrival)
      atomicOr(&c.reach_bits[j * (kMaxSources / 32) + (i >> 5)], 1u << (i & 31));
  }
  __syncthreads();
  for (int s = threadIdx.x; s < nslots; s += blockDim.x)
    if (s_cnt[s]) atomicAdd(&c.counts[s], (unsigned long long)s_cnt[s]);
}

// Block q: query q's candidates in seed order -- real seeds, component numbers, reach counts, the
// early exits -- and its next K, from a shared copy of its rows of the pair matrix.
__device__ void cc_validate(const CcArgs& c, int q, int base, int n, uint32_t (*reaches)[kMaxSources / 32],
                            uint32_t* s_cnt, int32_t* s_cand) {
  for (int e = threadIdx.x; e < n * (kMaxSources / 32); e += blockDim.x)
    (&reaches[0][0])[e] = __ldcg(c.reach_bits + (size_t)base * (kMaxSources / 32) + e);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    s_cnt[j] = (uint32_t)__ldcg(c.counts + base + j);
    s_cand[j] = __ldcg(c.cand + base + j);
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  CcBatchState* st = c.st + q;
  int64_t total = __ldcg(&st->total);
  int32_t v = __ldcg(&st->v), comp = __ldcg(&st->comp), small_run = __ldcg(&st->small_run);
  int32_t K = __ldcg(&st->K);
  bool stop = false;
  uint32_t real[kMaxSources / 32] = {};  // bits by slot
  int checked = 0, ninvalid = 0;
  int64_t useful = 0, wasted = 0;
  for (int j = 0; j < n; ++j) {
    const int64_t cnt = s_cnt[j];
    bool hit = false;
#pragma unroll
    for (int k = 0; k < kMaxSources / 32; ++k) hit |= (reaches[j][k] & real[k]) != 0;
    if (hit) {
      ++checked;
      ++ninvalid;
      wasted += cnt;
      c.comp_of[base + j] = -1;
      continue;
    }
    if (c.early && total > c.limit) {
      stop = true;
      break;
    }
    ++checked;
    real[(base + j) >> 5] |= 1u << ((base + j) & 31);
    useful += cnt;
    const int64_t reach = cnt - 1;  // the seed's own arrival is set before its traversal
    c.comp_of[base + j] = comp++;
    total += reach + 1;
    small_run = (reach + 1 < 5) ? small_run + 1 : 0;
    v = s_cand[j] + 1;
    if (c.early && small_run > 50) {
      stop = true;
      break;
    }
  }
  for (int j = checked; j < n; ++j) c.comp_of[base + j] = -1;
  if (!stop && n > 0) v = s_cand[n - 1] + 1;
  // Over the limit now: the next real seed would stop the loop before labelling anything.
  if (c.early && total > c.limit) stop = true;
  if (8 * wasted <= useful + kCcWasteAllowance) K = min(2 * K, kMaxSources);
  else if (wasted > useful + kCcWasteAllowance) K = max(c.min_k, K / 2);
  st->total = total;
  st->v = v;
  st->comp = comp;
  st->small_run = small_run;
  st->K = K;
  if (stop) st->stop = 1;
}

// All blocks: every touched vertex takes, for each query, the component of the query's last real
// seed of the batch that reached it; then its arrivals of the batch go back to "unreached" (one
// warp per vertex; lane q < nq resolves query q from the warp's 256-bit mask of real seeds).
__device__ void cc_label_reset(const MultiArgs& a, const CcArgs& c, const CcSlots& sl) {
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nslots = sl.base[c.nq - 1] + sl.n[c.nq - 1];
  const int nt = __ldcg(a.ntouched);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  const int64_t nv = a.nv;
  for (int i = warp; i < nt; i += nwarps) {
    const int u = __ldcg(a.touched + i);
    uint32_t realw[kSlots];  // word k: slots k * 32 .. k * 32 + 31 that are real seeds reaching u
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const int j = k * 32 + lane;
      bool r = false;
      if (j < nslots) {
        const size_t at = arr_at(a, u, j);
        // prev is only ever set to an arrival, so an unset arrival has an unset prev as well
        if (__ldcg(a.arr + at) != kNoArrival) {
          r = __ldcg(c.comp_of + j) >= 0;
          a.arr[at] = kNoArrival;
          a.prev[at] = kNoArrival;
        }
      }
      realw[k] = __ballot_sync(kFull, r);
    }
    if (lane < c.nq && sl.n[lane] > 0) {
      const int lo = sl.base[lane], hi = lo + sl.n[lane];  // slots [lo, hi)
      int best = -1;
      for (int k = (hi - 1) >> 5; k >= (lo >> 5) && best < 0; --k) {
        uint32_t w = realw[0];
#pragma unroll
        for (int kk = 1; kk < kSlots; ++kk)
          if (kk == k) w = realw[kk];
        const int wlo = k * 32;
        if (hi - wlo < 32) w &= (1u << (hi - wlo)) - 1;
        if (lo > wlo) w &= ~((1u << (lo - wlo)) - 1);
        if (w) best = wlo + 31 - __clz(w);
      }
      if (best >= 0) {
        c.label[(size_t)lane * nv + u] = __ldcg(c.comp_of + best);
        c.reached[(size_t)lane * nv + u] = 1;
      }
    }
  }
}

__global__ void TGA_DECODE_BOUNDS k_cc_batches(GraphView g, MultiArgs a, CcArgs c) {
  __shared__ int64_t slo[kMaxSources], shi[kMaxSources];
  __shared__ int32_t scol[kMaxSources];
  __shared__ uint32_t reaches[kMaxSources][kMaxSources / 32];
  __shared__ uint32_t s_cnt[kMaxSources];
  __shared__ int32_t s_cand[kMaxSources];
  __shared__ int32_t s_wsum[kBlock / 32], s_count;
  __shared__ CcSlots sl;
  __shared__ int32_t hids[kHotSlots];
  hot_load(g, hids);  // (the first cc_allot synchronises the block)
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  const uint32_t epoch0 = a.epoch;
  const uint64_t t_start = global_ns();
  unsigned long long mine = 0;
  int levels = 0, batch = 0;
  for (;; ++batch) {
    // Decided by one thread, read by all after the barrier: every block leaves at the same batch.
    if (lead) a.ctl->yield = c.budget_ns > 0 && batch > 0 && (int64_t)(global_ns() - t_start) > c.budget_ns;
    cc_allot(c, sl);
    if (blockIdx.x < c.nq) cc_candidates(c, blockIdx.x, sl.base[blockIdx.x], sl.k[blockIdx.x], a.nv, s_wsum, &s_count);
    if (blockIdx.x == 0) {
      for (int s = threadIdx.x; s < kMaxSources; s += blockDim.x) c.counts[s] = 0;
      for (int e = threadIdx.x; e < kMaxSources * (kMaxSources / 32); e += blockDim.x) c.reach_bits[e] = 0;
      if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) a.ctl->cnt[k] = a.ctl->next[k] = a.ctl->dcnt[k] = a.ctl->dnext[k] = 0;
        *a.ntouched = 0;
      }
    }
    if (!grid_sync(a.ctl, g)) return;
    // A batch left here is redone by the next launch: its candidate scan changed nothing but
    // ncand/exhausted, which the scan recomputes from the same state.
    if (__ldcg(&a.ctl->yield)) break;
    // Live slots: [base_q, base_q + n_q) hold query q's candidates.
    if (threadIdx.x == 0) {
      int total = 0;
      for (int q = 0; q < c.nq; ++q) {
        sl.n[q] = __ldcg(&c.st[q].ncand);
        total += sl.n[q];
      }
      sl.total = total;
    }
    __syncthreads();
    if (sl.total == 0) {
      // No window has candidates: the exhausted ones are done (no block allots slots any more).
      if (lead)
        for (int q = 0; q < c.nq; ++q)
          if (__ldcg(&c.st[q].exhausted)) c.st[q].done = 1;
      break;
    }
    for (int s = threadIdx.x; s < kMaxSources; s += blockDim.x) {
      int q = 0;
      while (q + 1 < c.nq && s >= sl.base[q + 1]) ++q;
      const bool live = s >= sl.base[q] && s < sl.base[q] + sl.n[q];
      slo[s] = live ? c.q_lo[q] : 0;
      shi[s] = live ? c.q_hi[q] : 0;
      scol[s] = live ? q : 0;
    }
    __syncthreads();
    a.epoch = epoch0 + (uint32_t)batch;
    // Seeds: each live slot's candidate at max(lo, 0), as level 0's relaxation.
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < kMaxSources; s += gridDim.x * blockDim.x) {
      if (shi[s] <= slo[s]) continue;
      const int v = __ldcg(c.cand + s);
      a.arr[arr_at(a, v, s)] = (uint32_t)(slo[s] > 0 ? slo[s] : 0);
      if (atomicExch(&a.stamp[v], a.epoch) != a.epoch) a.touched[atomicAdd(a.ntouched, 1)] = v;
      if (v < a.nv_lists) {
        atomicOr((unsigned long long*)(a.F[1] + (size_t)v * kWords + s / 64), (unsigned long long)(1ull << (s & 63)));
        atomicOr(&a.dirty[v >> 5], 1u << (v & 31));
      }
    }
    if (!grid_sync(a.ctl, g)) return;
    int lv = 0;
    if (!multi_levels(g, a, slo, shi, scol, mine, lv, hids)) return;
    levels += lv;
    cc_count(a, c, sl, scol, s_cnt);
    if (!grid_sync(a.ctl, g)) return;
    if (blockIdx.x < c.nq) {
      if (threadIdx.x == 0 && __ldcg(&c.st[blockIdx.x].exhausted)) c.st[blockIdx.x].done = 1;
      if (sl.n[blockIdx.x] > 0) cc_validate(c, blockIdx.x, sl.base[blockIdx.x], sl.n[blockIdx.x], reaches, s_cnt, s_cand);
    }
    if (!grid_sync(a.ctl, g)) return;
    cc_label_reset(a, c, sl);
    if (!grid_sync(a.ctl, g)) return;
  }
  add_edges(a.edges, mine);
  if (lead) {
    a.ctl->levels = levels;
    a.ctl->batches = batch;
  }
}

__global__ void k_fill_column(int32_t* p, int32_t v, int64_t rows, int32_t stride) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < rows) p[i * stride] = v;
}

}  // namespace tga

// A CC job: up to `cap` windows in flight through k_cc_batches, each in its own slot with its own
// state, labels and run-table column.  Windows are added and taken between steps; a step runs
// batches until its time budget is used, always stopping at a batch boundary, where every batch
// has reset the multi-source state it used (other batched calls on the handle may run between
// steps).
struct tga_cc_job {
  tga::GraphHandle* h = nullptr;
  int32_t cap = 0, flags = 0;
  tga::DevBuf lab;    // labels [cap][nv] | reached [cap][nv]
  tga::DevBuf meta;   // states [cap] | lo [cap] | hi [cap] | counts | comp_of | pair matrix | run table [nruns][cap]
  std::vector<uint8_t> used;
  std::vector<tga::CcBatchState> st;  // host copy after the last step
  tga::CcArgs args{};
  int32_t* run_table = nullptr;  // [nruns][cap] for the decomposition of generation work_gen
  uint32_t work_gen = 0;
  ~tga_cc_job() {
    lab.release();
    meta.release();
  }
};

void tga::CcJobDeleter::operator()(tga_cc_job* j) const { delete j; }

size_t tga::cc_cache_bytes(const GraphHandle& h) {
  return h.cc_cache ? h.cc_cache->lab.bytes + h.cc_cache->meta.bytes : 0;
}

namespace tga {

static int cc_job_create(GraphHandle& h, int32_t cap, int32_t flags, tga_cc_job** out) {
  if (cap < 1 || cap > kMaxCcQueries) return fail(TGA_E_ARG, "CC job capacity must be 1..32");
  auto j = std::make_unique<tga_cc_job>();
  j->h = &h;
  j->cap = cap;
  j->flags = flags;
  j->work_gen = h.work_gen;
  const size_t nv = (size_t)h.view.max_vertex;
  const size_t st_bytes = (size_t)cap * sizeof(CcBatchState);
  const size_t fixed = st_bytes + (size_t)cap * 16 + kMaxSources * (8 + 4) + kMaxSources * kMaxSources / 8;
  TGA_TRY(j->lab.ensure((size_t)cap * nv * 5));
  TGA_TRY(j->meta.ensure(fixed + (size_t)std::max(h.nruns, 1) * cap * 4));
  CcArgs& c = j->args;
  c.nq = cap;
  c.label = j->lab.as<int32_t>();
  c.reached = reinterpret_cast<uint8_t*>(c.label + (size_t)cap * nv);
  c.st = j->meta.as<CcBatchState>();
  int64_t* win = reinterpret_cast<int64_t*>(j->meta.as<char>() + st_bytes);
  c.q_lo = win;
  c.q_hi = win + cap;
  c.counts = reinterpret_cast<unsigned long long*>(win + 2 * cap);
  c.comp_of = reinterpret_cast<int32_t*>(c.counts + kMaxSources);
  c.reach_bits = reinterpret_cast<uint32_t*>(c.comp_of + kMaxSources);
  j->run_table = reinterpret_cast<int32_t*>(j->meta.as<char>() + fixed);
  c.deg = h.d_deg.as<int32_t>();
  c.cand = nullptr;  // set per step (the handle's source slots)
  c.end = std::min(std::min(h.view.max_label, (int32_t)nv), h.view.n);
  c.early = (flags & TGA_CC_EARLY_EXIT) ? 1 : 0;
  c.min_k = c.end >= kCcLargeGraph ? kCcMinKLarge : kCcMinKSmall;
  c.limit = (int64_t)(0.8 * h.view.max_label);
  j->used.assign((size_t)cap, 0);
  j->st.assign((size_t)cap, CcBatchState{});
  for (auto& s0 : j->st) s0.done = 1;  // free slots take no source slots
  TGA_CUDA_TRY(cudaMemcpyAsync(c.st, j->st.data(), st_bytes, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  *out = j.release();
  return TGA_OK;
}

static int cc_job_current(const tga_cc_job* j) {
  if (j->work_gen != j->h->work_gen)
    return fail(TGA_E_ARG, "the graph's work decomposition changed after the CC job was created");
  return TGA_OK;
}

static int cc_job_add(tga_cc_job* j, int64_t t_lo, int64_t t_hi, int32_t* slot) {
  GraphHandle& h = *j->h;
  TGA_TRY(cc_job_current(j));
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  int32_t q = 0;
  while (q < j->cap && j->used[(size_t)q]) ++q;
  if (q == j->cap) return fail(TGA_E_AGAIN, "CC job full");
  const size_t nv = (size_t)h.view.max_vertex;
  CcArgs& c = j->args;
  CcBatchState s0{};
  s0.v = std::max(h.cfg.cc_vertex_begin, 0);
  s0.K = c.min_k;
  j->st[(size_t)q] = s0;
  // Pageable sources: each copy is staged before the call returns.
  TGA_CUDA_TRY(cudaMemcpyAsync(c.st + q, &s0, sizeof s0, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(const_cast<int64_t*>(c.q_lo) + q, &t_lo, 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(const_cast<int64_t*>(c.q_hi) + q, &t_hi, 8, cudaMemcpyHostToDevice, h.stream));
  KL(k_fill_i32, grid_for((int64_t)nv, kBlock))(c.label + (size_t)q * nv, -1, (int64_t)nv);
  TGA_CUDA_TRY(cudaMemsetAsync(c.reached + (size_t)q * nv, 0, nv, h.stream));
  if (h.nruns > 0) {
    KL(k_fill_column, grid_for(h.nruns, kBlock))(j->run_table + q, INT32_MAX, h.nruns, j->cap);
    KL(k_run_first_multi, grid_for(h.nrun_pairs, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_runs.as<RunInfo>(),
                                                         h.d_run_pairs.as<int2>(), h.nrun_pairs, c.q_lo + q,
                                                         c.q_hi + q, 1, j->run_table + q, j->cap);
  }
  TGA_CUDA_TRY(cudaGetLastError());
  j->used[(size_t)q] = 1;
  *slot = q;
  return TGA_OK;
}

// Runs batches until the windows in flight are all finished or budget_ms (> 0) of device time has
// passed.  finished (may be NULL): bit q set when slot q holds a finished window.
static int cc_job_step(tga_cc_job* j, double budget_ms, uint32_t* finished) {
  GraphHandle& h = *j->h;
  TGA_TRY(cc_job_current(j));
  TGA_TRY(multi_buffers(h, kMaxSources));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  MultiArgs a;
  TGA_TRY(multi_prepare(h, kMaxSources, edges, a));
  a.run_first = j->run_table;
  a.run_stride = j->cap;
  CcArgs c = j->args;
  c.cand = multi_src(h);
  c.budget_ns = budget_ms > 0 ? (int64_t)(budget_ms * 1e6) : 0;
  void* args[] = {&h.view, &a, &c};
  TravCtl ctl;
  TGA_TRY(multi_launch(h, (const void*)k_cc_batches, args, &ctl));
  h.m_epoch = a.epoch + (uint32_t)std::max(ctl.batches, 0);  // every batch reset its own entries
  TGA_CUDA_TRY(cudaMemcpyAsync(j->st.data(), j->args.st, (size_t)j->cap * sizeof(CcBatchState), cudaMemcpyDeviceToHost,
                               h.stream));
  h.timing.iterations = ctl.levels;
  const int rc = finish(h, edges);  // synchronizes the stream
  if (rc) return rc;
  if (finished) {
    uint32_t f = 0;
    for (int q = 0; q < j->cap; ++q)
      if (j->used[(size_t)q] && (j->st[(size_t)q].stop || j->st[(size_t)q].done)) f |= 1u << q;
    *finished = f;
  }
  return TGA_OK;
}

// Frees a slot whatever its state (a window left behind by a failed call).
static int cc_job_drop(tga_cc_job* j, int32_t slot) {
  GraphHandle& h = *j->h;
  CcBatchState off{};
  off.done = 1;
  j->st[(size_t)slot] = off;
  TGA_CUDA_TRY(cudaMemcpyAsync(j->args.st + slot, &off, sizeof off, cudaMemcpyHostToDevice, h.stream));
  j->used[(size_t)slot] = 0;
  return TGA_OK;
}

static int cc_job_take(tga_cc_job* j, int32_t slot, int32_t* label_out, int32_t* components_out) {
  GraphHandle& h = *j->h;
  if (slot < 0 || slot >= j->cap || !j->used[(size_t)slot]) return fail(TGA_E_ARG, "no window in this CC job slot");
  const CcBatchState& s0 = j->st[(size_t)slot];
  if (!s0.stop && !s0.done) return fail(TGA_E_AGAIN, "CC window not finished");
  const size_t nv = (size_t)h.view.max_vertex;
  if (label_out)
    TGA_CUDA_TRY(cudaMemcpyAsync(label_out, j->args.label + (size_t)slot * nv, nv * 4, cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  if (components_out) *components_out = s0.comp;
  j->used[(size_t)slot] = 0;
  return TGA_OK;
}

// One-shot form: nq (<= kMaxCcQueries) windows to completion in one launch, through the handle's
// cached job (kept between calls, so repeated calls allocate nothing).
static int cc_multi(GraphHandle& h, int32_t nq, const int64_t* t_lo, const int64_t* t_hi, int32_t flags,
                    int32_t* label_out, int32_t* components_out) {
  const size_t nv = (size_t)h.view.max_vertex;
  if (!h.cc_cache || h.cc_cache->flags != flags || h.cc_cache->cap < nq) {
    tga_cc_job* j = nullptr;
    h.cc_cache.reset();
    TGA_TRY(cc_job_create(h, kMaxCcQueries, flags, &j));
    h.cc_cache.reset(j);
  }
  tga_cc_job* j = h.cc_cache.get();
  for (int q = 0; q < j->cap; ++q)
    if (j->used[(size_t)q]) TGA_TRY(cc_job_drop(j, q));  // left over by a failed call
  std::vector<int32_t> slots((size_t)nq);
  for (int q = 0; q < nq; ++q) TGA_TRY(cc_job_add(j, t_lo[q], t_hi[q], &slots[(size_t)q]));
  uint32_t fin = 0;
  TGA_TRY(cc_job_step(j, 0.0, &fin));
  const tga_timing t = h.timing;
  for (int q = 0; q < nq; ++q)
    TGA_TRY(cc_job_take(j, slots[(size_t)q], label_out ? label_out + (size_t)q * nv : nullptr,
                        components_out ? components_out + q : nullptr));
  h.timing = t;
  return TGA_OK;
}

// ---------------------------------------------------------------------------------------------
// Multi-query PageRank: up to kMaxRankQueries windowed PageRanks as one strided vector
// (rank[v * S + q], S the smallest power of two >= the query count), each list decoded once per
// iteration.  Per edge the temporal weight is computed once and the contribution scattered to
// every query whose window holds the edge (first in-window occurrence of equal consecutive
// successors per query, as tga_pagerank).  Queries may ask for different iteration counts: the
// batch runs the largest, each query's result is taken after its own last iteration, and from then
// on its column is no longer scattered.

constexpr int kMaxRankQueries = 32;
constexpr int kSumParts = 128;  // blocks per query of the per-iteration sum

struct PrMultiArgs {
  const float* invdeg;       // [nv][S] 1 / in-window outdegree (windowed queries)
  const int32_t* deg;        // outdegrees (other queries)
  const float* in;
  float* out;
  float* reset;
  const double* sums_prev;   // [kMaxRankQueries] sums of the previous iteration, or null
  const int64_t* lo;
  const int64_t* hi;
  const int32_t* run_first;  // [nruns][kMaxSources]
  uint32_t windowed;         // bit q: query q uses its in-window outdegree
  uint32_t active;           // bit q: query q still iterating
  int32_t nq, nv, S;
  float damping, alpha, base;
  unsigned long long* edges;
};

__device__ __forceinline__ float temporal_weight_multi(float alpha, int64_t t) {
  const float a = alpha * (float)t;
  return a > 18.0f ? 1.0f : 1.0f - expf(-a);
}

// One iteration of the batch over the lean schedule (one entry per thread).  Contributions to the
// hot targets (hot.cuh) are summed per block and query in shared memory and added once per block:
// the queries' entries of one vertex share a cache line, so without that every query's adds to a
// hot vertex would queue at the same L2 slice.
__global__ void TGA_DECODE_BOUNDS k_pr_multi_iter(GraphView g, LeanWork lw, PrMultiArgs a) {
  __shared__ int64_t slo[kMaxRankQueries], shi[kMaxRankQueries];
  __shared__ float sinv[kMaxRankQueries];
  __shared__ int32_t hids[kHotSlots], hidx[kHotSlots];
  __shared__ float hacc[kHotMax * kMaxRankQueries];
  hot_load(g, hids, hidx);
  for (int i = threadIdx.x; i < kHotMax * kMaxRankQueries; i += blockDim.x) hacc[i] = 0.0f;
  for (int q = threadIdx.x; q < kMaxRankQueries; q += blockDim.x) {
    slo[q] = q < a.nq ? a.lo[q] : 0;
    shi[q] = q < a.nq ? a.hi[q] : 0;
    sinv[q] = (q < a.nq && a.sums_prev) ? (float)(1.0 / a.sums_prev[q]) : 1.0f;
  }
  __syncthreads();
  const int S = a.S;
  const int64_t total = (int64_t)a.nv * S;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
    a.reset[i] = a.base;
  float c0[kMaxRankQueries];
  uint32_t act = 0, seen = 0;
  int yprev = -1;
  constexpr int kKeepSeen = -3;
  const unsigned long long mine = run_lean<false, true, true>(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int v) { return v >= g.active_begin && v < g.max_label; },
      [&](int x, int first, int, int run) {
        act = 0;
        const float inv_all = a.deg[x] > 0 ? 1.0f / (float)a.deg[x] : 0.0f;
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q) {
          float c = 0.0f;
          if ((a.active >> q) & 1u) {
            const float inv = ((a.windowed >> q) & 1u) ? a.invdeg[(size_t)x * S + q] : inv_all;
            if (inv > 0.0f) c = a.damping * (a.in[(size_t)x * S + q] * sinv[q]) * inv;
          }
          c0[q] = c;
          if (c != 0.0f) act |= 1u << q;
        }
        seen = 0;
        yprev = -1;
        if (run >= 0) {
          const int32_t* rf = a.run_first + (size_t)run * kMaxSources;
          for (uint32_t c = act; c; c &= c - 1) {
            const int q = __ffs(c) - 1;
            if (__ldg(rf + q) < first) seen |= 1u << q;
          }
          yprev = kKeepSeen;
        }
        return act != 0;
      },
      [&](int, int y, int64_t t) {
        if (yprev == kKeepSeen) {
          yprev = y;
        } else if (y != yprev) {
          seen = 0;
          yprev = y;
        }
        const bool usable = y >= g.active_begin && y < g.max_vertex;
        const int hk = usable ? hot_index(hids, hidx, y) : -1;
        float wgt = 0.0f;
        bool have_w = false;
        for (uint32_t c = act & ~seen; c; c &= c - 1) {
          const int q = __ffs(c) - 1;
          if (t < slo[q] || t >= shi[q]) continue;
          seen |= 1u << q;
          if (!usable) continue;
          if (!have_w) {
            wgt = temporal_weight_multi(a.alpha, t);
            have_w = true;
          }
          if (hk >= 0) atomicAdd(&hacc[hk * S + q], c0[q] * wgt);
          else atomicAdd(&a.out[(size_t)y * S + q], c0[q] * wgt);
        }
        return true;
      },
      [](int) {});
  __syncthreads();
  for (int i = threadIdx.x; i < kHotSlots * S; i += blockDim.x) {
    const int sl = i / S, q = i % S;
    if (hids[sl] < 0) continue;
    const float v = hacc[hidx[sl] * S + q];
    if (v != 0.0f) atomicAdd(&a.out[(size_t)hids[sl] * S + q], v);
  }
  add_edges(a.edges, mine);
}

// In-window outdegree per query (lists counted by slices), then 1/count.
__global__ void TGA_DECODE_BOUNDS k_window_count_multi(GraphView g, LeanWork lw, const int64_t* lo, const int64_t* hi,
                                                     int32_t nq, int32_t S, int32_t* cnt, unsigned long long* edges) {
  __shared__ int64_t slo[kMaxRankQueries], shi[kMaxRankQueries];
  for (int q = threadIdx.x; q < kMaxRankQueries; q += blockDim.x) {
    slo[q] = q < nq ? lo[q] : 0;
    shi[q] = q < nq ? hi[q] : 0;
  }
  __syncthreads();
  int k[kMaxRankQueries];
  const unsigned long long mine = run_lean<false, true>(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int v) { return v >= g.active_begin && v < g.max_label; },
      [&](int, int, int) {
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q) k[q] = 0;
        return true;
      },
      [&](int, int, int64_t t) {
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q) {
          if (q >= nq) break;
          k[q] += (t >= slo[q] && t < shi[q]);
        }
        return true;
      },
      [&](int v) {
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q)
          if (q < nq && k[q]) atomicAdd(&cnt[(size_t)v * S + q], k[q]);
      });
  add_edges(edges, mine);
}

__global__ void k_invert_multi(const int32_t* cnt, float* inv, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) inv[i] = cnt[i] ? 1.0f / (float)cnt[i] : 0.0f;
}

// Per-iteration sums in FP64, deterministic: block (b, q) sums query q's entries of vertices
// b, b + kSumParts, ... into part[q][b]; then one thread per query adds its parts in order.
__global__ void k_sums_multi_part(const float* buf, int32_t nv, int32_t S, double* part) {
  const int q = blockIdx.y, b = blockIdx.x;
  double s = 0.0;
  for (int v = b * blockDim.x + threadIdx.x; v < nv; v += kSumParts * blockDim.x) s += (double)buf[(size_t)v * S + q];
  const double bs = block_sum(s);
  if (threadIdx.x == 0) part[q * kSumParts + b] = bs;
}

__global__ void k_sums_multi_fin(const double* part, int32_t nq, double* sums) {
  const int q = threadIdx.x;
  if (q >= nq) return;
  double s = 0.0;
  for (int b = 0; b < kSumParts; ++b) s += part[q * kSumParts + b];
  sums[q] = s;
}

// Results of the queries in `done` (bit q): out[q][v] = buf[v][q] / sums[q].
__global__ void k_pr_multi_final(const float* buf, const double* sums, uint32_t done, int32_t nq, int32_t nv,
                                 int32_t S, float* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nq * nv) return;
  const int q = (int)(i / nv), v = (int)(i % nv);
  if ((done >> q) & 1u) out[i] = (float)((double)buf[(size_t)v * S + q] / sums[q]);
}

// nq (<= kMaxRankQueries) queries, query q running iters[q] (>= 1) iterations.
// rows (optional): per query a destination of max_vertex entries (NULL: not copied) instead of
// the contiguous rank_out.
static int pagerank_multi_batch(GraphHandle& h, int32_t nq, const int32_t* iters, float damping, float alpha,
                                const int64_t* t_lo, const int64_t* t_hi, float* rank_out, float* const* rows = nullptr) {
  const size_t nv = (size_t)h.view.max_vertex;
  int32_t S = 1;
  while (S < nq) S <<= 1;
  int32_t maxit = 0;
  for (int q = 0; q < nq; ++q) maxit = std::max(maxit, iters[q]);
  const size_t vec = nv * (size_t)S;
  // s_a: 3 rank buffers | invdeg; s_b: counts; s_d: windows | sums | parts | run table; s_e: output
  TGA_TRY(h.s_a.ensure(vec * 4 * 4));
  TGA_TRY(h.s_b.ensure(vec * 4));
  const size_t run_bytes = (size_t)std::max(h.nruns, 1) * kMaxSources * 4;
  const size_t sums_off = kMaxSources * 16;
  const size_t sums_bytes = (size_t)(maxit + 1) * kMaxRankQueries * 8;
  const size_t part_bytes = (size_t)kMaxRankQueries * kSumParts * 8;
  TGA_TRY(h.s_d.ensure(sums_off + sums_bytes + part_bytes + run_bytes));
  TGA_TRY(h.s_e.ensure((size_t)nq * nv * 4));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  float* bufs[3] = {h.s_a.as<float>(), h.s_a.as<float>() + vec, h.s_a.as<float>() + 2 * vec};
  float* invdeg = h.s_a.as<float>() + 3 * vec;
  int32_t* cnt = h.s_b.as<int32_t>();
  int64_t* dlo = h.s_d.as<int64_t>();
  int64_t* dhi = dlo + kMaxSources;
  double* sums = reinterpret_cast<double*>(h.s_d.as<char>() + sums_off);
  double* part = reinterpret_cast<double*>(h.s_d.as<char>() + sums_off + sums_bytes);
  int32_t* drf = reinterpret_cast<int32_t*>(h.s_d.as<char>() + sums_off + sums_bytes + part_bytes);
  TGA_CUDA_TRY(cudaMemcpyAsync(dlo, t_lo, (size_t)nq * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dhi, t_hi, (size_t)nq * 8, cudaMemcpyHostToDevice, h.stream));
  uint32_t windowed = 0;
  for (int q = 0; q < nq; ++q)
    if (!(t_lo[q] <= 0 && t_hi[q] == TGA_T_MAX)) windowed |= 1u << q;
  if (h.nruns > 0) {
    KL(k_fill_i32, grid_for((int64_t)h.nruns * kMaxSources, kBlock))(drf, INT32_MAX, (int64_t)h.nruns * kMaxSources);
    KL(k_run_first_multi, grid_for(h.nrun_pairs, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_runs.as<RunInfo>(),
                                                         h.d_run_pairs.as<int2>(), h.nrun_pairs, dlo, dhi, nq, drf,
                                                         kMaxSources);
  }
  const float base = (1.0f - damping) / (float)h.view.max_label;
  KL(k_fill_f32, grid_for((int64_t)vec, kBlock))(bufs[0], 1.0f / (float)nv, (int64_t)vec);
  KL(k_fill_f32, grid_for((int64_t)vec, kBlock))(bufs[1], base, (int64_t)vec);
  if (windowed) {
    TGA_CUDA_TRY(cudaMemsetAsync(cnt, 0, vec * 4, h.stream));
    const LeanWork lw{h.d_lean.as<LeanEntry>(), h.nlean, h.d_slices.as<SliceState>(), h.d_run_first.as<int32_t>()};
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_window_count_multi, std::max(1u, grid_for(h.nlean, kBlock)))(h.view, lw, dlo, dhi, nq, S, cnt, edges);
    h.kernel_end(ev);
    KL(k_invert_multi, grid_for((int64_t)vec, kBlock))(cnt, invdeg, (int64_t)vec);
  }
  float* out = h.s_e.as<float>();
  // The iterations as one CUDA graph, replayed by later calls with the same parameters.
  std::vector<uint64_t> key = {ptr_key(bufs[0]), ptr_key(invdeg), ptr_key(sums), ptr_key(part), ptr_key(drf),
                               ptr_key(out), ptr_key(edges), (uint64_t)nq, (uint64_t)S, (uint64_t)nv,
                               (uint64_t)windowed, bits_of(damping), bits_of(alpha), ptr_key(dlo)};
  for (int q = 0; q < nq; ++q) key.push_back((uint64_t)iters[q]);
  TGA_TRY(run_loop(h, h.prm_loop, key, (size_t)maxit, [&]() -> int {
    const LeanWork lw{h.d_lean.as<LeanEntry>(), h.nlean, h.d_slices.as<SliceState>(), h.d_run_first.as<int32_t>()};
    for (int k = 0; k < maxit; ++k) {
      PrMultiArgs a{};
      a.invdeg = invdeg;
      a.deg = h.d_deg.as<int32_t>();
      a.in = bufs[k % 3];
      a.out = bufs[(k + 1) % 3];
      a.reset = bufs[(k + 2) % 3];
      a.sums_prev = k == 0 ? nullptr : sums + (size_t)(k - 1) * kMaxRankQueries;
      a.lo = dlo;
      a.hi = dhi;
      a.run_first = drf;
      a.windowed = windowed;
      uint32_t active = 0, done = 0;
      for (int q = 0; q < nq; ++q) {
        if (iters[q] > k) active |= 1u << q;
        if (iters[q] == k + 1) done |= 1u << q;
      }
      a.active = active;
      a.nq = nq;
      a.nv = (int32_t)nv;
      a.S = S;
      a.damping = damping;
      a.alpha = alpha;
      a.base = base;
      a.edges = edges;
      cudaEvent_t* ev = h.kernel_begin();
      KL(k_pr_multi_iter, std::max(1u, grid_for(h.nlean, kBlock)))(h.view, lw, a);
      h.kernel_end(ev);
      k_sums_multi_part<<<dim3(kSumParts, nq), kBlock, 0, h.stream>>>(a.out, (int32_t)nv, S, part);
      k_sums_multi_fin<<<1, kMaxRankQueries, 0, h.stream>>>(part, nq, sums + (size_t)k * kMaxRankQueries);
      h.timing.launches += 2;
      if (done)
        KL(k_pr_multi_final, grid_for((int64_t)nq * (int64_t)nv, kBlock))(a.out, sums + (size_t)k * kMaxRankQueries, done,
                                                                          nq, (int32_t)nv, S, out);
    }
    return TGA_OK;
  }));
  if (rank_out) TGA_CUDA_TRY(cudaMemcpyAsync(rank_out, out, (size_t)nq * nv * 4, cudaMemcpyDeviceToHost, h.stream));
  if (rows)
    for (int32_t q = 0; q < nq; ++q)
      if (rows[q]) TGA_CUDA_TRY(cudaMemcpyAsync(rows[q], out + (size_t)q * nv, nv * 4, cudaMemcpyDeviceToHost, h.stream));
  h.timing.iterations = maxit;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(maxit + (windowed ? 1 : 0)) *
                              (h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes);
  return rc;
}

int bfs_batch_rows(tga_graph* g, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                   int32_t* const* rows) {
  if (!g || nsrc < 0 || (nsrc && (!src || !t_lo || !t_hi || !rows))) return fail(TGA_E_ARG, "bad argument");
  GraphHandle& h = *g;
  for (int32_t i = 0; i < nsrc; ++i) {
    if (src[i] < 0 || src[i] >= h.view.max_vertex) return fail(TGA_E_ARG, "source out of range");
    if (t_lo[i] >= t_hi[i]) return fail(TGA_E_ARG, "empty time window");
  }
  for (int32_t b = 0; b < nsrc; b += kMaxSources)
    TGA_TRY(bfs_multi_batch(h, std::min(kMaxSources, nsrc - b), src + b, t_lo + b, t_hi + b, nullptr, rows + b));
  return TGA_OK;
}

int pagerank_batch_rows(tga_graph* g, int32_t nq, const int32_t* iters, float damping, float alpha,
                        const int64_t* t_lo, const int64_t* t_hi, float* const* rows) {
  if (!g || nq < 0 || (nq && (!iters || !t_lo || !t_hi || !rows))) return fail(TGA_E_ARG, "bad argument");
  GraphHandle& h = *g;
  for (int32_t i = 0; i < nq; ++i)
    if (t_lo[i] >= t_hi[i]) return fail(TGA_E_ARG, "empty time window");
  std::vector<int32_t> it((size_t)nq);
  for (int32_t i = 0; i < nq; ++i) it[(size_t)i] = iters[i] > 0 ? iters[i] : std::max(h.cfg.pr_iters, 1);
  for (int32_t b = 0; b < nq; b += kMaxRankQueries)
    TGA_TRY(pagerank_multi_batch(h, std::min(kMaxRankQueries, nq - b), it.data() + b, damping, alpha, t_lo + b, t_hi + b,
                                 nullptr, rows + b));
  return TGA_OK;
}

int cc_seed_batches(GraphHandle& h, int64_t t_lo, int64_t t_hi, int32_t flags, int32_t* label_out,
                    int32_t* components_out) {
  return cc_multi(h, 1, &t_lo, &t_hi, flags, label_out, components_out);
}

}  // namespace tga

using namespace tga;

extern "C" {

int tga_cc_job_create(tga_graph* g, int32_t capacity, int32_t flags, tga_cc_job** out) {
  if (!g || !out) return fail(TGA_E_ARG, "null argument");
  if (flags & ~TGA_CC_EARLY_EXIT) return fail(TGA_E_ARG, "tga_cc_job_create: only TGA_CC_EARLY_EXIT applies");
  return cc_job_create(*g, capacity, flags, out);
}

int tga_cc_job_add(tga_cc_job* j, int64_t t_lo, int64_t t_hi, int32_t* slot) {
  if (!j || !slot) return fail(TGA_E_ARG, "null argument");
  return cc_job_add(j, t_lo, t_hi, slot);
}

int tga_cc_job_step(tga_cc_job* j, double budget_ms, uint32_t* finished) {
  TGA_TRACE("tga_cc_job_step");
  if (!j) return fail(TGA_E_ARG, "null job");
  return cc_job_step(j, budget_ms, finished);
}

int tga_cc_job_take(tga_cc_job* j, int32_t slot, int32_t* label_out, int32_t* components_out) {
  if (!j) return fail(TGA_E_ARG, "null job");
  return cc_job_take(j, slot, label_out, components_out);
}

int tga_cc_job_destroy(tga_cc_job* j) {
  if (!j) return fail(TGA_E_ARG, "null job");
  cudaStreamSynchronize(j->h->stream);
  delete j;
  return TGA_OK;
}

int tga_cc_batch(tga_graph* g, int32_t nq, const int64_t* t_lo, const int64_t* t_hi, int32_t flags,
                 int32_t* label_out, int32_t* components_out) {
  TGA_TRACE("tga_cc_batch");
  if (!g || nq < 0 || (nq && (!t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  if (flags & ~TGA_CC_EARLY_EXIT) return fail(TGA_E_ARG, "tga_cc_batch: only TGA_CC_EARLY_EXIT applies");
  GraphHandle& h = *g;
  const size_t nv = (size_t)h.view.max_vertex;
  for (int32_t i = 0; i < nq; ++i)
    if (t_lo[i] >= t_hi[i]) return fail(TGA_E_ARG, "empty time window");
  tga_timing total{};
  for (int32_t b = 0; b < nq; b += kMaxCcQueries) {
    const int32_t k = std::min(kMaxCcQueries, nq - b);
    const int rc = cc_multi(h, k, t_lo + b, t_hi + b, flags, label_out ? label_out + (size_t)b * nv : nullptr,
                            components_out ? components_out + b : nullptr);
    if (rc) return rc;
    total.total_ms += h.timing.total_ms;
    total.decode_ms += h.timing.decode_ms;
    total.decode_launches += h.timing.decode_launches;
    total.edges_decoded += h.timing.edges_decoded;
    total.iterations += h.timing.iterations;
    total.launches += h.timing.launches;
  }
  h.timing = total;
  return TGA_OK;
}

int tga_bfs_batch(tga_graph* g, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                  int32_t* arrival_out) {
  TGA_TRACE("tga_bfs_batch");
  if (!g || nsrc < 0 || (nsrc && (!src || !t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  GraphHandle& h = *g;
  const size_t nv = (size_t)h.view.max_vertex;
  for (int32_t i = 0; i < nsrc; ++i) {
    if (src[i] < 0 || src[i] >= h.view.max_vertex) return fail(TGA_E_ARG, "source out of range");
    if (t_lo[i] >= t_hi[i]) return fail(TGA_E_ARG, "empty time window");
  }
  tga_timing total{};
  for (int32_t b = 0; b < nsrc; b += kMaxSources) {
    const int32_t k = std::min(kMaxSources, nsrc - b);
    const int rc = bfs_multi_batch(h, k, src + b, t_lo + b, t_hi + b, arrival_out ? arrival_out + (size_t)b * nv : nullptr);
    if (rc) return rc;
    total.total_ms += h.timing.total_ms;
    total.decode_ms += h.timing.decode_ms;
    total.decode_launches += h.timing.decode_launches;
    total.edges_decoded += h.timing.edges_decoded;
    total.iterations += h.timing.iterations;
    total.launches += h.timing.launches;
  }
  h.timing = total;
  return TGA_OK;
}

static int pagerank_batch_all(tga_graph* g, int32_t nq, const int32_t* iters, float damping, float alpha,
                              const int64_t* t_lo, const int64_t* t_hi, float* rank_out) {
  GraphHandle& h = *g;
  for (int32_t i = 0; i < nq; ++i)
    if (t_lo[i] >= t_hi[i]) return fail(TGA_E_ARG, "empty time window");
  const size_t nv = (size_t)h.view.max_vertex;
  std::vector<int32_t> it((size_t)nq);
  for (int32_t i = 0; i < nq; ++i) it[(size_t)i] = iters[i] > 0 ? iters[i] : std::max(h.cfg.pr_iters, 1);
  tga_timing total{};
  for (int32_t b = 0; b < nq; b += kMaxRankQueries) {
    const int32_t k = std::min(kMaxRankQueries, nq - b);
    const int rc = pagerank_multi_batch(h, k, it.data() + b, damping, alpha, t_lo + b, t_hi + b,
                                        rank_out ? rank_out + (size_t)b * nv : nullptr);
    if (rc) return rc;
    total.total_ms += h.timing.total_ms;
    total.decode_ms += h.timing.decode_ms;
    total.decode_launches += h.timing.decode_launches;
    total.edges_decoded += h.timing.edges_decoded;
    total.compressed_bytes += h.timing.compressed_bytes;
    total.iterations = std::max(total.iterations, h.timing.iterations);
    total.launches += h.timing.launches;
  }
  h.timing = total;
  return TGA_OK;
}

int tga_pagerank_batch(tga_graph* g, int32_t nq, int32_t iters, float damping, float alpha, const int64_t* t_lo,
                       const int64_t* t_hi, float* rank_out) {
  TGA_TRACE("tga_pagerank_batch");
  if (!g || nq < 0 || (nq && (!t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  std::vector<int32_t> it((size_t)nq, iters);
  return pagerank_batch_all(g, nq, it.data(), damping, alpha, t_lo, t_hi, rank_out);
}

int tga_pagerank_batch_iters(tga_graph* g, int32_t nq, const int32_t* iters, float damping, float alpha,
                             const int64_t* t_lo, const int64_t* t_hi, float* rank_out) {
  TGA_TRACE("tga_pagerank_batch_iters");
  if (!g || nq < 0 || (nq && (!iters || !t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  return pagerank_batch_all(g, nq, iters, damping, alpha, t_lo, t_hi, rank_out);
}

}  // extern "C"
