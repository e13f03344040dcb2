// Fused decode + algorithm kernels and their C ABI entry points (sweeps: neighbour access, raw
// decode, PageRank, HITS, degree centrality; colouring).  Every kernel decodes the
// successor lists and timestamps it needs straight from the compressed streams; decoded edges
// live only in registers.
//
// Work decomposition (slices.cuh): lists longer than a slice are cut into resumable slices.
// Sweeps over all lists follow a schedule built at load time in which lists are grouped by work
// class (outdegree bins), so the 32 lanes of a warp open lists together and decode lists of nearly
// equal length: with power-law outdegrees, lanes of mixed lists spend most of their time waiting
// for the longest list or for a neighbour opening its next one.  Traversals pull queue entries (a
// vertex id >= 0 or -(slice + 1)) from an atomic counter in a flat loop in which one iteration
// either decodes one edge or opens the next list.
#include <curand_kernel.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "gridsync.cuh"
#include "hot.cuh"
#include "lean.cuh"
#include "sweep.cuh"
#include "trace.cuh"

namespace tga {

// ---------------------------------------------------------------------------------------------
// Neighbour access and raw decode

__global__ void TGA_LEAN_BOUNDS k_neighbor_access(GraphView g, LeanWork lw, int32_t begin, int32_t end,
                                                         unsigned long long* csum, unsigned long long* edges) {
  uint64_t h = 0;
  uint32_t k = 0;
  const unsigned long long mine = run_lean(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int v) { return v >= begin && v < end; },
      [&](int, int first, int) {
        h = 0;
        k = (uint32_t)first;
        return true;
      },
      [&](int v, int y, int64_t t) {
        h += edge_hash((uint32_t)v, k++, y, t);
        return true;
      },
      [&](int v) { atomicAdd(&csum[v], (unsigned long long)h); });
  add_edges(edges, mine);
}

// Largest timestamp over all lists (a pass over the timestamp streams; run once at load).
// Largest (out[0]) and smallest (out[1]) timestamp of the graph.
__global__ void TGA_SWEEP_BOUNDS k_max_timestamp(GraphView g, Work w, long long* out) {
  long long m = LLONG_MIN, mn = LLONG_MAX;
  run_order<false>(
      g, w, [&](int) { return true; }, [&](int, int, int) { return true; },
      [&](int, int, int64_t t) {
        m = max(m, (long long)t);
        mn = min(mn, (long long)t);
        return true;
      },
      [&](int) {});
  for (int o = 16; o; o >>= 1) {
    m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0 && m != LLONG_MIN) atomicMax(out, m);
  if ((threadIdx.x & 31) == 0 && mn != LLONG_MAX) atomicMin(out + 1, mn);
}

__global__ void k_small_flags(const int32_t* deg, uint8_t* small, int32_t begin, int32_t end) {
  const int v = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (v < end) small[v] = deg[v] < 4;
}

__global__ void TGA_SWEEP_BOUNDS k_decode_csr(GraphView g, LeanWork lw, const int64_t* off, int32_t* dst, int64_t* ts,
                                               int64_t cap) {
  int64_t o = 0;
  run_lean(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int) { return true; },
      [&](int v, int first, int) {
        o = off[v] + first;
        return true;
      },
      [&](int, int y, int64_t t) {
        if (o < cap) {
          dst[o] = y;
          ts[o] = t;
        }
        ++o;
        return true;
      },
      [&](int) {});
}

__global__ void k_neighbors(GraphView g, int32_t v, int32_t* dst, int64_t* ts, int32_t cap, int32_t* count) {
  LeanCursor c;
  const int d = c.open_vertex(g, v);
  int i = 0, y;
  int64_t t;
  while (c.next(g, y, t)) {
    if (i < cap) {
      dst[i] = y;
      ts[i] = t;
    }
    ++i;
  }
  *count = d;
}

// Windowed point queries, one thread each, as EvolvingMultiGraph.isNeighbor(node, neighbor, from,
// to) (cpu_java/src/main/java/gr/uoa/di/networkanalysis/EvolvingMultiGraph.java:343-389): find the
// run of `neighbor` in node's successor list and report whether one of its timestamps lies in
// [from, to] (both ends inclusive).  Lists are sorted, so the run is the only one, and a sliced list
// is entered at its last slice whose first successor is below `neighbor` (binary search over the
// checkpoints, reading one successor per probe), then scanned slice by slice.
__global__ void TGA_DECODE_BOUNDS k_is_neighbor(GraphView g, int32_t nq, const int32_t* node, const int32_t* nbr,
                                                const int64_t* t_from, const int64_t* t_to, uint8_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const int x = node[i], want = nbr[i];
  const int64_t lo = t_from[i], hi = t_to[i];
  uint8_t found = 0;
  if (x >= 0 && x < g.n && want >= 0) {
    LeanCursor c;
    const int s0 = __ldg(g.slice_first + x), s1 = __ldg(g.slice_first + x + 1);
    int y;
    int64_t t;
    if (s1 - s0 > 1) {
      int a = s0, b = s1 - 1;
#pragma unroll 1
      while (a < b) {
        const int mid = (a + b + 1) >> 1;
        c.restore(g, g.slices[mid]);
        if (c.next<false>(g, y, t) && y < want) a = mid;
        else b = mid - 1;
      }
      bool stop = false;
#pragma unroll 1
      for (int k = a; k < s1 && !stop && !found; ++k) {
        c.restore(g, g.slices[k]);
        while (c.next(g, y, t)) {
          if (y < want) continue;
          if (y > want) {
            stop = true;
            break;
          }
          if (t >= lo && t <= hi) {
            found = 1;
            break;
          }
        }
      }
    } else {
      c.open_vertex(g, x);
      while (c.next<true>(g, y, t)) {
        if (y < want) continue;
        if (y > want) break;
        if (t >= lo && t <= hi) {
          found = 1;
          break;
        }
      }
    }
  }
  out[i] = found;
}

// ---------------------------------------------------------------------------------------------
// PageRank: one launch per iteration.  Three rank buffers rotate: iteration k reads IN (the
// unnormalised result of k-1, scaled by 1/sum[k-1]), scatters into OUT (already set to the base
// value) and resets RESET (read by iteration k-1, written by k+1) to the base value.

struct PrArgs {
  const float* invdeg;   // per-vertex 1/deg for a window, or nullptr (use outdegree)
  const int32_t* deg;
  const float* in;
  float* out;
  float* reset;
  double* sums;
  int32_t k;
  float damping, alpha, base;
  int64_t lo, hi;
  unsigned long long* edges;
};

// 1 - exp(-alpha t): for alpha*t > 18 expf is below 2^-25 and the difference rounds to 1.0f.
__device__ __forceinline__ float temporal_weight(float alpha, int64_t t) {
  const float a = alpha * (float)t;
  return a > 18.0f ? 1.0f : 1.0f - expf(-a);
}

// k_pr_iter over the lean schedule (kAll: the window holds every timestamp of the graph, so no
// edge is tested against it).
template <bool kAll>
__global__ void TGA_LEAN_BOUNDS k_pr_iter(GraphView g, LeanWork lw, PrArgs a) {
  TGA_HOT_SHARED(float, hot)
  hot.init(g);
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < g.max_vertex; x += gridDim.x * blockDim.x) a.reset[x] = a.base;
  const double s = a.k == 0 ? 1.0 : 1.0 / a.sums[a.k - 1];
  float local = 0.0f, c0 = 0.0f;
  double total = 0.0;
  int prev_y = -1;
  // The source's rank and degree are loaded when the entry is taken and used once the list is open,
  // so their latency overlaps the open instead of preceding it.
  float in_v = 0.0f, inv_v = 0.0f;
  int deg_v = 0;
  const unsigned long long mine = run_lean<true>(
      g, lw.e, lw.count, lw.slices, lw.run_first,
      [&](int v) {
        if (v < g.active_begin || v >= g.max_label) return false;
        in_v = __ldg(a.in + v);
        if (a.invdeg) inv_v = __ldg(a.invdeg + v);
        else deg_v = __ldg(a.deg + v);
        return true;
      },
      [&](int v, int, int) {
        const float inv = a.invdeg ? inv_v : (deg_v > 0 ? 1.0f / (float)deg_v : 0.0f);
        if (inv == 0.0f) return false;  // no (in-window) out-edges: nothing to scatter
        c0 = a.damping * (float)((double)in_v * s) * inv;
        prev_y = -1;
        local = 0.0f;
        return true;
      },
      [&](int, int y, int64_t t) {
        if (!(kAll ? keep_edge_all(g, y, prev_y) : keep_edge(g, a.lo, a.hi, y, t, prev_y))) return true;
        const float contrib = c0 * temporal_weight(a.alpha, t);
        if (!hot.add(y, contrib)) atomicAdd(&a.out[y], contrib);
        local += contrib;
        return true;
      },
      [&](int) { total += (double)local; });
  hot.flush(a.out);
  // (per warp: per-block sums measured 0.782 against 0.764 ms per launch here)
  add_edges(a.edges, mine);
  warp_add(&a.sums[a.k], total);
}

__global__ void k_pr_init_sums(double* sums, int n, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sums[i] = v;
}

__global__ void k_pr_final(const float* buf, const double* sums, int k, float* out, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)((double)buf[i] / sums[k]);
}

// In-window outdegree of each source, counted over items, then inverted.
__global__ void TGA_SWEEP_BOUNDS k_window_count(GraphView g, LeanWork lw, int64_t lo, int64_t hi, int32_t* cnt,
                                                 unsigned long long* edges) {
  int k = 0;
  const unsigned long long mine = run_lean(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int v) { return v >= g.active_begin && v < g.max_label; },
      [&](int, int, int) {
        k = 0;
        return true;
      },
      [&](int, int, int64_t t) {
        k += (t >= lo && t < hi);
        return true;
      },
      [&](int v) {
        if (k) atomicAdd(&cnt[v], k);
      });
  add_edges(edges, mine);
}

__global__ void k_invert(const int32_t* cnt, float* inv, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) inv[i] = cnt[i] ? 1.0f / (float)cnt[i] : 0.0f;
}

// ---------------------------------------------------------------------------------------------
// HITS.  Per iteration: hub base (vector), hub gather (items), sum hub^2, authority scatter
// (items), normalise hub, sum auth^2.  Authorities are kept unnormalised between iterations
// and scaled by 1/||auth|| when read.
//
// Per-edge arithmetic is FP32; the hub and authority accumulators are FP64.  With preferential
// in-degrees one authority receives about a million contributions per half step, each some 10^5
// times smaller than the running sum: in an FP32 accumulator every addition loses up to half an
// ulp of the sum, which biased that authority by 0.3% after one iteration on the 2M/40M graph.

__global__ void k_hits_base(double* hub, const double* auth_in, double* auth_next, const double* aprev, int java,
                            int32_t n) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  const double sa = (aprev && *aprev > 0) ? 1.0 / sqrt(*aprev) : 1.0;
  if (java) hub[x] = 0.0;
  auth_next[x] = java ? 0.0 : auth_in[x] * sa;
}

template <bool kTimes>
__global__ void TGA_LEAN_BOUNDS5 k_hits_hub(GraphView g, LeanWork lw, double* hub, const double* auth_in,
                                           const double* aprev, int64_t lo, int64_t hi, unsigned long long* edges) {
  const float sa = (aprev && *aprev > 0) ? (float)(1.0 / sqrt(*aprev)) : 1.0f;
  float acc = 0.0f;
  int prev_y = -1;
  const unsigned long long mine = run_lean<true, kTimes, false, !kTimes>(
      g, lw.e, lw.count, lw.slices, lw.run_first, [&](int v) { return v >= g.active_begin && v < g.max_label; },
      [&](int, int, int) {
        acc = 0.0f;
        prev_y = -1;
        return true;
      },
      [&](int, int y, int64_t t) {
        if (kTimes ? keep_edge(g, lo, hi, y, t, prev_y) : keep_edge_all(g, y, prev_y)) acc += (float)auth_in[y];
        return 2;  // repeats of y add nothing
      },
      [&](int v) {
        if (acc != 0.0f) atomicAdd(&hub[v], (double)(acc * sa));
      });
  block_add_edges(edges, mine);
}

template <bool kTimes>
__global__ void TGA_LEAN_BOUNDS5 k_hits_auth(GraphView g, LeanWork lw, const double* hub, const double* hsum,
                                            double* auth_next, int64_t lo, int64_t hi, unsigned long long* edges) {
  // Hot authorities take block-local FP32 partials (a few hundred contributions per block),
  // added to the FP64 accumulators once per block.
  TGA_HOT_SHARED(float, hot)
  hot.init(g);
  const double sh = *hsum > 0 ? 1.0 / sqrt(*hsum) : 1.0;
  float hn = 0.0f;
  double hub_v = 0.0;
  int prev_y = -1;
  const unsigned long long mine = run_lean<true, kTimes, false, !kTimes>(
      g, lw.e, lw.count, lw.slices, lw.run_first,
      [&](int v) {
        if (v < g.active_begin || v >= g.max_label) return false;
        hub_v = __ldg(hub + v);  // used once the list is open (see k_pr_iter)
        return true;
      },
      [&](int, int, int) {
        if (hub_v == 0.0) return false;
        hn = (float)(hub_v * sh);
        prev_y = -1;
        return true;
      },
      [&](int, int y, int64_t t) {
        if ((kTimes ? keep_edge(g, lo, hi, y, t, prev_y) : keep_edge_all(g, y, prev_y)) && !hot.add(y, hn))
          atomicAdd(&auth_next[y], (double)hn);
        return 2;  // repeats of y add nothing
      },
      [&](int) {});
  hot.flush(auth_next);
  block_add_edges(edges, mine);
}

__global__ void k_sumsq(const double* v, int32_t n, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double x = i < n ? v[i] : 0.0;
  const double bs = block_sum(x * x);
  if (threadIdx.x == 0 && bs != 0.0) atomicAdd(out, bs);
}

// out = v / ||v|| (out may be v).
template <class Out>
__global__ void k_scale(const double* v, const double* sumsq, Out* out, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = *sumsq > 0 ? 1.0 / sqrt(*sumsq) : 1.0;
  out[i] = (Out)(v[i] * s);
}

// ---------------------------------------------------------------------------------------------
// Degree centrality (Java semantics).  Short lists: one thread per list.

__global__ void TGA_TRAVERSE_BOUNDS k_degree(GraphView g, LeanWork lw, int64_t s, int64_t e, int32_t* deg, int64_t* avg,
                                           unsigned long long* edges) {
  const bool all = (s == 0 && e == 0);
  const int lim = min(g.max_label + 1, g.max_vertex);
  int32_t d = 0;
  int64_t mean = 0;
  const unsigned long long mine = run_lean(
      g, lw.e, lw.count, lw.slices, lw.run_first,
      [&](int v) { return v >= g.active_begin && v <= g.max_label && g.slice_first[v] == g.slice_first[v + 1]; },
      [&](int, int, int) {
        d = 0;
        mean = 0;
        return true;
      },
      [&](int, int y, int64_t t) {
        if (y >= g.active_begin && y < lim && (all || (s <= t && e >= t))) {
          ++d;
          mean += (t - mean) / d;
        }
        return true;
      },
      [&](int v) {
        if (s != e) d = (int32_t)(0.85 * d + 0.15 * d * (double)(mean - s) / (double)(e - s) + 1);
        deg[v] = d;
        avg[v] = mean;
      });
  add_edges(edges, mine);
}

// Long (sliced) lists in two phases: every slice decodes its edges in parallel and writes each
// edge's timestamp, or kDcSkip when the edge does not count, at its list position; then one thread
// per long list runs the sequential running mean over its segment (the Java mean truncates at
// every step, so it cannot be split), with a 32-bit division whenever the difference fits.
constexpr int64_t kDcSkip = INT64_MIN;

__global__ void TGA_TRAVERSE_BOUNDS k_degree_slices(GraphView g, const SliceState* slices, const int64_t* ebase,
                                                  int32_t nslices, int64_t s, int64_t e, int64_t* buf,
                                                  int32_t* scnt, unsigned long long* edges) {
  const bool all = (s == 0 && e == 0);
  const int lim = min(g.max_label + 1, g.max_vertex);
  unsigned long long mine = 0;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nslices) {
    const SliceState& sl = slices[j];
    int counted = 0;
    if (sl.v >= g.active_begin && sl.v <= g.max_label) {
      LeanCursor c;
      c.restore(g, sl);
      int64_t* out = buf + ebase[j];
      int y;
      int64_t t;
      while (c.next(g, y, t)) {
        const bool in = y >= g.active_begin && y < lim && (all || (s <= t && e >= t));
        *out++ = in ? t : kDcSkip;
        counted += in;
        ++mine;
      }
    }
    scnt[j] = counted;
  }
  add_edges(edges, mine);
}

// Where each slice's counted timestamps go in the compacted buffer: one warp per long list scans
// its slices' counts 32 at a time; cnt[i] = the list's counted total.
__global__ void k_degree_bases(const LongList* longs, int32_t nlong, const int32_t* slice_first, const int32_t* scnt,
                               int32_t active, int32_t max_label, int64_t* cbase, int32_t* cnt) {
  constexpr unsigned kFull = 0xffffffffu;
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (i >= nlong) return;  // (whole warps leave together)
  const int v = longs[i].v;
  if (v < active || v > max_label) return;
  const int a = slice_first[v], b = slice_first[v + 1];
  int64_t running = longs[i].base;
  for (int j0 = a; j0 < b; j0 += 32) {
    const int j = j0 + lane;
    const int c = j < b ? scnt[j] : 0;
    int incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += u;
    }
    if (j < b) cbase[j] = running + incl - c;
    running += __shfl_sync(kFull, incl, 31);
  }
  if (lane == 0) cnt[i] = (int32_t)(running - longs[i].base);
}

// The counted timestamps of every slice to their place in the compacted buffer (one thread per
// slice, so the longest list's compaction is spread over all of its slices).
__global__ void k_degree_gather(const SliceState* slices, int32_t nslices, const int64_t* ebase, const int64_t* cbase,
                                const int32_t* scnt, const int64_t* buf, int64_t* cbuf) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nslices || scnt[j] == 0) return;
  const int64_t* in = buf + ebase[j];
  int64_t* out = cbuf + cbase[j];
  const int n = slices[j].count;
  for (int k = 0; k < n; ++k) {
    const int64_t t = in[k];
    if (t != kDcSkip) *out++ = t;
  }
}

// kNarrow: every timestamp t of the graph satisfies 0 <= t - base < 2^31 (base = the smallest),
// so the mean is carried as mean - base in 32 bits; t - mean and every intermediate are the same
// integers as in 64 bits, and the recurrence's critical path is single-word arithmetic.
// One thread per long list runs the sequential truncating mean over its compacted counted
// timestamps (the Java mean truncates at every step, so it cannot be split).
template <bool kNarrow>
__global__ void k_degree_long(const LongList* longs, int32_t nlong, const int32_t* cnt, const int64_t* buf,
                              const uint2* divtab, int64_t base, int32_t active, int32_t max_label, int64_t s,
                              int64_t e, int32_t* deg, int64_t* avg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nlong) return;
  const int v = longs[i].v;
  if (v < active || v > max_label) return;
  const int64_t* p = buf + longs[i].base;
  const int n = cnt[i];
  int64_t mean = 0;     // 64-bit form
  int32_t mean32 = 0;   // narrow form: mean - base
  // Step d (the d-th counted timestamp t, d >= 2): mean += (t - mean) / d (Java long division,
  // towards zero); when |t - mean| < 2^31 the quotient is one multiply-high and one shift with d's
  // entry ml of the division table (ml.x = M, ml.y = l - 1).
  auto step = [&](int64_t t, uint2 ml, int d) {
    if constexpr (kNarrow) {
      const int32_t a = (int32_t)(t - base) - mean32;
      const uint32_t x = (uint32_t)(a < 0 ? -a : a);
      const int32_t q = (int32_t)(__umulhi(ml.x, x) >> ml.y);
      mean32 += a < 0 ? -q : q;
    } else {
      const int64_t a = t - mean;
      const uint64_t na = (uint64_t)(a < 0 ? -a : a);
      if (na < 0x80000000ull) {
        const uint32_t q = __umulhi(ml.x, (uint32_t)na) >> ml.y;
        mean += a < 0 ? -(int64_t)q : (int64_t)q;
      } else {
        mean += a / d;
      }
    }
  };
  if (n > 0) {
    // d = 1 sets the mean to the first timestamp.
    if constexpr (kNarrow) mean32 = (int32_t)(p[0] - base);
    else mean = p[0];
  }
  // Inputs and divisor entries in flight two batches ahead of the recurrence.
  constexpr int kBatch = 8;
  int64_t b0[kBatch], b1[kBatch];
  uint2 m0[kBatch], m1[kBatch];
  int k = 1;
  auto load = [&](int at, int64_t* tb, uint2* mb) {
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      tb[j] = __ldcs(p + at + j);
      mb[j] = __ldg(divtab + at + j + 1);
    }
  };
  if (n - 1 >= 2 * kBatch) {
    load(1, b0, m0);
    load(1 + kBatch, b1, m1);
    for (; k + 3 * kBatch <= n; k += kBatch) {
      int64_t tb[kBatch];
      uint2 mb[kBatch];
      load(k + 2 * kBatch, tb, mb);
#pragma unroll
      for (int j = 0; j < kBatch; ++j) step(b0[j], m0[j], k + j + 1);
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        b0[j] = b1[j];
        m0[j] = m1[j];
        b1[j] = tb[j];
        m1[j] = mb[j];
      }
    }
#pragma unroll
    for (int j = 0; j < kBatch; ++j) step(b0[j], m0[j], k + j + 1);
    k += kBatch;
#pragma unroll
    for (int j = 0; j < kBatch; ++j) step(b1[j], m1[j], k + j + 1);
    k += kBatch;
  }
  for (; k < n; ++k) step(p[k], __ldg(divtab + k + 1), k + 1);
  if constexpr (kNarrow) mean = n > 0 ? base + (int64_t)mean32 : 0;
  int32_t d = n;
  if (s != e) d = (int32_t)(0.85 * d + 0.15 * d * (double)(mean - s) / (double)(e - s) + 1);
  deg[v] = d;
  avg[v] = mean;
}

// Lists of length zero never reach the loop above; their centrality is the formula at d = 0.
__global__ void k_degree_empty(const int32_t* outdeg, int32_t active, int32_t max_label, int32_t n, int64_t s, int64_t e,
                               int32_t* deg) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n || v < active || v > max_label || outdeg[v] != 0) return;
  deg[v] = (s != e) ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// Jones-Plassmann colouring: per round a check over queue entries (vertices or slices) marks
// vertices that have a higher-priority uncoloured neighbour, then a decision pass colours the
// others and builds the next worklist; the check builds the next entry queue.

// The reference's cuRAND priorities: vertex v draws the first value of subsequence v of seed 123
// (curand_init(123, v, 0); curand() % 256).  curand_init jumps to subsequence v with one jump per
// set bit of v; the state of subsequence v + 1 is that of v advanced by one subsequence
// (skipahead_sequence(1, .)), one jump, so each thread initialises the first vertex of a run of
// kPrioRun vertices and steps through the others (2M vertices: 3.5 -> 0.3 ms).
constexpr int kPrioRun = 32;
__global__ void k_gc_prio_curand(uint32_t* prio, int32_t n) {
  const int64_t v0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * kPrioRun;
  if (v0 >= n) return;
  const int v1 = (int)(v0 + kPrioRun < (int64_t)n ? v0 + kPrioRun : (int64_t)n);
  curandState st;
  curand_init(123ull, (unsigned long long)v0, 0ull, &st);
  for (int v = (int)v0; v < v1; ++v) {
    curandState draw = st;
    prio[v] = curand(&draw) % 256u;
    if (v + 1 < v1) skipahead_sequence(1ull, &st);
  }
}

// Resume point of a colouring queue entry (a short list or a slice) that a neighbour blocked:
// the decoder state after that neighbour, and the neighbour.  A neighbour that does not block
// (lower priority, or coloured) never blocks later, since colours are only ever assigned, so the
// next round re-checks the blocking neighbour and goes on from there instead of decoding the
// entry again from its start; an entry that was not blocked is not checked again at all.
struct GcPoint {
  ListState top;
  uint32_t cnext, cend;
  int32_t remaining;
  int32_t yb;
};

// One round's check: one queue entry per thread (round 0 opens every entry, later rounds resume
// the blocked ones from their points).  A blocked entry marks its vertex (found = round + 1),
// saves its point and joins the next round's queue.
__global__ void TGA_LEAN_BOUNDS5 k_gc_check(GraphView g, const int32_t* entries, int32_t en, int32_t nv,
                                           const uint32_t* color, const uint32_t* prio, uint32_t round,
                                           uint32_t* found, GcPoint* pts, int32_t* next, int32_t* next_cnt,
                                           unsigned long long* edges) {
  constexpr unsigned kFull = 0xffffffffu;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  bool blocked = false;
  int e = 0;
  if (i < en) {
    e = __ldcg(entries + i);
    const int x = e >= 0 ? e : g.slices[-e - 1].v;
    const size_t pid = e >= 0 ? (size_t)e : (size_t)nv + (size_t)(-e - 1);
    const uint32_t px = prio[x];
    auto blocks = [&](int y) {
      const uint32_t py = prio[y];
      return (py > px || (py == px && y < x)) && color[y] >= round;
    };
    LeanCursor c;
    int prev_y = -1;
    bool go = true;
    if (round == 0) {
      if (e >= 0) c.open_vertex(g, e);
      else c.restore(g, g.slices[-e - 1]);
    } else {
      const GcPoint& p = pts[pid];
      const int yb = p.yb;
      if (blocks(yb)) {
        blocked = true;  // the same neighbour blocks again: the point stays
        go = false;
      } else {
        c.resume_successors(g, p.top, p.cnext, p.cend, p.remaining);
        prev_y = yb;
      }
    }
    if (go) {
      int y;
      int64_t t;
      while (c.template next<false>(g, y, t)) {
        ++mine;
        if (y == prev_y) continue;
        prev_y = y;
        if (y < g.active_begin || y >= g.max_vertex) continue;
        if (blocks(y)) {
          GcPoint& p = pts[pid];
          c.save_successors(g, p.top, p.cnext, p.cend);
          p.remaining = c.remaining;
          p.yb = y;
          blocked = true;
          break;
        }
      }
    }
    if (blocked) found[x] = round + 1;
  }
  // blocked entries to the next queue, one atomic per warp
  const unsigned m = __ballot_sync(kFull, blocked);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && m) base = atomicAdd(next_cnt, __popc(m));
  base = __shfl_sync(kFull, base, 0);
  if (blocked) next[base + __popc(m & ((1u << lane) - 1))] = e;
  add_edges(edges, mine);
}

__global__ void k_gc_decide(GraphView g, const int32_t* wl, int32_t wn, const int32_t* deg, uint32_t* color,
                            const uint32_t* found, uint32_t round, int java_isolated, int32_t* out_wl, int32_t* out_n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int x = -1;
  bool keep = false;  // stays uncoloured: joins the next worklist
  if (i < wn) {
    x = wl[i];
    if (x >= g.active_begin && x <= g.max_label && color[x] == kColorInf) {
      if (x >= g.n || deg[x] == 0) {
        if (java_isolated) color[x] = round;
      } else if (found[x] == round + 1) {
        keep = true;
      } else {
        color[x] = round;
      }
    }
  }
  // places reserved per warp (all lanes of the warp take part)
  const int at = warp_reserve(out_n, keep ? 1 : 0);
  if (keep) out_wl[at] = x;
}

// The first round: every vertex on the worklist (in order), the entries of every list with edges
// in the queue (places reserved per warp: one atomic per vertex on one counter would queue 2M
// requests at one L2 slice).
__global__ void k_gc_first(GraphView g, Work w, const int32_t* deg, int32_t n, int32_t* wl, int32_t* entries,
                           int32_t* en) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = x < n;
  if (in) wl[x] = x;
  const bool listed = in && x >= g.active_begin && x <= g.max_label && x < g.n && deg[x] > 0;
  const int at = warp_reserve(en, listed ? entry_count(w, x) : 0);
  if (listed) write_entries(w, x, entries, at);
}

// Host side: the queue entries of one vertex (itself or its slices).
int compute_max_timestamp(GraphHandle& h) {
  h.max_ts = INT64_MAX;
  h.min_ts_data = INT64_MIN;
  if (int rc = h.s_sum.ensure(4096)) return rc;
  long long* out = reinterpret_cast<long long*>(h.s_sum.as<char>() + 3968);
  const long long init[2] = {LLONG_MIN, LLONG_MAX};
  TGA_CUDA_TRY(cudaMemcpyAsync(out, init, 16, cudaMemcpyHostToDevice, h.stream));
  const Work w = work_of(h);
  k_max_timestamp<<<sweep_grid(h), kBlock, 0, h.stream>>>(h.view, w, out);
  TGA_CUDA_TRY(cudaGetLastError());
  long long m[2] = {LLONG_MIN, LLONG_MAX};
  TGA_CUDA_TRY(cudaMemcpyAsync(m, out, 16, cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  if (int rc = h.check_device_error()) return rc;
  h.max_ts = (m[0] == LLONG_MIN) ? h.view.min_ts : (int64_t)m[0];
  h.min_ts_data = (m[1] == LLONG_MAX) ? h.view.min_ts : (int64_t)m[1];
  return TGA_OK;
}

static LeanWork lean_work(const GraphHandle& h) {
  return LeanWork{h.d_lean.as<LeanEntry>(), h.nlean, h.d_slices.as<SliceState>(), h.d_run_first.as<int32_t>()};
}
static unsigned lean_grid(const GraphHandle& h) { return std::max(1u, grid_for(h.nlean, kBlock)); }

// Hot scatter targets (hot.cuh): in-degrees counted on the device, the largest kept on the host.
// TGA_HOT=0 leaves the table out (every target on the global path).
int build_hot(GraphHandle& h) {
  h.view.hot = nullptr;
  h.nhot = 0;
  const char* env = std::getenv("TGA_HOT");
  const int64_t n = (int64_t)h.degrees.size();
  if ((env && std::atoi(env) == 0) || n == 0 || h.nlean == 0) return publish_view(h);
  DevBuf d_in;
  if (int rc = d_in.ensure((size_t)n * 4)) return rc;
  TGA_CUDA_TRY(cudaMemsetAsync(d_in.p, 0, (size_t)n * 4, h.stream));
  k_in_degree<<<lean_grid(h), kBlock, 0, h.stream>>>(h.view, lean_work(h), d_in.as<int32_t>());
  TGA_CUDA_TRY(cudaGetLastError());
  std::vector<int32_t> indeg((size_t)n);
  TGA_CUDA_TRY(cudaMemcpyAsync(indeg.data(), d_in.p, (size_t)n * 4, cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  if (int rc = h.check_device_error()) return rc;
  std::vector<int32_t> ids((size_t)n);
  for (int64_t i = 0; i < n; ++i) ids[(size_t)i] = (int32_t)i;
  const size_t k = std::min<size_t>((size_t)kHotMax, ids.size());
  std::partial_sort(ids.begin(), ids.begin() + (ptrdiff_t)k, ids.end(), [&](int32_t a, int32_t b) {
    return indeg[(size_t)a] != indeg[(size_t)b] ? indeg[(size_t)a] > indeg[(size_t)b] : a < b;
  });
  const int64_t min_in = std::max<int64_t>(2, (int64_t)(h.info_edges / kHotMinShare));
  std::vector<int32_t> table(2 * kHotSlots, -1);  // ids, then compact indexes
  int placed = 0;
  for (size_t i = 0; i < k; ++i) {
    const int32_t y = ids[i];
    if (indeg[(size_t)y] < min_in) break;
    const size_t s = (size_t)hot_slot(y);
    if (table[s] < 0) {
      table[s] = y;
      table[kHotSlots + s] = placed++;
    }
  }
  for (size_t s = 0; s < (size_t)kHotSlots; ++s)
    if (table[s] < 0) table[kHotSlots + s] = 0;
  if (placed > 0) {
    if (int rc = h.d_hot.ensure(2 * kHotSlots * 4)) return rc;
    TGA_CUDA_TRY(cudaMemcpy(h.d_hot.p, table.data(), 2 * kHotSlots * 4, cudaMemcpyHostToDevice));
    h.view.hot = h.d_hot.as<int32_t>();
    h.nhot = placed;
  }
  return publish_view(h);
}

}  // namespace tga

using namespace tga;

// ---------------------------------------------------------------------------------------------
// C ABI

extern "C" {

int tga_neighbor_access(tga_graph* gp, uint8_t* small_out, uint64_t* checksum_out, int32_t* degree_out) {
  TGA_TRACE("tga_neighbor_access");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(h.s_a.ensure((size_t)nv));
  TGA_TRY(h.s_b.ensure((size_t)nv * 8));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  if (!edges) return fail(TGA_E_OOM, "counter allocation failed");
  cudaMemsetAsync(h.s_a.p, 0, (size_t)nv, h.stream);
  cudaMemsetAsync(h.s_b.p, 0, (size_t)nv * 8, h.stream);
  const int32_t b = h.view.active_begin, e = std::min(h.view.max_label, h.view.n);
  if (e > b) {
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_neighbor_access, lean_grid(h))(h.view, lean_work(h), b, e, h.s_b.as<unsigned long long>(), edges);
    h.kernel_end(ev);
    KL(k_small_flags, grid_for(e - b, kBlock))(h.d_deg.as<int32_t>(), h.s_a.as<uint8_t>(), b, e);
  }
  if (small_out) cudaMemcpyAsync(small_out, h.s_a.p, (size_t)nv, cudaMemcpyDeviceToHost, h.stream);
  if (checksum_out) cudaMemcpyAsync(checksum_out, h.s_b.p, (size_t)nv * 8, cudaMemcpyDeviceToHost, h.stream);
  if (degree_out) cudaMemcpyAsync(degree_out, h.d_deg.p, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = 1;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = pass_bytes(h);
  return rc;
}

int tga_neighbors(tga_graph* gp, int32_t v, int32_t* dst, int64_t* ts, int32_t cap, int32_t* count) {
  TGA_TRACE("tga_neighbors");
  if (!gp || !count) return fail(TGA_E_ARG, "null argument");
  GraphHandle& h = *gp;
  if (v < 0 || v >= h.view.n) return fail(TGA_E_ARG, "vertex out of range");
  if (cap < 0) cap = 0;
  TGA_TRY(h.s_c.ensure((size_t)cap * 4 + 64));
  TGA_TRY(h.s_d.ensure((size_t)cap * 8 + 64));
  TGA_TRY(h.s_cnt.ensure(64));
  TGA_TRY(h.begin_call());
  ++h.timing.launches;
  k_neighbors<<<1, 1, 0, h.stream>>>(h.view, v, h.s_c.as<int32_t>(), h.s_d.as<int64_t>(), cap, h.s_cnt.as<int32_t>());
  cudaMemcpyAsync(&h.h_pinned[16], h.s_cnt.p, 4, cudaMemcpyDeviceToHost, h.stream);
  TGA_TRY(h.end_call());
  *count = (int32_t)h.h_pinned[16];
  const int32_t k = std::min(cap, *count);
  if (k > 0) {
    if (dst) TGA_CUDA_TRY(cudaMemcpy(dst, h.s_c.p, (size_t)k * 4, cudaMemcpyDeviceToHost));
    if (ts) TGA_CUDA_TRY(cudaMemcpy(ts, h.s_d.p, (size_t)k * 8, cudaMemcpyDeviceToHost));
  }
  return TGA_OK;
}

int tga_is_neighbor(tga_graph* gp, int32_t nq, const int32_t* node, const int32_t* neighbor, const int64_t* t_from,
                    const int64_t* t_to, uint8_t* out) {
  TGA_TRACE("tga_is_neighbor");
  if (!gp || nq < 0 || (nq && (!node || !neighbor || !out))) return fail(TGA_E_ARG, "bad argument");
  GraphHandle& h = *gp;
  if (nq == 0) return TGA_OK;
  std::vector<int64_t> lo((size_t)nq, INT64_MIN), hi((size_t)nq, INT64_MAX);
  if (t_from) std::memcpy(lo.data(), t_from, (size_t)nq * 8);
  if (t_to) std::memcpy(hi.data(), t_to, (size_t)nq * 8);
  TGA_TRY(h.s_c.ensure((size_t)nq * 8));
  TGA_TRY(h.s_d.ensure((size_t)nq * 16));
  TGA_TRY(h.s_e.ensure((size_t)nq));
  TGA_TRY(h.begin_call());
  int32_t* dnode = h.s_c.as<int32_t>();
  int64_t* dlo = h.s_d.as<int64_t>();
  TGA_CUDA_TRY(cudaMemcpyAsync(dnode, node, (size_t)nq * 4, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dnode + nq, neighbor, (size_t)nq * 4, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dlo, lo.data(), (size_t)nq * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dlo + nq, hi.data(), (size_t)nq * 8, cudaMemcpyHostToDevice, h.stream));
  cudaEvent_t* ev = h.kernel_begin();
  KL(k_is_neighbor, grid_for(nq, kBlock))(h.view, nq, dnode, dnode + nq, dlo, dlo + nq, h.s_e.as<uint8_t>());
  h.kernel_end(ev);
  TGA_CUDA_TRY(cudaMemcpyAsync(out, h.s_e.p, (size_t)nq, cudaMemcpyDeviceToHost, h.stream));
  return h.end_call();
}

int tga_decode_all(tga_graph* gp, int64_t* offsets, int32_t* dst, int64_t* ts, int64_t cap) {
  TGA_TRACE("tga_decode_all");
  if (!gp || !offsets) return fail(TGA_E_ARG, "null argument");
  GraphHandle& h = *gp;
  const int32_t n = h.view.n;
  const int32_t nd = (int32_t)h.degrees.size();
  offsets[0] = 0;
  for (int32_t v = 0; v < n; ++v) offsets[v + 1] = offsets[v] + (v < nd ? h.degrees[(size_t)v] : 0);
  const int64_t m = offsets[n];
  if (!dst || !ts) return TGA_OK;  // size query
  if (cap < m) return fail(TGA_E_ARG, "capacity below the number of edges");
  TGA_TRY(h.s_e.ensure((size_t)(n + 1) * 8));
  TGA_TRY(h.s_f.ensure((size_t)std::max<int64_t>(m, 1) * 4));
  TGA_TRY(h.s_g.ensure((size_t)std::max<int64_t>(m, 1) * 8));
  TGA_CUDA_TRY(cudaMemcpy(h.s_e.p, offsets, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice));
  TGA_TRY(h.begin_call());
    KL(k_decode_csr, lean_grid(h))(h.view, lean_work(h), h.s_e.as<int64_t>(), h.s_f.as<int32_t>(),
                                                h.s_g.as<int64_t>(), m);
  cudaMemcpyAsync(dst, h.s_f.p, (size_t)m * 4, cudaMemcpyDeviceToHost, h.stream);
  cudaMemcpyAsync(ts, h.s_g.p, (size_t)m * 8, cudaMemcpyDeviceToHost, h.stream);
  return h.end_call();
}

int tga_pagerank(tga_graph* gp, int32_t iters, float damping, float alpha, int64_t t_lo, int64_t t_hi, float* rank_out) {
  TGA_TRACE("tga_pagerank");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (iters <= 0) iters = h.cfg.pr_iters;
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  const bool windowed = !(t_lo <= 0 && t_hi == TGA_T_MAX);
  const bool all_times = window_covers_all(h, t_lo, t_hi);
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));
  TGA_TRY(h.s_b.ensure((size_t)nv * 4));
  TGA_TRY(h.s_c.ensure((size_t)nv * 4));
  TGA_TRY(h.s_d.ensure((size_t)nv * 4));
  TGA_TRY(h.s_e.ensure((size_t)nv * 4));
  TGA_TRY(h.s_g.ensure((size_t)(iters + 1) * 8));
  TGA_TRY(h.begin_call());
  prepare_runs(h, t_lo, t_hi);
  unsigned long long* edges = edge_counter(h);
  const float base = (1.0f - damping) / (float)h.view.max_label;
  float* bufs[3] = {h.s_a.as<float>(), h.s_b.as<float>(), h.s_c.as<float>()};
  double* sums = h.s_g.as<double>();
  KL(k_fill_f32, grid_for(nv, kBlock))(bufs[0], 1.0f / (float)nv, nv);
  KL(k_fill_f32, grid_for(nv, kBlock))(bufs[1], base, nv);
  KL(k_pr_init_sums, grid_for(iters, kBlock))(sums, iters, (double)base * (double)nv);
  float* invdeg = nullptr;
  if (windowed) {
    int32_t* cnt = h.s_e.as<int32_t>();
    invdeg = h.s_d.as<float>();
    cudaMemsetAsync(cnt, 0, (size_t)nv * 4, h.stream);
        cudaEvent_t* ev = h.kernel_begin();
    KL(k_window_count, lean_grid(h))(h.view, lean_work(h), t_lo, t_hi, cnt, edges);
    h.kernel_end(ev);
    KL(k_invert, grid_for(nv, kBlock))(cnt, invdeg, nv);
  }
  const unsigned grid = sweep_grid(h);
  // The iterations as one CUDA graph, replayed by later calls with the same parameters.
  const std::vector<uint64_t> key = {ptr_key(bufs[0]), ptr_key(bufs[1]), ptr_key(bufs[2]), ptr_key(sums),
                                     ptr_key(invdeg), ptr_key(edges), (uint64_t)iters, (uint64_t)grid, (uint64_t)nv,
                                     bits_of(damping), bits_of(alpha), (uint64_t)t_lo, (uint64_t)t_hi};
  TGA_TRY(run_loop(h, h.pr_loop, key, (size_t)iters, [&]() -> int {
    for (int k = 0; k < iters; ++k) {
      PrArgs a{invdeg, h.d_deg.as<int32_t>(), bufs[k % 3], bufs[(k + 1) % 3], bufs[(k + 2) % 3], sums, k,
               damping, alpha, base, t_lo, t_hi, edges};
      cudaEvent_t* ev = h.kernel_begin();
      if (all_times) KL(k_pr_iter<true>, lean_grid(h))(h.view, lean_work(h), a);
      else KL(k_pr_iter<false>, lean_grid(h))(h.view, lean_work(h), a);
      h.kernel_end(ev);
    }
    return TGA_OK;
  }));
  float* out = bufs[iters % 3];
  float* fin = h.s_d.as<float>();
  KL(k_pr_final, grid_for(nv, kBlock))(out, sums, iters - 1, fin, nv);
  if (rank_out) cudaMemcpyAsync(rank_out, fin, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = iters;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(iters + (windowed ? 1 : 0)) * pass_bytes(h);
  return rc;
}

int tga_hits(tga_graph* gp, int32_t iters, int32_t mode, int64_t t_lo, int64_t t_hi, float* hub_out, float* auth_out) {
  TGA_TRACE("tga_hits");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (iters <= 0) iters = h.cfg.hits_iters;
  if (mode != TGA_HITS_GPU && mode != TGA_HITS_JAVA) return fail(TGA_E_ARG, "unknown HITS mode");
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(h.s_a.ensure((size_t)nv * 8));
  TGA_TRY(h.s_b.ensure((size_t)nv * 8));
  TGA_TRY(h.s_c.ensure((size_t)nv * 8));
  TGA_TRY(h.s_d.ensure((size_t)nv * 8));
  TGA_TRY(h.s_g.ensure((size_t)(2 * iters + 2) * 8));
  TGA_TRY(h.begin_call());
  // With a window that holds every timestamp, HITS depends only on the successor order: the
  // timestamp streams are not decoded.
  const bool all_times = window_covers_all(h, t_lo, t_hi);
  prepare_runs(h, t_lo, t_hi);
  unsigned long long* edges = edge_counter(h);
  double* hub = h.s_a.as<double>();
  double* auth[2] = {h.s_b.as<double>(), h.s_c.as<double>()};
  double* sums = h.s_g.as<double>();
  const int java = mode == TGA_HITS_JAVA;
  KL(k_fill_f64, grid_for(nv, kBlock))(hub, 1.0, nv);
  KL(k_fill_f64, grid_for(nv, kBlock))(auth[0], 1.0, nv);
  cudaMemsetAsync(sums, 0, (size_t)(2 * iters + 2) * 8, h.stream);
  // sums[2k] = sum hub^2 of iteration k, sums[2k+1] = sum auth^2 of iteration k.  The iterations
  // run as one CUDA graph, replayed by later calls with the same parameters.
  const std::vector<uint64_t> key = {ptr_key(hub), ptr_key(auth[0]), ptr_key(auth[1]), ptr_key(sums), ptr_key(edges),
                                     (uint64_t)iters, (uint64_t)java, (uint64_t)all_times, (uint64_t)nv,
                                     (uint64_t)t_lo, (uint64_t)t_hi};
  TGA_TRY(run_loop(h, h.hits_loop, key, (size_t)(2 * iters), [&]() -> int {
    for (int k = 0; k < iters; ++k) {
      const double* aprev = k == 0 ? nullptr : sums + 2 * k - 1;
      double* ain = auth[k & 1];
      double* anext = auth[(k + 1) & 1];
      KL(k_hits_base, grid_for(nv, kBlock))(hub, ain, anext, aprev, java, nv);
      cudaEvent_t* ev = h.kernel_begin();
      // (without decoded timestamps every edge reports t = 0, so the window check is opened fully)
      if (all_times) KL(k_hits_hub<false>, lean_grid(h))(h.view, lean_work(h), hub, ain, aprev, INT64_MIN, INT64_MAX, edges);
      else KL(k_hits_hub<true>, lean_grid(h))(h.view, lean_work(h), hub, ain, aprev, t_lo, t_hi, edges);
      h.kernel_end(ev);
      KL(k_sumsq, grid_for(nv, kBlock))(hub, nv, sums + 2 * k);
      ev = h.kernel_begin();
      if (all_times)
        KL(k_hits_auth<false>, lean_grid(h))(h.view, lean_work(h), hub, sums + 2 * k, anext, INT64_MIN, INT64_MAX, edges);
      else KL(k_hits_auth<true>, lean_grid(h))(h.view, lean_work(h), hub, sums + 2 * k, anext, t_lo, t_hi, edges);
      h.kernel_end(ev);
      KL(k_scale<double>, grid_for(nv, kBlock))(hub, sums + 2 * k, hub, nv);
      KL(k_sumsq, grid_for(nv, kBlock))(anext, nv, sums + 2 * k + 1);
    }
    return TGA_OK;
  }));
  // FP32 results: the hub as it stands (normalised), the authorities scaled by their last norm.
  float* hub32 = reinterpret_cast<float*>(auth[(iters + 1) & 1]);
  float* auth32 = h.s_d.as<float>();
  KL(k_to_f32, grid_for(nv, kBlock))(hub, hub32, nv);
  KL(k_scale<float>, grid_for(nv, kBlock))(auth[iters & 1], sums + 2 * iters - 1, auth32, nv);
  if (hub_out) cudaMemcpyAsync(hub_out, hub32, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (auth_out) cudaMemcpyAsync(auth_out, auth32, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = iters;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(2 * iters) * pass_bytes(h);
  return rc;
}

int tga_degree(tga_graph* gp, int64_t t_start, int64_t t_end, int32_t* degree_out, int64_t* avg_out) {
  TGA_TRACE("tga_degree");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));
  TGA_TRY(h.s_b.ensure((size_t)nv * 8));
  if (h.nlong > 0) {
    TGA_TRY(h.s_edges.ensure((size_t)h.long_edges * 8));  // per-edge timestamps (or skips) of the sliced lists
    TGA_TRY(h.s_f.ensure((size_t)h.long_edges * 8));      // their counted timestamps, compacted per list
    TGA_TRY(h.s_c.ensure((size_t)h.nlong * 4));           // counted per list
    TGA_TRY(h.s_d.ensure((size_t)h.nslices * 4));         // counted per slice
    TGA_TRY(h.s_e.ensure((size_t)h.nslices * 8));         // compacted base per slice
  }
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  cudaMemsetAsync(h.s_a.p, 0, (size_t)nv * 4, h.stream);
  cudaMemsetAsync(h.s_b.p, 0, (size_t)nv * 8, h.stream);
  cudaEvent_t* ev = h.kernel_begin();
  KL(k_degree, lean_grid(h))(h.view, lean_work(h), t_start, t_end, h.s_a.as<int32_t>(), h.s_b.as<int64_t>(), edges);
  h.kernel_end(ev);
  if (h.nlong > 0) {
    cudaEvent_t* ev2 = h.kernel_begin();
    KL(k_degree_slices, grid_for(h.nslices, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_slice_ebase.as<int64_t>(),
                                                     (int32_t)h.nslices, t_start, t_end, h.s_edges.as<int64_t>(),
                                                     h.s_d.as<int32_t>(), edges);
    h.kernel_end(ev2);
    // Narrow form when the graph's whole timestamp span fits 31 bits (max_ts found at load).
    const bool narrow = h.max_ts != INT64_MAX && h.min_ts_data >= 0 && h.max_ts - h.min_ts_data < INT32_MAX;
    int32_t* cnt = h.s_c.as<int32_t>();
    KL(k_degree_bases, grid_for((int64_t)h.nlong * 32, kBlock))(h.d_long.as<LongList>(), h.nlong,
                                                                h.d_slice_first.as<int32_t>(), h.s_d.as<int32_t>(),
                                                                h.view.active_begin, h.view.max_label,
                                                                h.s_e.as<int64_t>(), cnt);
    KL(k_degree_gather, grid_for(h.nslices, kBlock))(h.d_slices.as<SliceState>(), (int32_t)h.nslices,
                                                     h.d_slice_ebase.as<int64_t>(), h.s_e.as<int64_t>(),
                                                     h.s_d.as<int32_t>(), h.s_edges.as<int64_t>(), h.s_f.as<int64_t>());
    auto long_kernel = narrow ? k_degree_long<true> : k_degree_long<false>;
    KL(long_kernel, grid_for(h.nlong, kBlock))(h.d_long.as<LongList>(), h.nlong, cnt,
                                               h.s_f.as<int64_t>(), h.d_divtab.as<uint2>(), h.min_ts_data,
                                               h.view.active_begin, h.view.max_label, t_start, t_end,
                                               h.s_a.as<int32_t>(), h.s_b.as<int64_t>());
  }
  KL(k_degree_empty, grid_for(nv, kBlock))(h.d_deg.as<int32_t>(), h.view.active_begin, h.view.max_label,
                                           std::min(nv, h.view.n), t_start, t_end, h.s_a.as<int32_t>());
  if (degree_out) cudaMemcpyAsync(degree_out, h.s_a.p, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (avg_out) cudaMemcpyAsync(avg_out, h.s_b.p, (size_t)nv * 8, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = 1;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = pass_bytes(h);
  return rc;
}

// java.util.Random(seed).nextInt(bound) for a power-of-two bound (the JDK's documented LCG).
static void java_random_prio(uint32_t* out, int32_t n, int64_t seed) {
  uint64_t s = ((uint64_t)seed ^ 0x5DEECE66Dull) & ((1ull << 48) - 1);
  for (int32_t i = 0; i < n; ++i) {
    s = (s * 0x5DEECE66Dull + 0xBull) & ((1ull << 48) - 1);
    const int32_t bits = (int32_t)(s >> (48 - 31));
    out[i] = (uint32_t)(((int64_t)256 * (int64_t)bits) >> 31);
  }
}

int tga_color(tga_graph* gp, int32_t prio_mode, const uint32_t* prio_in, int32_t flags, uint32_t* color_out,
              uint32_t* prio_out, int32_t* rounds_out) {
  TGA_TRACE("tga_color");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  if (prio_mode == 2 && !prio_in) return fail(TGA_E_ARG, "priorities required for mode 2");
  if (prio_mode < 0 || prio_mode > 2) return fail(TGA_E_ARG, "unknown priority mode");
  const size_t qcap = (size_t)nv + (size_t)h.nslices + 1;
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));  // colours
  TGA_TRY(h.s_b.ensure((size_t)nv * 4));  // priorities
  TGA_TRY(h.s_c.ensure((size_t)nv * 4));  // found stamps
  TGA_TRY(h.s_q0.ensure((size_t)nv * 4));
  TGA_TRY(h.s_q1.ensure((size_t)nv * 4));
  TGA_TRY(h.s_d.ensure(qcap * 4));
  TGA_TRY(h.s_e.ensure(qcap * 4));
  TGA_TRY(h.s_cnt.ensure(64));
  TGA_TRY(h.s_f.ensure(((size_t)nv + (size_t)h.nslices) * sizeof(GcPoint)));  // resume points
  std::vector<uint32_t> host_prio;
  if (prio_mode == 1) {
    host_prio.resize((size_t)nv);
    java_random_prio(host_prio.data(), nv, 123);
    prio_in = host_prio.data();
  }
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  uint32_t* color = h.s_a.as<uint32_t>();
  uint32_t* prio = h.s_b.as<uint32_t>();
  uint32_t* found = h.s_c.as<uint32_t>();
  const Work w = work_of(h);
  if (prio_mode == 0) KL(k_gc_prio_curand, grid_for(((int64_t)nv + kPrioRun - 1) / kPrioRun, kBlock))(prio, nv);
  else cudaMemcpyAsync(prio, prio_in, (size_t)nv * 4, cudaMemcpyHostToDevice, h.stream);
  cudaMemsetAsync(color, 0xFF, (size_t)nv * 4, h.stream);
  cudaMemsetAsync(found, 0, (size_t)nv * 4, h.stream);
  int32_t* cnt = h.s_cnt.as<int32_t>();  // [0] worklist, [1] entries
  cudaMemsetAsync(cnt, 0, 8, h.stream);
  KL(k_gc_first, grid_for(nv, kBlock))(h.view, w, h.d_deg.as<int32_t>(), nv, h.s_q0.as<int32_t>(),
                                       h.s_d.as<int32_t>(), cnt + 1);
  DevBuf *wl = &h.s_q0, *nwl = &h.s_q1, *en = &h.s_d, *nen = &h.s_e;
  int32_t wn = nv, ne = 0;
  cudaMemcpyAsync(&h.h_pinned[24], cnt + 1, 4, cudaMemcpyDeviceToHost, h.stream);
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  ne = (int32_t)h.h_pinned[24];
  int round = 0;
  GcPoint* pts = h.s_f.as<GcPoint>();
  while (wn != 0 && round < 512) {
    cudaMemsetAsync(cnt, 0, 8, h.stream);
    if (ne > 0) {
      cudaEvent_t* ev = h.kernel_begin();
      KL(k_gc_check, grid_for(ne, kBlock))(h.view, en->as<int32_t>(), ne, nv, color, prio, (uint32_t)round, found, pts,
                                           nen->as<int32_t>(), cnt + 1, edges);
      h.kernel_end(ev);
    }
    KL(k_gc_decide, grid_for(wn, kBlock))(h.view, wl->as<int32_t>(), wn, h.d_deg.as<int32_t>(), color, found,
                                          (uint32_t)round, flags & TGA_GC_JAVA_ISOLATED, nwl->as<int32_t>(), cnt);
    cudaMemcpyAsync(&h.h_pinned[24], cnt, 8, cudaMemcpyDeviceToHost, h.stream);
    TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
    wn = (int32_t)h.h_pinned[24];
    ne = (int32_t)h.h_pinned[25];
    std::swap(wl, nwl);
    std::swap(en, nen);
    ++round;
  }
  if (color_out) cudaMemcpyAsync(color_out, color, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (prio_out) cudaMemcpyAsync(prio_out, prio, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (rounds_out) *rounds_out = round;
  h.timing.iterations = round;
  return finish(h, edges);
}

// tga_pagerank without any device allocation: the same kernels in the same order, with the
// handle's growable scratch replaced by the fixed per-device array of noalloc.cu and the result
// written to a caller-owned device buffer.  Only the call's total time is recorded (no per-kernel
// timers).  The scratch is shared by every handle on a device, so overlapping calls race.
int tga_pagerank_noalloc(tga_graph* gp, int32_t iters, float damping, float alpha, int64_t t_lo, int64_t t_hi,
                         float* rank_out_dev) {
  TGA_TRACE("tga_pagerank_noalloc");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (iters <= 0) iters = h.cfg.pr_iters;
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  if (!rank_out_dev) return fail(TGA_E_ARG, "null rank_out_dev");
  const int32_t nv = h.view.max_vertex;
  if (nv > kPrNoAllocMaxVertices)
    return fail(TGA_E_ARG, "tga_pagerank_noalloc: max_vertex " + std::to_string(nv) + " exceeds its fixed scratch of " +
                               std::to_string(kPrNoAllocMaxVertices) + " vertices; use tga_pagerank");
  if (iters > kPrNoAllocMaxIters)
    return fail(TGA_E_ARG, "tga_pagerank_noalloc: " + std::to_string(iters) + " iterations exceed its fixed scratch of " +
                               std::to_string(kPrNoAllocMaxIters) + "; use tga_pagerank");
  cudaPointerAttributes pa{};
  TGA_CUDA_TRY(cudaPointerGetAttributes(&pa, rank_out_dev));
  // Plain device memory only: for managed memory pa.device names the allocating device, not where
  // the pages are.
  if (pa.type != cudaMemoryTypeDevice || pa.device != h.device)
    return fail(TGA_E_ARG, "tga_pagerank_noalloc: rank_out_dev must be device memory of the graph's device");
  unsigned char* s = nullptr;
  TGA_TRY(pr_noalloc_scratch(h.device, &s));
  float* bufs[3] = {reinterpret_cast<float*>(s), reinterpret_cast<float*>(s + kPrNoAllocVec),
                    reinterpret_cast<float*>(s + 2 * kPrNoAllocVec)};
  float* invdeg_buf = reinterpret_cast<float*>(s + 3 * kPrNoAllocVec);
  int32_t* cnt = reinterpret_cast<int32_t*>(s + 4 * kPrNoAllocVec);
  double* sums = reinterpret_cast<double*>(s + kPrNoAllocSumsOff);
  unsigned long long* edges = reinterpret_cast<unsigned long long*>(s + kPrNoAllocCountersOff);
  int32_t* next = reinterpret_cast<int32_t*>(s + kPrNoAllocCountersOff + 8);

  h.timing = tga_timing{};
  h.ktimer_used = 0;
  TGA_CUDA_TRY(cudaMemsetAsync(h.d_err.p, 0, sizeof(uint32_t), h.stream));
  TGA_CUDA_TRY(cudaEventRecord(h.ev_begin, h.stream));
  // Edge counter and work counter start at zero.
  TGA_CUDA_TRY(cudaMemsetAsync(s + kPrNoAllocCountersOff, 0, 256, h.stream));
  const Work w{h.d_items.as<WorkItem>(), h.d_slices.as<SliceState>(), h.d_slice_first.as<int32_t>(), next, h.nitems,
               h.d_order.as<int32_t>(), h.norder, h.d_run_first.as<int32_t>()};
  prepare_runs(h, t_lo, t_hi);  // fills the handle's run table (allocated at open)
  const bool windowed = !(t_lo <= 0 && t_hi == TGA_T_MAX);
  const bool all_times = window_covers_all(h, t_lo, t_hi);
  const float base = (1.0f - damping) / (float)h.view.max_label;
  KL(k_fill_f32, grid_for(nv, kBlock))(bufs[0], 1.0f / (float)nv, nv);
  KL(k_fill_f32, grid_for(nv, kBlock))(bufs[1], base, nv);
  KL(k_pr_init_sums, grid_for(iters, kBlock))(sums, iters, (double)base * (double)nv);
  float* invdeg = nullptr;
  if (windowed) {
    invdeg = invdeg_buf;
    // The in-window outdegrees are accumulated with atomics and start at zero.
    TGA_CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)nv * 4, h.stream));
    KL(k_window_count, lean_grid(h))(h.view, lean_work(h), t_lo, t_hi, cnt, edges);
    KL(k_invert, grid_for(nv, kBlock))(cnt, invdeg, nv);
  }
  const unsigned grid = sweep_grid(h);
  for (int k = 0; k < iters; ++k) {
    PrArgs a{invdeg, h.d_deg.as<int32_t>(), bufs[k % 3], bufs[(k + 1) % 3], bufs[(k + 2) % 3], sums, k,
             damping, alpha, base, t_lo, t_hi, edges};
    if (all_times) KL(k_pr_iter<true>, lean_grid(h))(h.view, lean_work(h), a);
    else KL(k_pr_iter<false>, lean_grid(h))(h.view, lean_work(h), a);
  }
  KL(k_pr_final, grid_for(nv, kBlock))(bufs[iters % 3], sums, iters - 1, rank_out_dev, nv);
  h.timing.iterations = iters;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(iters + (windowed ? 1 : 0)) * pass_bytes(h);
  return rc;
}

}  // extern "C"
