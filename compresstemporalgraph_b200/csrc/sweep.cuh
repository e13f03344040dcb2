// Shared pieces of the fused decode kernels: the launch macro, work views, queue handling and
// the two sweep drivers (class-ordered schedule and frontier queues), plus the host-side helpers
// that every entry point uses.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.hpp"
#include "leancursor.cuh"

namespace tga {

constexpr int kBlock = 256;
constexpr uint64_t kTpInf = ~0ull;
constexpr uint32_t kColorInf = 0xFFFFFFFFu;
constexpr int kNoRunFilter = -2;

// Launches a kernel of kBlock threads on the handle's stream and counts it in the call's timing.
#define KL(kernel, grid) ++h.timing.launches, kernel<<<(grid), kBlock, 0, h.stream>>>
// Decode kernels of colouring, batched BFS, point queries, batched PageRank and the run
// pre-passes: 2 blocks of 256 threads per SM (up to 128 registers).
#define TGA_DECODE_BOUNDS __launch_bounds__(kBlock, 2)
// BFS, CC (single and batched seeds) and degree centrality: 3 blocks per SM (up to 85 registers);
// measured against 2 on the 2M/40M graph: BFS 16.4 / 17.2 ms, CC 67.0 / 68.1 ms, DC 17.3 / 17.7 ms.
// Colouring (22.9 / 22.1 ms) and the 256-source batched BFS (17.0 / 15.5 ms) were slower at 3.
#define TGA_TRAVERSE_BOUNDS __launch_bounds__(kBlock, 3)
// Full sweeps over the schedule (neighbour access, PageRank, HITS, window counts, raw decode):
// 4 blocks per SM (up to 64 registers, a few spills), measured faster than 2 on these kernels
// because more resident warps hide the decoder's dependent loads.
#define TGA_SWEEP_BOUNDS __launch_bounds__(kBlock, 4)

// Per-edge term of the neighbour-access checksum: the checksum of a list is the sum (mod 2^64)
// of edge_hash over its edges, so slices can add their parts; the edge index keeps it
// order-sensitive.  The oracle computes the same sum.
__host__ __device__ __forceinline__ uint64_t edge_hash(uint32_t v, uint32_t i, int32_t y, int64_t t) {
  uint64_t z = (((uint64_t)v << 32) | i) * 0x9E3779B97F4A7C15ull;
  z ^= (uint64_t)(uint32_t)y * 0xC2B2AE3D27D4EB4Full;
  z ^= (uint64_t)t * 0x165667B19E3779F9ull;
  z ^= z >> 31;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 29;
  z *= 0x94D049BB133111EBull;
  return z ^ (z >> 32);
}

__device__ __forceinline__ void add_edges(unsigned long long* ctr, unsigned long long mine) {
  for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(ctr, mine);
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kBlock / 32];
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

// Edge count summed over the block and added once per block (every thread of the block must call
// it): a sweep of 12,653 blocks would otherwise send 101K atomics to one L2 slice.  The count
// passes through a double, exact below 2^53.
__device__ __forceinline__ void block_add_edges(unsigned long long* ctr, unsigned long long mine) {
  const double s = block_sum((double)mine);
  if (threadIdx.x == 0 && s != 0.0) atomicAdd(ctr, (unsigned long long)s);
  __syncthreads();  // (the shared partials are free again)
}

// Sum of v over the warp, added to *out by lane 0 (no block barrier: warps leave independently).
__device__ __forceinline__ void warp_add(double* out, double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out, v);
}

struct Work {
  const WorkItem* items;
  const SliceState* slices;
  const int32_t* slice_first;
  int32_t* next;          // work counter of the launch (zeroed before it)
  int32_t nitems;
  const int32_t* order;   // sweep schedule grouped by work class (vertex ids and -(slice+1))
  int32_t norder;
  // per run of equal successors cut by slices: list index of its first in-window edge for the
  // call's window (INT32_MAX: none); read by the drivers with kRuns
  const int32_t* run_first;
};

// Opens queue entry e: a whole list (e >= 0) or one slice.  Returns the vertex; `lead` is the
// leading-run filter of the entry (see RunFilter).
__device__ __forceinline__ int open_entry(const GraphView& g, const Work& w, int e, LeanCursor& c, int& first,
                                          int& count, int& lead, int& run) {
  lead = kNoRunFilter;
  run = -1;
  if (e >= 0) {
    first = 0;
    count = c.open_vertex(g, e);
    return e;
  }
  const SliceState& s = w.slices[-e - 1];
  c.restore(g, s);
  first = s.first;
  count = s.count;
  if (s.run >= 0 && w.run_first) lead = __ldg(w.run_first + s.run);
  run = s.run;
  return s.v;
}

// Dedup of a slice that starts inside a run of equal successors: while the slice's edges continue
// that run, only the run's first in-window edge (list index `lead`, computed for the call's
// window) reaches the algorithm; afterwards every edge does.  Algorithms that keep only the first
// in-window occurrence of equal consecutive successors (keep_edge) run their sweeps with it.
struct RunFilter {
  int lead;   // list index to pass, or kNoRunFilter once past the leading run
  int y_run;  // successor of the leading run (-1 before the first edge)
  int idx;    // list index of the next edge
  __device__ __forceinline__ void start(int lead_idx, int first) {
    lead = lead_idx;
    y_run = -1;
    idx = first;
  }
  // true if edge (y) passes the filter
  __device__ __forceinline__ bool pass(int y) {
    const int i = idx++;
    if (lead == kNoRunFilter) return true;
    if (y_run < 0) y_run = y;
    if (y == y_run) return i == lead;
    lead = kNoRunFilter;
    return true;
  }
};

// Appends y (or all slices of y) to a queue.
__device__ __forceinline__ void enqueue(const Work& w, int y, int32_t* q, int32_t* cnt) {
  const int a = w.slice_first[y], b = w.slice_first[y + 1];
  if (a == b) {
    q[atomicAdd(cnt, 1)] = y;
  } else {
    const int base = atomicAdd(cnt, b - a);
    for (int j = a; j < b; ++j) q[base + j - a] = -(j + 1);
  }
}

// Edge filter shared by every traversal: in-window, first of equal consecutive successors,
// successor inside [active_begin, max_vertex).
__device__ __forceinline__ bool keep_edge(const GraphView& g, int64_t lo, int64_t hi, int y, int64_t t, int& prev_y) {
  if (t < lo || t >= hi) return false;
  if (y == prev_y) return false;
  prev_y = y;
  return y >= g.active_begin && y < g.max_vertex;
}
// The same for a window that holds every timestamp of the graph (no time test).
__device__ __forceinline__ bool keep_edge_all(const GraphView& g, int y, int& prev_y) {
  if (y == prev_y) return false;
  prev_y = y;
  return y >= g.active_begin && y < g.max_vertex;
}

// Rank of the calling warp when warps are dealt round-robin over the blocks (warp k of block b has
// rank k * gridDim.x + b): consecutive 32-entry chunks then go to different blocks, so a run of
// entries of one long list is spread over the SMs instead of filling the first blocks.
__device__ __forceinline__ int spread_warp_rank() {
  return (int)((threadIdx.x >> 5) * gridDim.x + blockIdx.x);
}

// Sweep over the class-ordered schedule: thread i decodes entry i (a whole list or a slice).
// Entries of one warp belong to the same work class, so the lanes open their lists together and
// finish together.  Hooks (each inlined at its single call site): want(x) -> bool,
// begin(x, first, count) -> bool (false: skip the list), edge(x, y, t) -> bool (false: stop the
// list), end(x).  kWhole: a sliced list is decoded whole by the thread that draws its first slice
// (for workloads that are sequential per list); its other slices are skipped.
// kSpread: chunks of 32 entries are dealt by spread_warp_rank() (for persistent grids, where the
// blocks holding the first entries would otherwise get all the slices of the first long lists).
// kRuns: slices that start inside a run of equal successors pass their edges through RunFilter.
// kTimes = false: timestamps are not decoded (edge() sees t = 0).
// kRunArg: begin() takes a fourth argument, the index of the run of equal successors that a slice
// starts inside (-1 for whole lists and slices that start at a new successor).
template <bool kWhole, bool kSpread = false, bool kRuns = false, bool kTimes = true, bool kRunArg = false, class Want,
          class Begin, class Edge, class End>
__device__ __forceinline__ unsigned long long run_order(const GraphView& g, const Work& w, Want want, Begin begin,
                                                        Edge edge, End end) {
  unsigned long long edges = 0;
  const int start = kSpread ? spread_warp_rank() * 32 + (int)(threadIdx.x & 31) : (int)(blockIdx.x * blockDim.x + threadIdx.x);
  for (int i = start; i < w.norder; i += gridDim.x * blockDim.x) {
    const int e = w.order[i];
    LeanCursor c;
    RunFilter rf;
    int x, first = 0, count, lead = kNoRunFilter, run = -1;
    if (e >= 0) {
      x = e;
      if (!want(x)) continue;
      count = c.open_vertex(g, x);
    } else {
      const SliceState& s = w.slices[-e - 1];
      x = s.v;
      if (!want(x)) continue;
      if (kWhole) {
        if (s.first != 0) continue;
        count = c.open_vertex(g, x);
      } else {
        c.restore(g, s);
        first = s.first;
        count = s.count;
        if (kRuns && s.run >= 0) lead = __ldg(w.run_first + s.run);
        run = s.run;
      }
    }
    bool go;
    if constexpr (kRunArg) go = count > 0 && begin(x, first, count, run);
    else go = count > 0 && begin(x, first, count);
    if (!go) continue;
    if (kRuns) rf.start(lead, first);
    int y;
    int64_t t;
    while (c.template next<kTimes>(g, y, t)) {
      ++edges;
      if (kRuns && !rf.pass(y)) continue;
      if (!edge(x, y, t)) break;
    }
    end(x);
  }
  return edges;
}

// Flat loop over the entries q[0..qn) of a queue (vertices or slices); q may have been written
// earlier in the same launch by other blocks (it is read through L2).  kRuns, kTimes, kRunArg as
// in run_order.
// Next index of a shared work counter for the calling lane: the lanes of the warp that ask at the
// same time take consecutive indexes with one atomic.  (One atomic per entry sends every request
// of the level to one L2 slice: on the 2M/40M graph's CC, levels of 1.4M entries spent most of
// their time queued there.)
__device__ __forceinline__ int take_next(int32_t* counter) {
  const unsigned act = __activemask();
  const int lane = (int)(threadIdx.x & 31);
  const int leader = __ffs(act) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(act));
  base = __shfl_sync(act, base, leader);
  return base + __popc(act & ((1u << lane) - 1u));
}

template <bool kRuns = false, bool kTimes = true, bool kRunArg = false, class Begin, class Edge, class End>
__device__ __forceinline__ unsigned long long drive_queue(const GraphView& g, const Work& w, const int32_t* q, int qn,
                                                          Begin begin, Edge edge, End end) {
  LeanCursor c;
  RunFilter rf;
  rf.start(kNoRunFilter, 0);
  c.remaining = 0;
  int cur = -1;
  unsigned long long edges = 0;
  // The first entry of a thread comes from its spread warp rank (consecutive entries, such as the
  // slices of one list, land on different SMs); later ones come from the counter, offset by the
  // thread count, so a queue shorter than the grid costs no atomics at all.  A short queue is
  // dealt to m lanes per warp, m the smallest power of two that covers it: lanes decoding
  // different lists diverge, so fewer lanes per warp finish a small level sooner.
  const int nthreads = (int)(gridDim.x * blockDim.x), lane = (int)(threadIdx.x & 31);
  int m = 32;
  if (qn < nthreads) {
    m = 1;
    while (m < 32 && m * (nthreads >> 5) < qn) m <<= 1;
  }
  int i = lane < m ? spread_warp_rank() * m + lane : qn;
  for (;;) {
    if (c.remaining <= 0) {
      if (cur >= 0) {
        end(cur);
        cur = -1;
      }
      if (i < 0) i = nthreads + take_next(w.next);
      if (i >= qn) break;
      int first, count, lead, run;
      const int x = open_entry(g, w, __ldcg(q + i), c, first, count, lead, run);
      i = -1;
      bool go;
      if constexpr (kRunArg) go = count > 0 && begin(x, first, count, run);
      else go = count > 0 && begin(x, first, count);
      if (!go) {
        c.remaining = 0;
        continue;
      }
      if (kRuns) rf.start(lead, first);
      cur = x;
      continue;
    }
    int y;
    int64_t t;
    if (!c.template next<kTimes>(g, y, t)) continue;
    ++edges;
    if (kRuns && !rf.pass(y)) continue;
    if (!edge(cur, y, t)) c.remaining = 0;
  }
  return edges;
}

// ---------------------------------------------------------------------------------------------
// Fills

static __global__ void k_fill_u64(uint64_t* p, uint64_t v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
// Per-call pre-pass for the runs of equal successors that slices cut: one thread per (run, slice
// overlapping it) decodes the slice from its checkpoint and lowers run_first[run] to the list
// index of the first in-window edge of the run within that slice.
static __global__ void TGA_DECODE_BOUNDS k_run_first(GraphView g, const SliceState* slices, const RunInfo* runs,
                                                     const int2* pairs, int32_t npairs, int64_t lo, int64_t hi,
                                                     int32_t* run_first) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const int2 pr = pairs[p];
  const RunInfo r = runs[pr.x];
  const SliceState& s = slices[pr.y];
  LeanCursor c;
  c.restore(g, s);
  int idx = s.first, y_run = -1, y;
  int64_t t;
  while (c.next(g, y, t)) {
    const int i = idx++;
    if (i < r.start) continue;
    if (y_run < 0) y_run = y;
    else if (y != y_run) break;
    if (t >= lo && t < hi) {
      atomicMin(&run_first[pr.x], i);
      break;
    }
  }
}

static __global__ void k_fill_f32(float* p, float v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
static __global__ void k_fill_f64(double* p, double v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
static __global__ void k_to_f32(const double* in, float* out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}
static __global__ void k_fill_i32(int32_t* p, int32_t v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}


static int32_t seed_entries(const GraphHandle& h, int32_t v, std::vector<int32_t>& out) {
  out.clear();
  const int32_t a = h.slice_first_host[(size_t)v], b = h.slice_first_host[(size_t)v + 1];
  if (a == b) out.push_back(v);
  else
    for (int32_t j = a; j < b; ++j) out.push_back(-(j + 1));
  return (int32_t)out.size();
}

// Work view of a handle with a freshly zeroed counter (one per decode launch, in stream order).
static Work work_of(GraphHandle& h) {
  int32_t* ctr = reinterpret_cast<int32_t*>(h.s_sum.as<char>() + 4000);
  cudaMemsetAsync(ctr, 0, sizeof(int32_t), h.stream);
  return Work{h.d_items.as<WorkItem>(), h.d_slices.as<SliceState>(), h.d_slice_first.as<int32_t>(), ctr, h.nitems,
              h.d_order.as<int32_t>(), h.norder, h.d_run_first.as<int32_t>()};
}

// Computes the handle's run_first table for the window [lo, hi) (one small kernel over the slices
// that overlap a cut run; nothing when no run is cut).
static void prepare_runs(GraphHandle& h, int64_t lo, int64_t hi) {
  if (h.nruns == 0) return;
  int32_t* rf = h.d_run_first.as<int32_t>();
  KL(k_fill_i32, grid_for(h.nruns, kBlock))(rf, INT32_MAX, h.nruns);
  KL(k_run_first, grid_for(h.nrun_pairs, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_runs.as<RunInfo>(),
                                                  h.d_run_pairs.as<int2>(), h.nrun_pairs, lo, hi, rf);
}

// Grid of a persistent decode launch over `work` units.
static unsigned decode_grid(const GraphHandle& h, int64_t work) {
  const int64_t cap = (int64_t)h.sm_count * 2;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cap, (work + kBlock - 1) / kBlock));
}

// Grid of a sweep over the schedule: one entry per thread.
static unsigned sweep_grid(const GraphHandle& h) { return std::max(1u, grid_for(h.norder, kBlock)); }

// Runs body (which enqueues an iteration loop on h.stream and returns a status) through a CUDA
// graph: captured and instantiated the first time `key` is seen, replayed while it stays the
// same.  The key must hold every pointer and value baked into the loop's launches; the handle's
// decomposition generation, the view and the index of the first kernel timer are added here.
// timers: kernel timer pairs the loop records (created before the capture starts).
template <class Body>
static int run_loop(GraphHandle& h, LoopGraph& lg, std::vector<uint64_t> key, size_t timers, Body body) {
  key.push_back(h.work_gen);
  key.push_back((uint64_t)(uintptr_t)h.view.self);
  key.push_back((uint64_t)h.ktimer_used);
  key.push_back(h.time_kernels ? 1u : 0u);
  if (lg.exec && lg.key == key && h.ktimer_used + lg.timers <= h.ktimers.size()) {
    h.ktimer_used += lg.timers;
    h.timing.launches += lg.launches;
    h.timing.decode_launches += lg.decodes;
    TGA_CUDA_TRY(cudaGraphLaunch(lg.exec, h.stream));
    return TGA_OK;
  }
  if (lg.exec) {
    cudaGraphExecDestroy(lg.exec);
    lg.exec = nullptr;
  }
  const size_t t0 = h.ktimer_used;
  const int64_t l0 = h.timing.launches, d0 = h.timing.decode_launches;
  if (h.time_kernels) TGA_TRY(h.reserve_timers(timers));
  TGA_CUDA_TRY(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
  h.capturing = true;
  const int brc = body();
  h.capturing = false;
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(h.stream, &graph);
  if (brc || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return brc ? brc : fail(TGA_E_CUDA, std::string("loop capture failed: ") + cudaGetErrorString(ec));
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    return fail(TGA_E_CUDA, std::string("loop graph instantiation failed: ") + cudaGetErrorString(ei));
  }
  lg.exec = exec;
  lg.key = std::move(key);
  lg.timers = h.ktimer_used - t0;
  lg.launches = h.timing.launches - l0;
  lg.decodes = h.timing.decode_launches - d0;
  TGA_CUDA_TRY(cudaGraphLaunch(exec, h.stream));
  return TGA_OK;
}

static inline uint64_t bits_of(double x) {
  uint64_t b;
  std::memcpy(&b, &x, 8);
  return b;
}
static inline uint64_t ptr_key(const void* p) { return (uint64_t)(uintptr_t)p; }

static int finish(GraphHandle& h, unsigned long long* edges_dev) {
  if (edges_dev) {
    unsigned long long e = 0;
    cudaMemcpyAsync(&h.h_pinned[8], edges_dev, sizeof e, cudaMemcpyDeviceToHost, h.stream);
    const int rc = h.end_call();
    std::memcpy(&e, &h.h_pinned[8], sizeof e);
    h.timing.edges_decoded = (int64_t)e;
    return rc;
  }
  return h.end_call();
}

static unsigned long long* edge_counter(GraphHandle& h) {
  if (h.s_sum.ensure(4096)) return nullptr;
  unsigned long long* p = reinterpret_cast<unsigned long long*>(h.s_sum.as<char>() + 4032);
  cudaMemsetAsync(p, 0, sizeof(unsigned long long), h.stream);
  return p;
}

static uint64_t pass_bytes(const GraphHandle& h) {
  return h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes;
}

}  // namespace tga
