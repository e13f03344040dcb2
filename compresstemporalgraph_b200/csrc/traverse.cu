// Temporal BFS and connected components (per-seed temporal reach), each as ONE cooperative
// launch that runs every frontier level on the device.
//
// A level decodes the lists of its frontier.  A short frontier is a queue of entries (vertex ids
// and -(slice + 1)) that lanes pull one at a time; a frontier of at least `dense_min` entries is
// processed by the class-ordered sweep over all lists with "in the frontier" as the filter, so
// warps decode lists of similar length together.  Levels are separated by a grid barrier whose
// wait is bounded in time: a wait that runs out marks the launch failed and every block returns
// at its next barrier (the host then reports TGA_E_TIMEOUT).  The reference runs one kernel per
// level with a host round trip each (shared/bfs.cu:1999-2038, connected_components.cu:2091-2149).
//
// Relaxations never wait on an atomic: an edge issues a reduction (RED.MIN on the arrival, or the
// hop level) and sets the successor's bit in a dirty bitmap, both without a return value, so the
// decode of the next edge overlaps them.  After a barrier, a scan over the dirty words compares
// each marked vertex with its last enqueued value and builds the next queue with one atomic per
// warp; a second barrier ends the level.
//
// Counters rotate over three slots: level L reads the queue length cnt[L % 3], appends to
// cnt[(L + 1) % 3] and clears cnt[(L + 2) % 3] (read by level L-1, written next by level L+1),
// so no slot is cleared while another block may still read it.  Values written by other blocks
// during the launch are read with __ldcg (L2), never through a possibly stale L1 line.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gridsync.cuh"
#include "hot.cuh"
#include "trace.cuh"

namespace tga {

struct TravArgs {
  Work w;
  LeanWork lw;           // lean schedule for the dense levels (run_first: the call's run table)
  TravCtl* ctl;
  int32_t* q[2];
  uint64_t* tp;          // arrival << 32 per vertex (all ones = unreached)
  uint64_t* tp_prev;     // arrival at which the vertex was last enqueued
  uint32_t* dirty;       // bit per vertex: relaxed in the current level
  int32_t ndirty;        // words of the bitmap
  uint32_t* mark[2];     // frontier marks: level L's frontier has mark[L & 1][x] == wave0 + L
  uint32_t* hops;        // BFS phase 2: hop level (all ones = unclaimed)
  int64_t lo, hi;
  uint64_t start;        // arrival << 32 of a source
  uint32_t wave0;
  int32_t dense_min;     // frontier size from which a level sweeps all lists
  int32_t level_cap;
  int32_t src;           // BFS source
  unsigned long long* edges;
  // connected components
  int32_t* label;
  uint8_t* reached;
  int32_t* touched;
  const int32_t* deg;
  int32_t cc_begin, cc_end, limit, early;
};

// Appends the entries of vertex v (v itself or its slices) to q at L's slot; one thread.
__device__ __forceinline__ void seed_queue(const Work& w, TravArgs& a, int L, int v) {
  int32_t* q = a.q[L & 1];
  const int s0 = w.slice_first[v], s1 = w.slice_first[v + 1];
  int k = 0;
  if (s0 == s1) q[k++] = v;
  else
    for (int j = s0; j < s1; ++j) q[k++] = -(j + 1);
  a.ctl->cnt[L % 3] = k;
}

// Scan over the dirty bitmap after a level: keep(v) decides (once per marked vertex, the marked
// vertices of a warp's words dealt over its lanes) whether v joins the next frontier; its entries are appended to nq,
// its frontier mark set, and touched(v) -> bool adds it to the touched list (CC).  Clears the
// bitmap.
template <class Keep, class Touched>
__device__ __forceinline__ void scan_dirty(TravArgs& a, int32_t* nq, int32_t* ncnt, uint32_t* mark, uint32_t wave,
                                           Keep keep, Touched touched) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = warp * 32; base < a.ndirty; base += nwarps * 32) {
    const int i = base + lane;
    uint32_t bits = 0;
    if (i < a.ndirty) {
      bits = __ldcg(a.dirty + i);
      if (bits) a.dirty[i] = 0;
    }
    deal_dirty(bits, base, [&](int v) {
      bool t = false;
      const bool k = v >= 0 && keep(v, t);
      const int at = warp_reserve(ncnt, k ? entry_count(a.w, v) : 0);
      const int tat = touched(0) ? warp_reserve(&a.ctl->tcnt, (k && t) ? 1 : 0) : 0;
      if (k) {
        write_entries(a.w, v, nq, at);
        mark[v] = wave;
        if (t) a.touched[tat] = v;
      }
    });
  }
}

// Runs levels from the queue at level L until a level appends nothing: level(w, q, qn, L, dense)
// relaxes, then, after a barrier, scan(nq, ncnt, L) builds the next queue.  Returns false if the
// launch failed.
template <class Level, class Scan>
__device__ __forceinline__ bool level_loop(const GraphView& g, TravArgs& a, int& L, Level level, Scan scan) {
  for (;;) {
    const int qn = __ldcg(&a.ctl->cnt[L % 3]);
    if (qn == 0) return true;
    if (L >= a.level_cap) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        set_err(g, kErrTimeout);
        a.ctl->status = 1;
      }
      return false;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.ctl->cnt[(L + 2) % 3] = 0;
      a.ctl->next[(L + 1) % 3] = 0;
    }
    Work w = a.w;
    w.next = &a.ctl->next[L % 3];
    level(w, a.q[L & 1], qn, L, qn >= a.dense_min);
    if (!grid_sync(a.ctl, g)) return false;
    scan(a.q[(L + 1) & 1], &a.ctl->cnt[(L + 1) % 3], L);
    if (!grid_sync(a.ctl, g)) return false;
    ++L;
  }
}

// Phase 1 level: tp[v] holds arrival << 32 and only decreases (RED.MIN); the scan enqueues every
// relaxed vertex whose arrival dropped below the one it was last enqueued with.
__device__ __forceinline__ unsigned long long relax_level(const GraphView& g, TravArgs& a, const Work& w,
                                                          const int32_t* q, int qn, int L, bool dense,
                                                          const int32_t* hids) {
  const uint32_t wcur = a.wave0 + (uint32_t)L;
  const uint32_t* mcur = a.mark[L & 1];
  uint32_t ax = 0;
  int prev_y = -1;
  auto begin = [&](int x, int, int) {
    if (x < g.active_begin || x > g.max_label) return false;
    ax = (uint32_t)(__ldcg(&a.tp[x]) >> 32);
    prev_y = -1;
    return true;
  };
  auto edge = [&](int, int y, int64_t t) {
    if (!keep_edge(g, a.lo, a.hi, y, t, prev_y)) return true;
    if ((int64_t)ax > t || t >= 0xFFFFFFFFll) return true;
    const bool hot = hot_is(hids, y);
    // (a hot successor's arrival has usually dropped to t or below already: no atomic then)
    if (hot && (int64_t)(__ldcg(&a.tp[y]) >> 32) <= t) return true;
    atomicMin((unsigned long long*)&a.tp[y], (unsigned long long)t << 32);
    if (!hot || !((__ldcg(&a.dirty[y >> 5]) >> (y & 31)) & 1u)) atomicOr(&a.dirty[y >> 5], 1u << (y & 31));
    return true;
  };
  if (dense) return run_lean_grid<true>(g, a.lw, [&](int x) { return __ldcg(&mcur[x]) == wcur; }, begin, edge, [](int) {});
  return drive_queue<true>(g, w, q, qn, begin, edge, [](int) {});
}

template <bool kTouched>
__device__ __forceinline__ void relax_scan(TravArgs& a, int32_t* nq, int32_t* ncnt, int L) {
  scan_dirty(
      a, nq, ncnt, a.mark[(L + 1) & 1], a.wave0 + (uint32_t)L + 1,
      [&](int v, bool& touched) {
        const uint64_t now = __ldcg(&a.tp[v]), before = __ldcg(&a.tp_prev[v]);
        if (now >= before) return false;
        a.tp_prev[v] = now;
        touched = kTouched && (before >> 32) == 0xFFFFFFFFull;
        return true;
      },
      [](int) { return kTouched; });
}

// Phase 2 level h: with the final arrivals fixed, an edge passing the same filters is tight when
// arrival(x) <= t == arrival(y); RED.MIN(hops[y], h + 1) claims y, and the scan enqueues the
// vertices whose hop level became h + 1 (earlier claims keep their smaller level).
__device__ __forceinline__ unsigned long long hop_level(const GraphView& g, TravArgs& a, const Work& w,
                                                        const int32_t* q, int qn, uint32_t h, bool dense,
                                                        const int32_t* hids) {
  uint32_t ax = 0;
  int prev_y = -1;
  auto begin = [&](int x, int, int) {
    if (x < g.active_begin || x > g.max_label) return false;
    ax = (uint32_t)(__ldcg(&a.tp[x]) >> 32);
    prev_y = -1;
    return true;
  };
  auto edge = [&](int, int y, int64_t t) {
    if (!keep_edge(g, a.lo, a.hi, y, t, prev_y)) return true;
    if ((int64_t)ax > t || t >= 0xFFFFFFFFll) return true;
    if ((int64_t)(__ldcg(&a.tp[y]) >> 32) != t) return true;
    const bool hot = hot_is(hids, y);
    if (hot && __ldcg(&a.hops[y]) <= h + 1) return true;  // claimed already
    atomicMin(&a.hops[y], h + 1);
    if (!hot || !((__ldcg(&a.dirty[y >> 5]) >> (y & 31)) & 1u)) atomicOr(&a.dirty[y >> 5], 1u << (y & 31));
    return true;
  };
  if (dense) return run_lean_grid<true>(g, a.lw, [&](int x) { return __ldcg(&a.hops[x]) == h; }, begin, edge, [](int) {});
  return drive_queue<true>(g, w, q, qn, begin, edge, [](int) {});
}

// Self-test of the bounded grid barrier: block 1 never arrives, so block 0's wait runs out after
// limit_ns; the launch ends with ctl->status set instead of waiting for ever.
__global__ void k_barrier_selftest(TravCtl* ctl, uint32_t* err, uint64_t limit_ns) {
  if (blockIdx.x != 0) return;  // the block that never arrives
  grid_sync_limit(ctl, err, limit_ns);
}

__global__ void TGA_TRAVERSE_BOUNDS k_bfs(GraphView g, TravArgs a) {
  __shared__ int32_t hids[kHotSlots];
  hot_load(g, hids);  // (the first grid barrier synchronises the block)
  int L = 0;
  unsigned long long mine = 0;
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  if (lead && a.src < g.n) {
    a.tp[a.src] = a.start;
    a.tp_prev[a.src] = a.start;
    a.mark[0][a.src] = a.wave0;
    seed_queue(a.w, a, 0, a.src);
  }
  if (!grid_sync(a.ctl, g)) return;
  const bool ok1 = level_loop(
      g, a, L,
      [&](const Work& w, const int32_t* q, int qn, int lv, bool dense) { mine += relax_level(g, a, w, q, qn, lv, dense, hids); },
      [&](int32_t* nq, int32_t* ncnt, int lv) { relax_scan<false>(a, nq, ncnt, lv); });
  if (!ok1) return;
  // Phase 2 from the source again; its levels continue the level numbering of the queues.  The
  // barrier keeps the seeding below from overwriting cnt[L % 3] before every block has read the
  // zero that ended phase 1.
  if (!grid_sync(a.ctl, g)) return;
  const int L2 = L;
  if (lead && a.src < g.n) seed_queue(a.w, a, L, a.src);
  if (!grid_sync(a.ctl, g)) return;
  const bool ok2 = level_loop(
      g, a, L,
      [&](const Work& w, const int32_t* q, int qn, int lv, bool dense) {
        mine += hop_level(g, a, w, q, qn, (uint32_t)(lv - L2), dense, hids);
      },
      [&](int32_t* nq, int32_t* ncnt, int lv) {
        const uint32_t claim = (uint32_t)(lv - L2) + 1;
        scan_dirty(
            a, nq, ncnt, a.mark[(lv + 1) & 1], a.wave0 + (uint32_t)lv + 1,
            [&](int v, bool&) { return __ldcg(&a.hops[v]) == claim; }, [](int) { return false; });
      });
  if (!ok2) return;
  add_edges(a.edges, mine);
  if (lead) a.ctl->levels = L;
}

// Seeds ascend from cc_begin below cc_end: the smallest unreached vertex with outdegree > 9
// starts a phase-1 traversal; every vertex it reaches gets its component number (last seed wins).
__global__ void TGA_TRAVERSE_BOUNDS k_cc(GraphView g, TravArgs a) {
  __shared__ int32_t hids[kHotSlots];
  hot_load(g, hids);
  __syncthreads();
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  int L = 0, comp = 0, small_run = 0;
  int64_t total = 0;
  unsigned long long mine = 0;
  int v = a.cc_begin;
  while (v < a.cc_end) {
    if (a.early && total > a.limit) break;
    int seed = INT32_MAX;
    for (int64_t from = v, chunk = 4096; from < a.cc_end; from += chunk, chunk = min(chunk * 2, (int64_t)1 << 22)) {
      const int to = (int)min(from + chunk, (int64_t)a.cc_end);
      for (int u = (int)from + tid; u < to; u += nthreads)
        if (!__ldcg(&a.reached[u]) && a.deg[u] > 9) atomicMin(&a.ctl->best, u);
      if (!grid_sync(a.ctl, g)) return;
      seed = __ldcg(&a.ctl->best);
      if (seed != INT32_MAX) break;
    }
    if (seed == INT32_MAX) break;
    if (lead) {
      a.ctl->tcnt = 0;
      a.tp[seed] = a.start;
      a.tp_prev[seed] = a.start;
      a.mark[L & 1][seed] = a.wave0 + (uint32_t)L;
      if (seed < g.n) seed_queue(a.w, a, L, seed);
    }
    if (!grid_sync(a.ctl, g)) return;
    const bool ok = level_loop(
        g, a, L,
        [&](const Work& w, const int32_t* q, int qn, int lv, bool dense) { mine += relax_level(g, a, w, q, qn, lv, dense, hids); },
        [&](int32_t* nq, int32_t* ncnt, int lv) { relax_scan<true>(a, nq, ncnt, lv); });
    if (!ok) return;
    const int reach = __ldcg(&a.ctl->tcnt);
    for (int i = tid; i < reach; i += nthreads) {
      const int y = __ldcg(&a.touched[i]);
      a.label[y] = comp;
      a.reached[y] = 1;
      a.tp[y] = kTpInf;
      a.tp_prev[y] = kTpInf;
    }
    if (lead) {
      a.label[seed] = comp;
      a.reached[seed] = 1;
      a.tp[seed] = kTpInf;
      a.tp_prev[seed] = kTpInf;
      a.ctl->best = INT32_MAX;  // every thread read it before the seeding barrier
    }
    if (!grid_sync(a.ctl, g)) return;
    ++comp;
    total += reach + 1;
    small_run = (reach + 1 < 5) ? small_run + 1 : 0;
    if (a.early && small_run > 50) break;
    v = seed + 1;
  }
  add_edges(a.edges, mine);
  if (lead) {
    a.ctl->levels = L;
    a.ctl->comps = comp;
  }
}

__global__ void k_unpack_bfs(const uint64_t* tp, const uint32_t* hops_in, int32_t* arr, int32_t* hops, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t wd = tp[i];
  const bool inf = (wd >> 32) == 0xFFFFFFFFull;
  arr[i] = inf ? INT32_MAX : (int32_t)(wd >> 32);
  const uint32_t hv = hops_in[i];
  hops[i] = (inf || hv == 0xFFFFFFFFu) ? INT32_MAX : (int32_t)hv;
}

// Buffers of a traversal: s_a arrivals and enqueued arrivals, s_b/s_c the two mark arrays, s_d
// hops (BFS) or labels (CC), s_g the dirty bitmap, s_q0/s_q1 queues, s_cnt the control block.
static int trav_buffers(GraphHandle& h) {
  const size_t nv = (size_t)h.view.max_vertex;
  const size_t qcap = nv + (size_t)h.nslices + 1;
  const size_t dirty = ((nv + 31) / 32) * 4;
  int rc;
  if ((rc = h.s_a.ensure(nv * 16)) || (rc = h.s_b.ensure(nv * 4)) || (rc = h.s_c.ensure(nv * 4)) ||
      (rc = h.s_d.ensure(nv * 4)) || (rc = h.s_q0.ensure(qcap * 4)) || (rc = h.s_q1.ensure(qcap * 4)) ||
      (rc = h.s_g.ensure(dirty)) || (rc = h.s_cnt.ensure(sizeof(TravCtl))))
    return rc;
  return TGA_OK;
}

// Common set-up of the launch arguments: arrivals unreached, marks cleared, control block zeroed.
static TravArgs trav_args(GraphHandle& h, int64_t t_lo, int64_t t_hi, unsigned long long* edges) {
  const int32_t nv = h.view.max_vertex;
  TravArgs a{};
  a.w = Work{h.d_items.as<WorkItem>(), h.d_slices.as<SliceState>(), h.d_slice_first.as<int32_t>(), nullptr, h.nitems,
             h.d_order.as<int32_t>(), h.norder, h.d_run_first.as<int32_t>()};
  a.lw = LeanWork{h.d_lean.as<LeanEntry>(), h.nlean, h.d_slices.as<SliceState>(), h.d_run_first.as<int32_t>()};
  prepare_runs(h, t_lo, t_hi);
  a.ctl = h.s_cnt.as<TravCtl>();
  a.q[0] = h.s_q0.as<int32_t>();
  a.q[1] = h.s_q1.as<int32_t>();
  a.tp = h.s_a.as<uint64_t>();
  a.tp_prev = a.tp + nv;
  a.dirty = h.s_g.as<uint32_t>();
  a.ndirty = (nv + 31) / 32;
  a.mark[0] = h.s_b.as<uint32_t>();
  a.mark[1] = h.s_c.as<uint32_t>();
  a.lo = t_lo;
  a.hi = t_hi;
  a.start = (uint64_t)std::max<int64_t>(t_lo, 0) << 32;
  a.wave0 = 1;
  a.dense_min = std::max<int32_t>(h.dense_min, 1);
  a.level_cap = 1 << 20;
  a.edges = edges;
  KL(k_fill_u64, grid_for(2 * (int64_t)nv, kBlock))(a.tp, kTpInf, 2 * (int64_t)nv);
  cudaMemsetAsync(a.dirty, 0, (size_t)a.ndirty * 4, h.stream);
  cudaMemsetAsync(a.mark[0], 0, (size_t)nv * 4, h.stream);
  cudaMemsetAsync(a.mark[1], 0, (size_t)nv * 4, h.stream);
  TravCtl ctl{};
  ctl.best = INT32_MAX;
  std::memcpy(h.h_pinned + 32, &ctl, sizeof ctl);
  cudaMemcpyAsync(a.ctl, h.h_pinned + 32, sizeof ctl, cudaMemcpyHostToDevice, h.stream);
  return a;
}

// Cooperative launch of a traversal kernel on all SMs; then reads the control block back.
template <class K>
static int trav_launch(GraphHandle& h, K kernel, TravArgs& a, TravCtl& out) {
  int per_sm = 0;
  TGA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
  if (per_sm < 1) return fail(TGA_E_CUDA, "traversal kernel cannot be resident");
  void* args[] = {&h.view, &a};
  cudaEvent_t* ev = h.kernel_begin();
  ++h.timing.launches;
  TGA_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kernel, dim3(per_sm * h.sm_count), dim3(kBlock), args, 0,
                                           h.stream));
  h.kernel_end(ev);
  TGA_CUDA_TRY(cudaMemcpyAsync(h.h_pinned + 32, a.ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  std::memcpy(&out, h.h_pinned + 32, sizeof out);
  if (out.status) return fail(TGA_E_TIMEOUT, "a grid barrier wait ran out");
  return TGA_OK;
}

}  // namespace tga

using namespace tga;

extern "C" {

int tga_barrier_selftest(double limit_ms, int32_t* status_out) {
  if (limit_ms <= 0 || limit_ms > 10000) return fail(TGA_E_ARG, "limit must be in (0, 10 s]");
  TravCtl* ctl = nullptr;
  uint32_t* err = nullptr;
  TGA_CUDA_TRY(cudaMalloc((void**)&ctl, sizeof(TravCtl) + 16));
  err = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(ctl) + sizeof(TravCtl));
  int rc = TGA_OK;
  TravCtl host{};
  uint32_t herr = 0;
  uint64_t limit = (uint64_t)(limit_ms * 1e6);
  void* args[] = {&ctl, &err, &limit};
  if (cudaMemset(ctl, 0, sizeof(TravCtl) + 16) != cudaSuccess ||
      cudaLaunchCooperativeKernel((const void*)k_barrier_selftest, dim3(2), dim3(32), args, 0, nullptr) != cudaSuccess ||
      cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(&host, ctl, sizeof host, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(TGA_E_CUDA, std::string("barrier self-test: ") + cudaGetErrorString(cudaGetLastError()));
  cudaFree(ctl);
  if (rc) return rc;
  if (status_out) *status_out = host.status && (herr & kErrTimeout) ? 1 : 0;
  return TGA_OK;
}

int tga_bfs(tga_graph* gp, int32_t src, int64_t t_lo, int64_t t_hi, int32_t* arrival_out, int32_t* hops_out) {
  TGA_TRACE("tga_bfs");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (src < 0) src = h.cfg.bfs_start_vertex;
  if (src < 0 || src >= h.view.max_vertex) return fail(TGA_E_ARG, "source out of range");
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(trav_buffers(h));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  TravArgs a = trav_args(h, t_lo, t_hi, edges);
  a.src = src;
  a.hops = h.s_d.as<uint32_t>();
  cudaMemsetAsync(a.hops, 0xFF, (size_t)nv * 4, h.stream);
  cudaMemsetAsync(a.hops + src, 0, 4, h.stream);
  if (src >= h.view.n) {  // no list: only the source itself is reached
    cudaMemcpyAsync(a.tp + src, &a.start, 8, cudaMemcpyHostToDevice, h.stream);
  }
  TravCtl ctl{};
  TGA_TRY(trav_launch(h, k_bfs, a, ctl));
  int32_t* arr = h.s_q0.as<int32_t>();
  int32_t* hops = h.s_q1.as<int32_t>();
  KL(k_unpack_bfs, grid_for(nv, kBlock))(a.tp, a.hops, arr, hops, nv);
  if (arrival_out) cudaMemcpyAsync(arrival_out, arr, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (hops_out) cudaMemcpyAsync(hops_out, hops, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = ctl.levels;
  return finish(h, edges);
}

int tga_cc(tga_graph* gp, int64_t t_lo, int64_t t_hi, int32_t flags, int32_t* label_out, int32_t* components_out) {
  TGA_TRACE("tga_cc");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  if (!(flags & TGA_CC_ONE_SEED)) return cc_seed_batches(h, t_lo, t_hi, flags, label_out, components_out);
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(trav_buffers(h));
  TGA_TRY(h.s_e.ensure((size_t)nv));       // reached
  TGA_TRY(h.s_f.ensure((size_t)nv * 4));   // touched list
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  TravArgs a = trav_args(h, t_lo, t_hi, edges);
  a.label = h.s_d.as<int32_t>();
  a.reached = h.s_e.as<uint8_t>();
  a.touched = h.s_f.as<int32_t>();
  a.deg = h.d_deg.as<int32_t>();
  a.cc_begin = std::max(h.cfg.cc_vertex_begin, 0);
  a.cc_end = std::min(std::min(h.view.max_label, nv), h.view.n);
  a.limit = (int32_t)(0.8 * h.view.max_label);
  a.early = (flags & TGA_CC_EARLY_EXIT) ? 1 : 0;
  KL(k_fill_i32, grid_for(nv, kBlock))(a.label, -1, nv);
  cudaMemsetAsync(a.reached, 0, (size_t)nv, h.stream);
  TravCtl ctl{};
  TGA_TRY(trav_launch(h, k_cc, a, ctl));
  if (label_out) cudaMemcpyAsync(label_out, a.label, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (components_out) *components_out = ctl.comps;
  h.timing.iterations = ctl.levels;
  return finish(h, edges);
}

}  // extern "C"
