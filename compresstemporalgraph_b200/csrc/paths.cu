// Temporal path queries composed from the batched traversal (host code only: every kernel it runs
// is the multi-source BFS of batch.cu).
#include <algorithm>
#include <climits>
#include <new>
#include <system_error>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "trace.cuh"

using namespace tga;

namespace {

void add_timing(tga_timing& sum, const tga_timing& t) {
  sum.total_ms += t.total_ms;
  sum.decode_ms += t.decode_ms;
  sum.decode_launches += t.decode_launches;
  sum.edges_decoded += t.edges_decoded;
  sum.compressed_bytes += t.compressed_bytes;
  sum.iterations += t.iterations;
  sum.launches += t.launches;
}

}  // namespace

// Fastest paths (temporal_ligra apps/temporal/Fastest-Compute.C:1-174 asks for the least elapsed
// time from a source within [start, end]; there edges have a start and an end time, here an edge
// happens at one instant).  A path's duration is the time of its last edge minus the time of its
// first edge, its first edge leaving src at one of the distinct in-window timestamps d of src's
// out-edges.  The earliest arrival from src over the window [d, t_hi) (tga_bfs) bounds the
// duration of every path that departs at d or later, and the bound is met by a path departing at
// exactly d when d minimises it, so
//     duration(v) = min over d of (arrival_d(v) - d),
// with paths following tga_bfs's edge rule.  The departures run as rows of the multi-source
// traversal, up to 256 per launch and fewer when max_vertex is large (host rows are bounded to
// about 256 MiB).  Host work is O(departures x max_vertex) for the minimum, on up to 32 threads.
static int tga_fastest_impl(tga_graph* gp, int32_t src, int64_t t_lo, int64_t t_hi, int64_t* duration_out,
                            int64_t* departure_out) {
  TGA_TRACE("tga_fastest");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  if (src < 0 || src >= nv) return fail(TGA_E_ARG, "source out of range");
  if (t_lo < 0 || t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");

  tga_timing sum{};
  std::vector<int64_t> dep;
  if (src < h.view.n) {
    int32_t cnt = 0;
    TGA_TRY(tga_neighbors(gp, src, nullptr, nullptr, 0, &cnt));
    add_timing(sum, h.timing);
    std::vector<int32_t> dst((size_t)std::max(cnt, 1));
    std::vector<int64_t> ts((size_t)std::max(cnt, 1));
    TGA_TRY(tga_neighbors(gp, src, dst.data(), ts.data(), cnt, &cnt));
    add_timing(sum, h.timing);
    for (int32_t i = 0; i < cnt; ++i)
      if (ts[(size_t)i] >= t_lo && ts[(size_t)i] < t_hi) dep.push_back(ts[(size_t)i]);
    std::sort(dep.begin(), dep.end());
    dep.erase(std::unique(dep.begin(), dep.end()), dep.end());
  }

  std::vector<int64_t> best((size_t)nv, -1), when((size_t)nv, -1);
  best[(size_t)src] = 0;
  const int64_t row_cap = std::max<int64_t>(1, (int64_t(256) << 20) / (4 * (int64_t)nv));
  const int32_t per = (int32_t)std::min<int64_t>(256, row_cap);
  std::vector<int32_t> rows;
  std::vector<int32_t> srcs((size_t)per, src);
  std::vector<int64_t> his((size_t)per, t_hi);
  for (size_t b = 0; b < dep.size(); b += (size_t)per) {
    const int32_t k = (int32_t)std::min<size_t>((size_t)per, dep.size() - b);
    rows.resize((size_t)k * (size_t)nv);
    TGA_TRY(tga_bfs_batch(gp, k, srcs.data(), dep.data() + b, his.data(), rows.data()));
    add_timing(sum, h.timing);
    // Rows ascend in departure time, so a strict improvement keeps the earliest departure.  Each
    // vertex's minimum is independent: large batches are split by vertex range over host threads.
    auto fold = [&](int32_t v0, int32_t v1) {
      for (int32_t i = 0; i < k; ++i) {
        const int64_t d = dep[b + (size_t)i];
        const int32_t* arr = rows.data() + (size_t)i * (size_t)nv;
        for (int32_t v = v0; v < v1; ++v) {
          if (arr[v] == INT32_MAX || v == src) continue;
          const int64_t dur = (int64_t)arr[v] - d;
          if (best[(size_t)v] < 0 || dur < best[(size_t)v]) {
            best[(size_t)v] = dur;
            when[(size_t)v] = d;
          }
        }
      }
    };
    const int64_t work = (int64_t)k * nv;
    const int threads = work < (int64_t(1) << 18)
                            ? 1
                            : (int)std::min<unsigned>(32, std::max(1u, std::thread::hardware_concurrency()));
    // Vertices [0, covered) go to threads; whatever no thread could be started for runs here.
    int32_t covered = 0;
    std::vector<std::thread> pool;
    if (threads > 1) {
      const int32_t chunk = (int32_t)((nv + threads - 1) / threads);
      try {
        for (int t = 0; t < threads; ++t) {
          const int32_t v0 = (int32_t)std::min<int64_t>((int64_t)t * chunk, nv);
          const int32_t v1 = (int32_t)std::min<int64_t>((int64_t)v0 + chunk, nv);
          if (v0 < v1) {
            pool.emplace_back(fold, v0, v1);
            covered = v1;
          }
        }
      } catch (const std::system_error&) {
      }
    }
    for (auto& th : pool) th.join();
    if (covered < nv) fold(covered, nv);
  }
  if (duration_out) std::copy(best.begin(), best.end(), duration_out);
  if (departure_out) std::copy(when.begin(), when.end(), departure_out);
  h.timing = sum;
  return TGA_OK;
}

// Time-reversed copy of a graph, for latest-departure queries (temporal_ligra
// apps/temporal/LatestDeparture-Compute.C:1-149 transposes the graph and walks it from the target).
// The lists are decoded on the device (tga_decode_all) and written on the host (tga_write_reversed):
// edge (x -> y, t) becomes (y -> x, pivot - t).
static int tga_reverse_impl(tga_graph* gp, int64_t pivot, const char* dir, const char* base, int64_t* pivot_out) {
  TGA_TRACE("tga_reverse");
  if (!gp || !dir || !base) return fail(TGA_E_ARG, "null argument");
  GraphHandle& h = *gp;
  const int64_t n = h.view.n;
  std::vector<int64_t> off((size_t)n + 1);
  TGA_TRY(tga_decode_all(gp, off.data(), nullptr, nullptr, 0));
  const int64_t m = off[(size_t)n];
  std::vector<int32_t> dst((size_t)std::max<int64_t>(m, 1));
  std::vector<int64_t> ts((size_t)std::max<int64_t>(m, 1));
  TGA_TRY(tga_decode_all(gp, off.data(), dst.data(), ts.data(), m));
  if (pivot < 0) pivot = m ? *std::max_element(ts.begin(), ts.begin() + m) : 0;
  TGA_TRY(tga_write_reversed(off.data(), dst.data(), ts.data(), n, pivot, dir, base, nullptr));
  if (pivot_out) *pivot_out = pivot;
  return TGA_OK;
}

// Latest departures towards one target: out[v] = the latest time a path v -> target can leave v,
// using edges with t in [t_lo, t_hi).  On the reversed copy a forward path v -> target leaving at d
// is a path target -> v arriving at pivot - d, and the window maps to (pivot - t_hi, pivot - t_lo],
// so one earliest-arrival traversal from the target gives every vertex's latest departure.
static int tga_latest_departure_impl(tga_graph* rev, int64_t pivot, int32_t target, int64_t t_lo,
                                     int64_t t_hi, int64_t* out) {
  TGA_TRACE("tga_latest_departure");
  if (!rev) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *rev;
  const int32_t nv = h.view.max_vertex;
  if (target < 0 || target >= nv) return fail(TGA_E_ARG, "target out of range");
  if (t_lo < 0 || t_lo >= t_hi || pivot < 0) return fail(TGA_E_ARG, "empty time window");
  std::vector<int32_t> arr((size_t)nv);
  if (t_lo > pivot) {  // every edge is earlier than the window
    if (out) std::fill(out, out + nv, int64_t(-1));
    if (out) out[target] = std::min(t_hi - 1, pivot);
    return TGA_OK;
  }
  const int64_t lo = t_hi > pivot ? 0 : pivot - t_hi + 1;
  const int64_t hi = pivot - t_lo + 1;
  TGA_TRY(tga_bfs(rev, target, lo, hi, arr.data(), nullptr));
  if (out)
    for (int32_t v = 0; v < nv; ++v) out[v] = arr[(size_t)v] == INT32_MAX ? -1 : pivot - arr[(size_t)v];
  return TGA_OK;
}

// C entry points: host allocation failures come back as TGA_E_OOM instead of unwinding into C.
extern "C" int tga_fastest(tga_graph* g, int32_t src, int64_t t_lo, int64_t t_hi, int64_t* duration_out,
                           int64_t* departure_out) {
  try {
    return tga_fastest_impl(g, src, t_lo, t_hi, duration_out, departure_out);
  } catch (const std::bad_alloc&) {
    return fail(TGA_E_OOM, "host allocation failed");
  }
}

extern "C" int tga_reverse(tga_graph* g, int64_t pivot, const char* dir, const char* base, int64_t* pivot_out) {
  try {
    return tga_reverse_impl(g, pivot, dir, base, pivot_out);
  } catch (const std::bad_alloc&) {
    return fail(TGA_E_OOM, "host allocation failed");
  }
}

extern "C" int tga_latest_departure(tga_graph* rev, int64_t pivot, int32_t target, int64_t t_lo, int64_t t_hi,
                                    int64_t* out) {
  try {
    return tga_latest_departure_impl(rev, pivot, target, t_lo, t_hi, out);
  } catch (const std::bad_alloc&) {
    return fail(TGA_E_OOM, "host allocation failed");
  }
}

// ---------------------------------------------------------------------------------------------
// Fewest-hop temporal paths (temporal_ligra apps/temporal/Shortest-Compute.C asks for the shortest
// time-respecting paths from a source within [start, end]; its update keeps a label only when it is
// both earlier and shorter, which depends on the visiting order).  Here the value is exact: hops[v]
// = the fewest edges on a time-respecting path from src to v within [t_lo, t_hi), with tga_bfs's
// edge rule (edge (x->y, t) usable when arrival(x) <= t, first in-window occurrence of equal
// consecutive successors).  Level-synchronous relaxation:
//     A_k[v] = min(A_{k-1}[v], min over usable edges (x->v, t) with A_{k-1}[x] <= t of t),
// where only the vertices whose A dropped at level k-1 are expanded, reading A_{k-1} (prev) while
// writing A_k (next) with RED.MIN, so every level is deterministic; hops[v] is the first k with
// A_k[v] finite, and the last A is the earliest arrival (tga_bfs's).
#include "gridsync.cuh"

namespace tga {

namespace {

constexpr uint32_t kSpInf = 0xFFFFFFFFu;

struct SpArgs {
  const uint32_t* prev;
  uint32_t* next;
  uint32_t* dirty;
  int64_t lo, hi;
  unsigned long long* edges;
};

__global__ void TGA_TRAVERSE_BOUNDS k_sp_relax(GraphView g, Work w, SpArgs a, const int32_t* q, int32_t qn) {
  uint32_t ax = kSpInf;
  int prev_y = -1;
  const unsigned long long mine = drive_queue<true>(
      g, w, q, qn,
      [&](int x, int, int) {
        if (x < g.active_begin || x > g.max_label) return false;
        ax = __ldcg(a.prev + x);
        prev_y = -1;
        return ax != kSpInf;
      },
      [&](int, int y, int64_t t) {
        if (!keep_edge(g, a.lo, a.hi, y, t, prev_y)) return true;
        if ((int64_t)ax > t || t >= (int64_t)kSpInf) return true;
        if (atomicMin(a.next + y, (uint32_t)t) > (uint32_t)t) atomicOr(a.dirty + (y >> 5), 1u << (y & 31));
        return true;
      },
      [](int) {});
  add_edges(a.edges, mine);
}

// After level `level`: every vertex whose arrival dropped takes it, gets its hop count if it was
// unreached, and joins the next queue (itself, or all its slices).
// (the marked vertices of a warp's 32 words dealt over its lanes, queue places reserved per warp)
__global__ void k_sp_scan(Work w, uint32_t* prev, const uint32_t* next, uint32_t* dirty, int32_t* hops, int32_t nwords,
                          int32_t level, int32_t* q, int32_t* qcnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int base = i & ~31;
  if (base >= nwords) return;  // (whole warps leave together)
  uint32_t bits = 0;
  if (i < nwords) {
    bits = dirty[i];
    if (bits) dirty[i] = 0;
  }
  deal_dirty(bits, base, [&](int y) {
    if (y >= 0) {
      if (prev[y] == kSpInf) hops[y] = level;
      prev[y] = next[y];
    }
    const int at = warp_reserve(qcnt, y >= 0 ? entry_count(w, y) : 0);
    if (y >= 0) write_entries(w, y, q, at);
  });
}

__global__ void k_sp_unpack(const uint32_t* prev, int32_t* arr, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) arr[i] = prev[i] == kSpInf ? INT32_MAX : (int32_t)prev[i];
}

}  // namespace

static int tga_shortest_impl(tga_graph* gp, int32_t src, int64_t t_lo, int64_t t_hi, int32_t* hops_out,
                             int32_t* arrival_out) {
  TGA_TRACE("tga_shortest");
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  if (src < 0 || src >= nv) return fail(TGA_E_ARG, "source out of range");
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nwords = (nv + 31) / 32;
  const size_t qcap = (size_t)nv + (size_t)h.nslices + 1;
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));
  TGA_TRY(h.s_b.ensure((size_t)nv * 4));
  TGA_TRY(h.s_c.ensure((size_t)nv * 4));
  TGA_TRY(h.s_d.ensure((size_t)nwords * 4));
  TGA_TRY(h.s_q0.ensure(qcap * 4));
  TGA_TRY(h.s_q1.ensure(qcap * 4));
  TGA_TRY(h.s_cnt.ensure(64));
  TGA_TRY(h.begin_call());
  prepare_runs(h, t_lo, t_hi);
  unsigned long long* edges = edge_counter(h);
  uint32_t* prev = h.s_a.as<uint32_t>();
  uint32_t* next = h.s_b.as<uint32_t>();
  int32_t* hops = h.s_c.as<int32_t>();
  uint32_t* dirty = h.s_d.as<uint32_t>();
  int32_t* q[2] = {h.s_q0.as<int32_t>(), h.s_q1.as<int32_t>()};
  int32_t* qcnt = h.s_cnt.as<int32_t>();
  cudaMemsetAsync(prev, 0xFF, (size_t)nv * 4, h.stream);
  cudaMemsetAsync(next, 0xFF, (size_t)nv * 4, h.stream);
  KL(k_fill_i32, grid_for(nv, kBlock))(hops, INT32_MAX, nv);
  cudaMemsetAsync(dirty, 0, (size_t)nwords * 4, h.stream);
  const uint32_t start = (uint32_t)(t_lo > 0 ? std::min<int64_t>(t_lo, (int64_t)kSpInf - 1) : 0);
  const int32_t zero = 0;
  TGA_CUDA_TRY(cudaMemcpyAsync(prev + src, &start, 4, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(next + src, &start, 4, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(hops + src, &zero, 4, cudaMemcpyHostToDevice, h.stream));
  std::vector<int32_t> first;
  int32_t qn = src < h.view.n ? seed_entries(h, src, first) : 0;
  if (qn) TGA_CUDA_TRY(cudaMemcpyAsync(q[0], first.data(), (size_t)qn * 4, cudaMemcpyHostToDevice, h.stream));
  const SpArgs a{prev, next, dirty, t_lo, t_hi, edges};
  int32_t level = 0;
  for (; qn > 0; ++level) {
    if (level >= nv) return fail(TGA_E_TIMEOUT, "tga_shortest: more levels than vertices");
    const Work w = work_of(h);
    TGA_CUDA_TRY(cudaMemsetAsync(qcnt, 0, 4, h.stream));
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_sp_relax, decode_grid(h, qn))(h.view, w, a, q[level & 1], qn);
    h.kernel_end(ev);
    KL(k_sp_scan, grid_for(nwords, kBlock))(w, prev, next, dirty, hops, nwords, level + 1, q[(level + 1) & 1], qcnt);
    TGA_CUDA_TRY(cudaMemcpyAsync(&h.h_pinned[20], qcnt, 4, cudaMemcpyDeviceToHost, h.stream));
    TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
    qn = (int32_t)h.h_pinned[20];
  }
  int32_t* arr = reinterpret_cast<int32_t*>(next);  // next is no longer needed
  KL(k_sp_unpack, grid_for(nv, kBlock))(prev, arr, nv);
  if (hops_out) cudaMemcpyAsync(hops_out, hops, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (arrival_out) cudaMemcpyAsync(arrival_out, arr, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = level;
  return finish(h, edges);
}

}  // namespace tga

extern "C" int tga_shortest(tga_graph* g, int32_t src, int64_t t_lo, int64_t t_hi, int32_t* hops_out,
                            int32_t* arrival_out) {
  try {
    return tga::tga_shortest_impl(g, src, t_lo, t_hi, hops_out, arrival_out);
  } catch (const std::bad_alloc&) {
    return fail(TGA_E_OOM, "host allocation failed in tga_shortest");
  }
}
