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
// dropped, clears the finished level's masks and builds the next queue.  Same queue rotation,
// dense-level sweep and bounded barrier as the single-source traversal (traverse.cu).
#include <algorithm>
#include <cstring>
#include <vector>

#include "gridsync.cuh"

namespace tga {

constexpr int kMaxSources = 256;
constexpr int kWords = kMaxSources / 64;
constexpr uint32_t kNoArrival = 0xFFFFFFFFu;

struct MultiArgs {
  Work w;
  TravCtl* ctl;
  int32_t* q[2];
  uint32_t* arr;             // [nsrc][nv] arrival of v for source s (kNoArrival: unreached)
  uint32_t* prev;            // [nsrc][nv] arrival at which v was last enqueued for s
  uint64_t* F[2];            // [nv][kWords] frontier masks: level L reads F[L & 1], fills F[(L+1) & 1]
  uint32_t* dirty;           // bit per vertex: relaxed in the current level
  int32_t ndirty;
  const int64_t* lo;         // [nsrc] windows [lo, hi)
  const int64_t* hi;
  const int32_t* run_first;  // [nruns][kMaxSources] list index of a cut run's first in-window edge
  int32_t nsrc, nv;
  int32_t dense_min, level_cap;
  unsigned long long* edges;
};

// Relaxes one level of the multi-source traversal.
__device__ __forceinline__ unsigned long long multi_relax(const GraphView& g, MultiArgs& a, const Work& w,
                                                          const int64_t* slo, const int64_t* shi, const int32_t* q,
                                                          int qn, int L, bool dense) {
  const uint64_t* Fc = a.F[L & 1];
  uint64_t* Fn = a.F[(L + 1) & 1];
  const size_t nv = (size_t)a.nv;
  uint64_t M[kWords], seen[kWords];
  int xcur = 0, yprev = -1;
  constexpr int kKeepSeen = -3;  // the first successor continues a run begun in an earlier slice
  auto begin = [&](int x, int first, int, int run) {
    if (x < g.active_begin || x > g.max_label) return false;
    uint64_t any = 0;
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      M[k] = __ldcg(Fc + (size_t)x * kWords + k);
      seen[k] = 0;
      any |= M[k];
    }
    if (!any) return false;
    xcur = x;
    yprev = -1;
    if (run >= 0) {
      // Sources whose first in-window edge of this run lies before the slice saw the run already.
      const int32_t* rf = a.run_first + (size_t)run * kMaxSources;
#pragma unroll
      for (int k = 0; k < kWords; ++k)
        for (uint64_t c = M[k]; c; c &= c - 1) {
          const int b = __ffsll((long long)c) - 1;
          if (__ldg(rf + k * 64 + b) < first) seen[k] |= 1ull << b;
        }
      yprev = kKeepSeen;
    }
    return true;
  };
  auto edge = [&](int, int y, int64_t t) {
    if (yprev == kKeepSeen) {
      yprev = y;
    } else if (y != yprev) {
#pragma unroll
      for (int k = 0; k < kWords; ++k) seen[k] = 0;
      yprev = y;
    }
    const bool usable = y >= g.active_begin && y < g.max_vertex && t >= 0 && t < 0xFFFFFFFFll;
    bool any = false;
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      for (uint64_t c = M[k] & ~seen[k]; c; c &= c - 1) {
        const int b = __ffsll((long long)c) - 1;
        const int s = k * 64 + b;
        if (t < slo[s] || t >= shi[s]) continue;
        seen[k] |= 1ull << b;
        if (!usable) continue;
        const uint32_t ax = __ldcg(a.arr + (size_t)s * nv + xcur);
        if ((int64_t)ax > t) continue;
        atomicMin(a.arr + (size_t)s * nv + y, (uint32_t)t);
        atomicOr((unsigned long long*)(Fn + (size_t)y * kWords + k), (unsigned long long)(1ull << b));
        any = true;
      }
    }
    if (any) atomicOr(&a.dirty[y >> 5], 1u << (y & 31));
    return true;
  };
  if (dense) {
    return run_order<false, true, false, true, true>(
        g, w,
        [&](int x) {
          uint64_t any = 0;
#pragma unroll
          for (int k = 0; k < kWords; ++k) any |= __ldcg(Fc + (size_t)x * kWords + k);
          return any != 0;
        },
        begin, edge, [](int) {});
  }
  return drive_queue<false, true, true>(g, w, q, qn, begin, edge, [](int) {});
}

// After level L (targets F[(L+1) & 1]): clears the masks of level L's frontier (queue cq, cn), keeps
// per dirty vertex only the sources whose arrival dropped, and appends the vertices with any such
// source to the next queue.
__device__ __forceinline__ void multi_scan(MultiArgs& a, const int32_t* cq, int cn, int32_t* nq, int32_t* ncnt,
                                           int L) {
  uint64_t* Fc = a.F[L & 1];
  uint64_t* Fn = a.F[(L + 1) & 1];
  const size_t nv = (size_t)a.nv;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  for (int i = tid; i < cn; i += nthreads) {
    const int e = __ldcg(cq + i);
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
    uint32_t keep_bits = 0;
    int n = 0;
    for (uint32_t b = bits; b; b &= b - 1) {
      const int v = i * 32 + __ffs(b) - 1;
      bool keep = false;
#pragma unroll
      for (int k = 0; k < kWords; ++k) {
        const uint64_t m = __ldcg(Fn + (size_t)v * kWords + k);
        uint64_t kept = 0;
        for (uint64_t c = m; c; c &= c - 1) {
          const int bb = __ffsll((long long)c) - 1;
          const size_t at = (size_t)(k * 64 + bb) * nv + v;
          const uint32_t now = __ldcg(a.arr + at), before = __ldcg(a.prev + at);
          if (now < before) {
            a.prev[at] = now;
            kept |= 1ull << bb;
          }
        }
        if (kept != m) Fn[(size_t)v * kWords + k] = kept;
        keep |= kept != 0;
      }
      if (keep) {
        keep_bits |= b & (~b + 1);
        n += entry_count(a.w, v);
      }
    }
    int at = warp_reserve(ncnt, n);
    for (uint32_t b = keep_bits; b; b &= b - 1) {
      const int v = i * 32 + __ffs(b) - 1;
      write_entries(a.w, v, nq, at);
      at += entry_count(a.w, v);
    }
  }
}

__global__ void TGA_DECODE_BOUNDS k_bfs_multi(GraphView g, MultiArgs a) {
  __shared__ int64_t slo[kMaxSources], shi[kMaxSources];
  for (int s = threadIdx.x; s < kMaxSources; s += blockDim.x) {
    slo[s] = s < a.nsrc ? a.lo[s] : 0;
    shi[s] = s < a.nsrc ? a.hi[s] : 0;
  }
  __syncthreads();
  unsigned long long mine = 0;
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  // The sources were seeded as level 0's relaxations: the scan turns them into level 1's queue.
  multi_scan(a, a.q[0], 0, a.q[1], &a.ctl->cnt[1], 0);
  if (!grid_sync(a.ctl, g)) return;
  int L = 1;
  for (;;) {
    const int qn = __ldcg(&a.ctl->cnt[L % 3]);
    if (qn == 0) break;
    if (L >= a.level_cap) {
      if (lead) {
        set_err(g, kErrTimeout);
        a.ctl->status = 1;
      }
      return;
    }
    if (lead) {
      a.ctl->cnt[(L + 2) % 3] = 0;
      a.ctl->next[(L + 1) % 3] = 0;
    }
    Work w = a.w;
    w.next = &a.ctl->next[L % 3];
    mine += multi_relax(g, a, w, slo, shi, a.q[L & 1], qn, L, qn >= a.dense_min);
    if (!grid_sync(a.ctl, g)) return;
    multi_scan(a, a.q[L & 1], qn, a.q[(L + 1) & 1], &a.ctl->cnt[(L + 1) % 3], L);
    if (!grid_sync(a.ctl, g)) return;
    ++L;
  }
  add_edges(a.edges, mine);
  if (lead) a.ctl->levels = L;
}

// Sources of the batch: arrival and level-0 relaxation of each source vertex.
__global__ void k_bfs_multi_seed(MultiArgs a, const int32_t* src, int32_t n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.nsrc) return;
  const int v = src[s];
  const int64_t start = a.lo[s] > 0 ? a.lo[s] : 0;
  a.arr[(size_t)s * a.nv + v] = (uint32_t)start;
  if (v < n) {
    atomicOr((unsigned long long*)(a.F[1] + (size_t)v * kWords + s / 64), (unsigned long long)(1ull << (s & 63)));
    atomicOr(&a.dirty[v >> 5], 1u << (v & 31));
  }
}

// Per-source first in-window edge of each run of equal successors cut by slices: one thread per
// (run, overlapping slice) decodes the run's part of the slice and lowers run_first[run][s] for
// every source s whose window holds one of those edges.
__global__ void TGA_DECODE_BOUNDS k_run_first_multi(GraphView g, const SliceState* slices, const RunInfo* runs,
                                                    const int2* pairs, int32_t npairs, const int64_t* lo,
                                                    const int64_t* hi, int32_t nsrc, int32_t* run_first) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const int2 pr = pairs[p];
  const RunInfo r = runs[pr.x];
  const SliceState& s = slices[pr.y];
  DeepState deep;
  EdgeCursor c(&deep);
  cursor_restore(g, c, s);
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
      atomicMin(&run_first[(size_t)pr.x * kMaxSources + q], i);
    }
  }
}

__global__ void k_multi_unpack(const uint32_t* arr, int32_t* out, int64_t total) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) {
    const uint32_t v = arr[i];
    out[i] = v == kNoArrival ? INT32_MAX : (int32_t)v;
  }
}

// One batch of at most kMaxSources sources: arrivals to arrival_out (nsrc x max_vertex, host).
static int bfs_multi_batch(GraphHandle& h, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                           int32_t* arrival_out) {
  const size_t nv = (size_t)h.view.max_vertex;
  const size_t qcap = nv + (size_t)h.nslices + 1;
  const size_t ndirty = (nv + 31) / 32;
  const size_t state = (size_t)nsrc * nv * 4;
  // s_a: arr | prev; s_b: F[0] | F[1]; s_c: dirty; s_q0/s_q1 queues; s_d: windows, sources and run table;
  // s_e: int32 output
  TGA_TRY(h.s_a.ensure(2 * state));
  TGA_TRY(h.s_b.ensure(2 * nv * kWords * 8));
  TGA_TRY(h.s_c.ensure(ndirty * 4));
  TGA_TRY(h.s_q0.ensure(qcap * 4));
  TGA_TRY(h.s_q1.ensure(qcap * 4));
  TGA_TRY(h.s_cnt.ensure(sizeof(TravCtl)));
  const size_t run_bytes = (size_t)std::max(h.nruns, 1) * kMaxSources * 4;
  TGA_TRY(h.s_d.ensure(kMaxSources * 20 + run_bytes));
  TGA_TRY(h.s_e.ensure(state));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  MultiArgs a{};
  a.w = Work{h.d_items.as<WorkItem>(), h.d_slices.as<SliceState>(), h.d_slice_first.as<int32_t>(), nullptr, h.nitems,
             h.d_order.as<int32_t>(), h.norder, nullptr};
  a.ctl = h.s_cnt.as<TravCtl>();
  a.q[0] = h.s_q0.as<int32_t>();
  a.q[1] = h.s_q1.as<int32_t>();
  a.arr = h.s_a.as<uint32_t>();
  a.prev = a.arr + (size_t)nsrc * nv;
  a.F[0] = h.s_b.as<uint64_t>();
  a.F[1] = a.F[0] + nv * kWords;
  a.dirty = h.s_c.as<uint32_t>();
  a.ndirty = (int32_t)ndirty;
  int64_t* dlo = h.s_d.as<int64_t>();
  int64_t* dhi = dlo + kMaxSources;
  int32_t* dsrc = reinterpret_cast<int32_t*>(dhi + kMaxSources);
  int32_t* drf = dsrc + kMaxSources;
  a.lo = dlo;
  a.hi = dhi;
  a.run_first = drf;
  a.nsrc = nsrc;
  a.nv = (int32_t)nv;
  a.dense_min = std::max<int32_t>(h.dense_min, 1);
  a.level_cap = 1 << 20;
  a.edges = edges;
  TGA_CUDA_TRY(cudaMemcpyAsync(dlo, t_lo, (size_t)nsrc * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dhi, t_hi, (size_t)nsrc * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dsrc, src, (size_t)nsrc * 4, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemsetAsync(a.arr, 0xFF, 2 * state, h.stream));
  TGA_CUDA_TRY(cudaMemsetAsync(a.F[0], 0, 2 * nv * kWords * 8, h.stream));
  TGA_CUDA_TRY(cudaMemsetAsync(a.dirty, 0, ndirty * 4, h.stream));
  TravCtl ctl{};
  std::memcpy(h.h_pinned + 32, &ctl, sizeof ctl);
  TGA_CUDA_TRY(cudaMemcpyAsync(a.ctl, h.h_pinned + 32, sizeof ctl, cudaMemcpyHostToDevice, h.stream));
  if (h.nruns > 0) {
    KL(k_fill_i32, grid_for((int64_t)h.nruns * kMaxSources, kBlock))(drf, INT32_MAX, (int64_t)h.nruns * kMaxSources);
    KL(k_run_first_multi, grid_for(h.nrun_pairs, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_runs.as<RunInfo>(),
                                                         h.d_run_pairs.as<int2>(), h.nrun_pairs, dlo, dhi, nsrc, drf);
  }
  KL(k_bfs_multi_seed, grid_for(nsrc, kBlock))(a, dsrc, h.view.n);
  int per_sm = 0;
  TGA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs_multi, kBlock, 0));
  if (per_sm < 1) return fail(TGA_E_CUDA, "batched traversal kernel cannot be resident");
  void* args[] = {&h.view, &a};
  cudaEvent_t* ev = h.kernel_begin();
  ++h.timing.launches;
  TGA_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_bfs_multi, dim3(per_sm * h.sm_count), dim3(kBlock), args, 0,
                                           h.stream));
  h.kernel_end(ev);
  TGA_CUDA_TRY(cudaMemcpyAsync(h.h_pinned + 32, a.ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  std::memcpy(&ctl, h.h_pinned + 32, sizeof ctl);
  if (ctl.status) return fail(TGA_E_TIMEOUT, "a grid barrier wait ran out");
  int32_t* out = h.s_e.as<int32_t>();
  KL(k_multi_unpack, grid_for((int64_t)nsrc * (int64_t)nv, kBlock))(a.arr, out, (int64_t)nsrc * (int64_t)nv);
  if (arrival_out) TGA_CUDA_TRY(cudaMemcpyAsync(arrival_out, out, state, cudaMemcpyDeviceToHost, h.stream));
  h.timing.iterations = ctl.levels;
  return finish(h, edges);
}

// ---------------------------------------------------------------------------------------------
// Multi-query PageRank: up to kMaxRankQueries windowed PageRanks as one strided vector
// (rank[v * kMaxRankQueries + q]), each list decoded once per iteration.  Per edge the temporal
// weight is computed once and the contribution scattered to every query whose window holds the
// edge (first in-window occurrence of equal consecutive successors per query, as tga_pagerank).

constexpr int kMaxRankQueries = 32;

struct PrMultiArgs {
  const float* invdeg;       // [nv][kMaxRankQueries] 1 / in-window outdegree (windowed queries)
  const int32_t* deg;        // outdegrees (other queries)
  const float* in;
  float* out;
  float* reset;
  const double* sums_prev;   // [kMaxRankQueries] sums of the previous iteration, or null
  const int64_t* lo;
  const int64_t* hi;
  const int32_t* run_first;  // [nruns][kMaxSources]
  uint32_t windowed;         // bit q: query q uses its in-window outdegree
  int32_t nq, nv;
  float damping, alpha, base;
  unsigned long long* edges;
};

__device__ __forceinline__ float temporal_weight_multi(float alpha, int64_t t) {
  const float a = alpha * (float)t;
  return a > 18.0f ? 1.0f : 1.0f - expf(-a);
}

__global__ void TGA_DECODE_BOUNDS k_pr_multi_iter(GraphView g, Work w, PrMultiArgs a) {
  __shared__ int64_t slo[kMaxRankQueries], shi[kMaxRankQueries];
  __shared__ float sinv[kMaxRankQueries];
  for (int q = threadIdx.x; q < kMaxRankQueries; q += blockDim.x) {
    slo[q] = q < a.nq ? a.lo[q] : 0;
    shi[q] = q < a.nq ? a.hi[q] : 0;
    sinv[q] = (q < a.nq && a.sums_prev) ? (float)(1.0 / a.sums_prev[q]) : 1.0f;
  }
  __syncthreads();
  const int64_t total = (int64_t)a.nv * kMaxRankQueries;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
    a.reset[i] = a.base;
  float c0[kMaxRankQueries];
  uint32_t act = 0, seen = 0;
  int yprev = -1;
  constexpr int kKeepSeen = -3;
  const unsigned long long mine = run_order<false, false, false, true, true>(
      g, w, [&](int v) { return v >= g.active_begin && v < g.max_label; },
      [&](int x, int first, int, int run) {
        act = 0;
        const float inv_all = a.deg[x] > 0 ? 1.0f / (float)a.deg[x] : 0.0f;
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q) {
          float c = 0.0f;
          if (q < a.nq) {
            const float inv = ((a.windowed >> q) & 1u) ? a.invdeg[(size_t)x * kMaxRankQueries + q] : inv_all;
            if (inv > 0.0f) c = a.damping * (a.in[(size_t)x * kMaxRankQueries + q] * sinv[q]) * inv;
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
          atomicAdd(&a.out[(size_t)y * kMaxRankQueries + q], c0[q] * wgt);
        }
        return true;
      },
      [](int) {});
  add_edges(a.edges, mine);
}

// In-window outdegree per query (lists counted by slices), then 1/count.
__global__ void TGA_DECODE_BOUNDS k_window_count_multi(GraphView g, Work w, const int64_t* lo, const int64_t* hi,
                                                     int32_t nq, int32_t* cnt, unsigned long long* edges) {
  __shared__ int64_t slo[kMaxRankQueries], shi[kMaxRankQueries];
  for (int q = threadIdx.x; q < kMaxRankQueries; q += blockDim.x) {
    slo[q] = q < nq ? lo[q] : 0;
    shi[q] = q < nq ? hi[q] : 0;
  }
  __syncthreads();
  int k[kMaxRankQueries];
  const unsigned long long mine = run_order<false>(
      g, w, [&](int v) { return v >= g.active_begin && v < g.max_label; },
      [&](int, int, int) {
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q) k[q] = 0;
        return true;
      },
      [&](int, int, int64_t t) {
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q) k[q] += (t >= slo[q] && t < shi[q]);
        return true;
      },
      [&](int v) {
#pragma unroll
        for (int q = 0; q < kMaxRankQueries; ++q)
          if (q < nq && k[q]) atomicAdd(&cnt[(size_t)v * kMaxRankQueries + q], k[q]);
      });
  add_edges(edges, mine);
}

__global__ void k_invert_multi(const int32_t* cnt, float* inv, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) inv[i] = cnt[i] ? 1.0f / (float)cnt[i] : 0.0f;
}

// sums[q] = sum over v of buf[v][q] (FP64), one block per query.
__global__ void k_sums_multi(const float* buf, int32_t nv, double* sums) {
  const int q = blockIdx.x;
  double s = 0.0;
  for (int v = threadIdx.x; v < nv; v += blockDim.x) s += (double)buf[(size_t)v * kMaxRankQueries + q];
  const double bs = block_sum(s);
  if (threadIdx.x == 0) sums[q] = bs;
}

__global__ void k_pr_multi_final(const float* buf, const double* sums, int32_t nq, int32_t nv, float* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nq * nv) return;
  const int q = (int)(i / nv), v = (int)(i % nv);
  out[i] = (float)((double)buf[(size_t)v * kMaxRankQueries + q] / sums[q]);
}

static int pagerank_multi_batch(GraphHandle& h, int32_t nq, int32_t iters, float damping, float alpha,
                                const int64_t* t_lo, const int64_t* t_hi, float* rank_out) {
  const size_t nv = (size_t)h.view.max_vertex;
  const size_t vec = nv * kMaxRankQueries;
  // s_a: 3 rank buffers | invdeg; s_b: counts; s_d: windows + sums + run table; s_e: output
  TGA_TRY(h.s_a.ensure(vec * 4 * 4));
  TGA_TRY(h.s_b.ensure(vec * 4));
  const size_t run_bytes = (size_t)std::max(h.nruns, 1) * kMaxSources * 4;
  const size_t sums_off = kMaxSources * 16;
  TGA_TRY(h.s_d.ensure(sums_off + (size_t)(iters + 1) * kMaxRankQueries * 8 + run_bytes));
  TGA_TRY(h.s_e.ensure((size_t)nq * nv * 4));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  float* bufs[3] = {h.s_a.as<float>(), h.s_a.as<float>() + vec, h.s_a.as<float>() + 2 * vec};
  float* invdeg = h.s_a.as<float>() + 3 * vec;
  int32_t* cnt = h.s_b.as<int32_t>();
  int64_t* dlo = h.s_d.as<int64_t>();
  int64_t* dhi = dlo + kMaxSources;
  double* sums = reinterpret_cast<double*>(h.s_d.as<char>() + sums_off);
  int32_t* drf = reinterpret_cast<int32_t*>(sums + (size_t)(iters + 1) * kMaxRankQueries);
  TGA_CUDA_TRY(cudaMemcpyAsync(dlo, t_lo, (size_t)nq * 8, cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(dhi, t_hi, (size_t)nq * 8, cudaMemcpyHostToDevice, h.stream));
  uint32_t windowed = 0;
  for (int q = 0; q < nq; ++q)
    if (!(t_lo[q] <= 0 && t_hi[q] == TGA_T_MAX)) windowed |= 1u << q;
  if (h.nruns > 0) {
    KL(k_fill_i32, grid_for((int64_t)h.nruns * kMaxSources, kBlock))(drf, INT32_MAX, (int64_t)h.nruns * kMaxSources);
    KL(k_run_first_multi, grid_for(h.nrun_pairs, kBlock))(h.view, h.d_slices.as<SliceState>(), h.d_runs.as<RunInfo>(),
                                                         h.d_run_pairs.as<int2>(), h.nrun_pairs, dlo, dhi, nq, drf);
  }
  const float base = (1.0f - damping) / (float)h.view.max_label;
  KL(k_fill_f32, grid_for((int64_t)vec, kBlock))(bufs[0], 1.0f / (float)nv, (int64_t)vec);
  KL(k_fill_f32, grid_for((int64_t)vec, kBlock))(bufs[1], base, (int64_t)vec);
  if (windowed) {
    TGA_CUDA_TRY(cudaMemsetAsync(cnt, 0, vec * 4, h.stream));
    const Work w = work_of(h);
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_window_count_multi, sweep_grid(h))(h.view, w, dlo, dhi, nq, cnt, edges);
    h.kernel_end(ev);
    KL(k_invert_multi, grid_for((int64_t)vec, kBlock))(cnt, invdeg, (int64_t)vec);
  }
  for (int k = 0; k < iters; ++k) {
    Work w = work_of(h);
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
    a.nq = nq;
    a.nv = (int32_t)nv;
    a.damping = damping;
    a.alpha = alpha;
    a.base = base;
    a.edges = edges;
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_pr_multi_iter, sweep_grid(h))(h.view, w, a);
    h.kernel_end(ev);
    k_sums_multi<<<nq, kBlock, 0, h.stream>>>(a.out, (int32_t)nv, sums + (size_t)k * kMaxRankQueries);
    ++h.timing.launches;
  }
  float* out = h.s_e.as<float>();
  KL(k_pr_multi_final, grid_for((int64_t)nq * (int64_t)nv, kBlock))(bufs[iters % 3],
                                                                    sums + (size_t)(iters - 1) * kMaxRankQueries, nq,
                                                                    (int32_t)nv, out);
  if (rank_out) TGA_CUDA_TRY(cudaMemcpyAsync(rank_out, out, (size_t)nq * nv * 4, cudaMemcpyDeviceToHost, h.stream));
  h.timing.iterations = iters;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(iters + (windowed ? 1 : 0)) *
                              (h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes);
  return rc;
}

}  // namespace tga

using namespace tga;

extern "C" {

int tga_bfs_batch(tga_graph* g, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                  int32_t* arrival_out) {
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

int tga_pagerank_batch(tga_graph* g, int32_t nq, int32_t iters, float damping, float alpha, const int64_t* t_lo,
                       const int64_t* t_hi, float* rank_out) {
  if (!g || nq < 0 || (nq && (!t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  GraphHandle& h = *g;
  if (iters <= 0) iters = h.cfg.pr_iters;
  for (int32_t i = 0; i < nq; ++i)
    if (t_lo[i] >= t_hi[i]) return fail(TGA_E_ARG, "empty time window");
  const size_t nv = (size_t)h.view.max_vertex;
  tga_timing total{};
  for (int32_t b = 0; b < nq; b += kMaxRankQueries) {
    const int32_t k = std::min(kMaxRankQueries, nq - b);
    const int rc = pagerank_multi_batch(h, k, iters, damping, alpha, t_lo + b, t_hi + b,
                                        rank_out ? rank_out + (size_t)b * nv : nullptr);
    if (rc) return rc;
    total.total_ms += h.timing.total_ms;
    total.decode_ms += h.timing.decode_ms;
    total.decode_launches += h.timing.decode_launches;
    total.edges_decoded += h.timing.edges_decoded;
    total.compressed_bytes += h.timing.compressed_bytes;
    total.iterations = h.timing.iterations;
    total.launches += h.timing.launches;
  }
  h.timing = total;
  return TGA_OK;
}

}  // extern "C"
