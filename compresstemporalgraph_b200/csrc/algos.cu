// Fused decode + algorithm kernels and their C ABI entry points.  Every kernel decodes the
// successor lists and timestamps it needs straight from the compressed streams; decoded edges
// live only in registers.
#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "decoder.cuh"
#include "engine.hpp"

namespace tga {

constexpr int kBlock = 256;
// Launches a kernel of kBlock threads on the handle's stream and counts it in the call's timing.
#define KL(kernel, grid) ++h.timing.launches, kernel<<<(grid), kBlock, 0, h.stream>>>
constexpr uint64_t kTpInf = ~0ull;
constexpr uint32_t kColorInf = 0xFFFFFFFFu;

// Order-sensitive hash of a successor list, also computed by the oracle.
__host__ __device__ __forceinline__ uint64_t mix_edge(uint64_t h, int32_t y, int64_t t) {
  const uint64_t k = ((uint64_t)(uint32_t)y * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)t * 0xC2B2AE3D27D4EB4Full);
  h ^= k;
  h = (h << 23) | (h >> 41);
  return h * 0x165667B19E3779F9ull;
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

// ---------------------------------------------------------------------------------------------
// Neighbour access and raw decode

__global__ void __launch_bounds__(kBlock) k_neighbor_access(GraphView g, int32_t begin, int32_t end, uint8_t* small,
                                                            uint64_t* csum, unsigned long long* edges) {
  const int x = begin + blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  if (x < end) {
    EdgeCursor c;
    const int d = c.open(g, x);
    small[x] = d < 4;
    uint64_t h = 0x27D4EB2F165667C5ull ^ (uint64_t)(uint32_t)x;
    int y;
    int64_t t;
    while (c.next(g, y, t)) h = mix_edge(h, y, t);
    csum[x] = h;
    mine = (unsigned long long)d;
  }
  add_edges(edges, mine);
}

__global__ void k_decode_csr(GraphView g, int32_t count, const int64_t* off, int32_t* dst, int64_t* ts, int64_t cap) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= count) return;
  EdgeCursor c;
  c.open(g, x);
  int64_t o = off[x];
  int y;
  int64_t t;
  while (c.next(g, y, t)) {
    if (o < cap) { dst[o] = y; ts[o] = t; }
    ++o;
  }
}

__global__ void k_neighbors(GraphView g, int32_t v, int32_t* dst, int64_t* ts, int32_t cap, int32_t* count) {
  EdgeCursor c;
  const int d = c.open(g, v);
  int i = 0, y;
  int64_t t;
  while (c.next(g, y, t)) {
    if (i < cap) { dst[i] = y; ts[i] = t; }
    ++i;
  }
  *count = d;
}

// ---------------------------------------------------------------------------------------------
// Temporal BFS (label-correcting, packed (arrival << 32 | hops) relaxation)

struct BfsArgs {
  const int32_t* q;
  int32_t* nq;
  int32_t* ncnt;
  uint64_t* tp;
  uint32_t* stamp;
  uint32_t wave;
  int64_t lo, hi;
  int32_t* touched;     // optional: vertices whose arrival became finite (CC)
  int32_t* tcnt;
  unsigned long long* edges;
};

__global__ void __launch_bounds__(kBlock) k_bfs_level(GraphView g, BfsArgs a, int32_t qn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  if (i < qn) {
    const int x = a.q[i];
    if (x >= g.active_begin && x <= g.max_label) {
      const uint64_t wx = a.tp[x];
      const uint32_t ax = (uint32_t)(wx >> 32), hx = (uint32_t)wx;
      EdgeCursor c;
      mine = (unsigned long long)c.open(g, x);
      int y, prev_y = -1;
      int64_t t;
      while (c.next(g, y, t)) {
        if (t < a.lo || t >= a.hi) continue;
        if (y == prev_y) continue;
        prev_y = y;
        if (y < g.active_begin || y >= g.max_vertex) continue;
        if ((int64_t)ax > t || t >= 0xFFFFFFFFll) continue;
        const uint64_t nv = ((uint64_t)t << 32) | (uint64_t)(hx + 1);
        const uint64_t old = atomicMin((unsigned long long*)&a.tp[y], (unsigned long long)nv);
        if (nv < old) {
          if (a.touched && (old >> 32) == 0xFFFFFFFFull) a.touched[atomicAdd(a.tcnt, 1)] = y;
          if (atomicMax(&a.stamp[y], a.wave) < a.wave) a.nq[atomicAdd(a.ncnt, 1)] = y;
        }
      }
    }
  }
  add_edges(a.edges, mine);
}

__global__ void k_fill_u64(uint64_t* p, uint64_t v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
__global__ void k_fill_f32(float* p, float v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
__global__ void k_fill_i32(int32_t* p, int32_t v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void k_unpack_tp(const uint64_t* tp, int32_t* arr, int32_t* hops, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t w = tp[i];
  const bool inf = (w >> 32) == 0xFFFFFFFFull;
  arr[i] = inf ? INT32_MAX : (int32_t)(w >> 32);
  hops[i] = inf ? INT32_MAX : (int32_t)(uint32_t)w;
}

// Runs the level loop from an initialised frontier; returns levels executed or <0 on error.
static int run_bfs_levels(GraphHandle& h, BfsArgs a, DevBuf& q0, DevBuf& q1, int32_t qn, uint32_t& wave, int& rc) {
  int levels = 0;
  DevBuf* cur = &q0;
  DevBuf* nxt = &q1;
  rc = TGA_OK;
  while (qn > 0) {
    if (levels > 1 << 22) { rc = fail(TGA_E_TIMEOUT, "BFS level cap reached"); return levels; }
    a.q = cur->as<int32_t>();
    a.nq = nxt->as<int32_t>();
    a.wave = ++wave;
    cudaMemsetAsync(a.ncnt, 0, sizeof(int32_t), h.stream);
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_bfs_level, grid_for(qn, kBlock))(h.view, a, qn);
    h.kernel_end(ev);
    cudaMemcpyAsync(h.h_pinned, a.ncnt, sizeof(int32_t), cudaMemcpyDeviceToHost, h.stream);
    if (cudaStreamSynchronize(h.stream) != cudaSuccess) { rc = fail(TGA_E_CUDA, "BFS level failed"); return levels; }
    qn = (int32_t)h.h_pinned[0];
    std::swap(cur, nxt);
    ++levels;
  }
  return levels;
}

static int bfs_buffers(GraphHandle& h) {
  const size_t nv = (size_t)h.view.max_vertex;
  int rc;
  if ((rc = h.s_a.ensure(nv * 8)) || (rc = h.s_b.ensure(nv * 4)) || (rc = h.s_q0.ensure(nv * 4)) ||
      (rc = h.s_q1.ensure(nv * 4)) || (rc = h.s_cnt.ensure(64)) || (rc = h.s_c.ensure(nv * 4)))
    return rc;
  return TGA_OK;
}

// ---------------------------------------------------------------------------------------------
// Connected components (per-seed temporal reach)

__global__ void k_cc_label(const int32_t* touched, const int32_t* tcnt, int32_t seed, int32_t comp, uint64_t* tp,
                           int32_t* label, uint8_t* reached) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *tcnt;
  if (i < n) {
    const int y = touched[i];
    label[y] = comp;
    reached[y] = 1;
    tp[y] = kTpInf;
  }
  if (i == 0) {
    label[seed] = comp;
    reached[seed] = 1;
    tp[seed] = kTpInf;
  }
}

__global__ void k_cc_find_seed(const uint8_t* reached, const int32_t* deg, int32_t from, int32_t to, int32_t* best) {
  const int v = from + blockIdx.x * blockDim.x + threadIdx.x;
  if (v < to && !reached[v] && deg[v] > 9) atomicMin(best, v);
}

// ---------------------------------------------------------------------------------------------
// PageRank

struct PrArgs {
  const float* invdeg;   // per-vertex 1/deg for a window, or nullptr (use outdegree)
  const int32_t* deg;
  float* in;
  float* out;
  double* sums;
  int32_t k;
  float damping, alpha, base;
  int64_t lo, hi;
  unsigned long long* edges;
};

__global__ void __launch_bounds__(kBlock) k_pr_iter(GraphView g, PrArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  double local = 0;
  unsigned long long mine = 0;
  if (x < g.max_vertex) {
    const double s = a.k == 0 ? 1.0 : 1.0 / a.sums[a.k - 1];
    const float r = (float)((double)a.in[x] * s);
    a.in[x] = a.base;
    if (x >= g.active_begin && x < g.max_label) {
      const int d = a.deg[x];
      const float inv = a.invdeg ? a.invdeg[x] : (d > 0 ? 1.0f / (float)d : 0.0f);
      if (d > 0 && inv > 0.0f) {
        const float c0 = a.damping * r * inv;
        EdgeCursor c;
        mine = (unsigned long long)c.open(g, x);
        int y, prev_y = -1;
        int64_t t;
        while (c.next(g, y, t)) {
          if (t < a.lo || t >= a.hi) continue;
          if (y == prev_y) continue;
          prev_y = y;
          if (y < g.active_begin || y >= g.max_vertex) continue;
          const float contrib = c0 * (1.0f - expf(-a.alpha * (float)t));
          atomicAdd(&a.out[y], contrib);
          local += contrib;
        }
      }
    }
  }
  add_edges(a.edges, mine);
  const double bs = block_sum(local);
  if (threadIdx.x == 0 && bs != 0.0) atomicAdd(&a.sums[a.k], bs);
}

__global__ void k_pr_init_sums(double* sums, int n, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sums[i] = v;
}

__global__ void k_pr_final(const float* buf, const double* sums, int k, float* out, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)((double)buf[i] / sums[k]);
}

// In-window outdegree of each source (timestamps only need decoding, ids come along).
__global__ void __launch_bounds__(kBlock) k_window_invdeg(GraphView g, int64_t lo, int64_t hi, float* invdeg,
                                                          unsigned long long* edges) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  if (x < g.max_vertex) {
    int cnt = 0;
    if (x >= g.active_begin && x < g.max_label) {
      EdgeCursor c;
      mine = (unsigned long long)c.open(g, x);
      int y;
      int64_t t;
      while (c.next(g, y, t)) cnt += (t >= lo && t < hi);
    }
    invdeg[x] = cnt ? 1.0f / (float)cnt : 0.0f;
  }
  add_edges(edges, mine);
}

// ---------------------------------------------------------------------------------------------
// HITS

struct HitsArgs {
  float* hub;
  const float* auth_in;   // current authority, not yet normalised
  float* auth_next;       // receives the base of the next authority, then the scatter
  double* hsum;           // sum of hub^2 of this iteration (accumulated by the hub kernel)
  const double* aprev;    // sum of auth^2 of the previous iteration (nullptr: scale 1)
  int java;
  int64_t lo, hi;
  unsigned long long* edges;
};

__global__ void __launch_bounds__(kBlock) k_hits_hub(GraphView g, HitsArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  double local = 0;
  unsigned long long mine = 0;
  if (x < g.max_vertex) {
    const double sa = (a.aprev && *a.aprev > 0) ? 1.0 / sqrt(*a.aprev) : 1.0;
    const float sf = (float)sa;
    float h = a.java ? 0.0f : a.hub[x];
    if (x >= g.active_begin && x < g.max_label) {
      EdgeCursor c;
      mine = (unsigned long long)c.open(g, x);
      int y, prev_y = -1;
      int64_t t;
      float acc = 0.0f;
      while (c.next(g, y, t)) {
        if (t < a.lo || t >= a.hi) continue;
        if (y == prev_y) continue;
        prev_y = y;
        if (y < g.active_begin || y >= g.max_vertex) continue;
        acc += a.auth_in[y];
      }
      h += acc * sf;
    }
    a.hub[x] = h;
    a.auth_next[x] = a.java ? 0.0f : a.auth_in[x] * sf;
    local = (double)h * (double)h;
  }
  add_edges(a.edges, mine);
  const double bs = block_sum(local);
  if (threadIdx.x == 0 && bs != 0.0) atomicAdd(a.hsum, bs);
}

__global__ void __launch_bounds__(kBlock) k_hits_auth(GraphView g, HitsArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  if (x < g.max_vertex) {
    const double sh = *a.hsum > 0 ? 1.0 / sqrt(*a.hsum) : 1.0;
    const float hn = (float)((double)a.hub[x] * sh);
    a.hub[x] = hn;
    if (x >= g.active_begin && x < g.max_label && hn != 0.0f) {
      EdgeCursor c;
      mine = (unsigned long long)c.open(g, x);
      int y, prev_y = -1;
      int64_t t;
      while (c.next(g, y, t)) {
        if (t < a.lo || t >= a.hi) continue;
        if (y == prev_y) continue;
        prev_y = y;
        if (y < g.active_begin || y >= g.max_vertex) continue;
        atomicAdd(&a.auth_next[y], hn);
      }
    }
  }
  add_edges(a.edges, mine);
}

__global__ void k_sumsq(const float* v, int32_t n, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double x = i < n ? (double)v[i] : 0.0;
  const double bs = block_sum(x * x);
  if (threadIdx.x == 0 && bs != 0.0) atomicAdd(out, bs);
}

__global__ void k_scale(const float* v, const double* sumsq, float* out, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = *sumsq > 0 ? 1.0 / sqrt(*sumsq) : 1.0;
  out[i] = (float)((double)v[i] * s);
}

// ---------------------------------------------------------------------------------------------
// Degree centrality (Java semantics)

__global__ void __launch_bounds__(kBlock) k_degree(GraphView g, int64_t s, int64_t e, int32_t* deg, int64_t* avg,
                                                   unsigned long long* edges) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  if (x < g.max_vertex) {
    int32_t d = 0;
    int64_t mean = 0;
    if (x >= g.active_begin && x <= g.max_label) {
      const bool all = (s == 0 && e == 0);
      const int lim = min(g.max_label + 1, g.max_vertex);
      EdgeCursor c;
      mine = (unsigned long long)c.open(g, x);
      int y;
      int64_t t;
      while (c.next(g, y, t)) {
        if (y < g.active_begin || y >= lim) continue;
        if (all || (s <= t && e >= t)) {
          ++d;
          mean += (t - mean) / d;
        }
      }
      if (s != e) d = (int32_t)(0.85 * d + 0.15 * d * (double)(mean - s) / (double)(e - s) + 1);
    }
    deg[x] = d;
    avg[x] = mean;
  }
  add_edges(edges, mine);
}

// ---------------------------------------------------------------------------------------------
// Jones-Plassmann colouring

__global__ void k_gc_prio_curand(uint32_t* prio, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  curandState st;
  curand_init(123ull, (unsigned long long)i, 0ull, &st);
  prio[i] = curand(&st) % 256u;
}

__global__ void __launch_bounds__(kBlock) k_gc_round(GraphView g, const int32_t* wl, int32_t wn, int32_t* out_wl,
                                                     int32_t* out_n, uint32_t* color, const uint32_t* prio, uint32_t round,
                                                     int java_isolated, unsigned long long* edges) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = 0;
  if (i < wn) {
    const int x = wl[i];
    if (x >= g.active_begin && color[x] == kColorInf && x <= g.max_label) {
      EdgeCursor c;
      const int d = c.open(g, x);
      if (d == 0) {
        if (java_isolated) color[x] = round;
      } else {
        const uint32_t px = prio[x];
        bool larger = false;
        int y, prev_y = -1;
        int64_t t;
        int seen = 0;
        while (c.next(g, y, t)) {
          ++seen;
          if (y == prev_y) continue;
          prev_y = y;
          if (y < g.active_begin || y >= g.max_vertex) continue;
          const uint32_t py = prio[y];
          if ((py > px || (py == px && y < x)) && color[y] >= round) {
            larger = true;
            break;
          }
        }
        mine = (unsigned long long)seen;
        if (larger) out_wl[atomicAdd(out_n, 1)] = x;
        else color[x] = round;
      }
    }
  }
  add_edges(edges, mine);
}

__global__ void k_iota(int32_t* p, int32_t n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

}  // namespace tga

using namespace tga;

// ---------------------------------------------------------------------------------------------
// C ABI

#define TGA_TRY(expr)            \
  do {                           \
    int rc_ = (expr);            \
    if (rc_) return rc_;         \
  } while (0)

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

extern "C" {

int tga_neighbor_access(tga_graph* gp, uint8_t* small_out, uint64_t* checksum_out, int32_t* degree_out) {
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
    KL(k_neighbor_access, grid_for(e - b, kBlock))(h.view, b, e, h.s_a.as<uint8_t>(),
                                                                        h.s_b.as<uint64_t>(), edges);
    h.kernel_end(ev);
  }
  if (small_out) cudaMemcpyAsync(small_out, h.s_a.p, (size_t)nv, cudaMemcpyDeviceToHost, h.stream);
  if (checksum_out) cudaMemcpyAsync(checksum_out, h.s_b.p, (size_t)nv * 8, cudaMemcpyDeviceToHost, h.stream);
  if (degree_out) cudaMemcpyAsync(degree_out, h.d_deg.p, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = 1;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes;
  return rc;
}

int tga_neighbors(tga_graph* gp, int32_t v, int32_t* dst, int64_t* ts, int32_t cap, int32_t* count) {
  if (!gp || !count) return fail(TGA_E_ARG, "null argument");
  GraphHandle& h = *gp;
  if (v < 0 || v >= h.view.n) return fail(TGA_E_ARG, "vertex out of range");
  if (cap < 0) cap = 0;
  TGA_TRY(h.s_c.ensure((size_t)cap * 4 + 64));
  TGA_TRY(h.s_d.ensure((size_t)cap * 8 + 64));
  TGA_TRY(h.s_cnt.ensure(64));
  TGA_TRY(h.begin_call());
  ++h.timing.launches, k_neighbors<<<1, 1, 0, h.stream>>>(h.view, v, h.s_c.as<int32_t>(), h.s_d.as<int64_t>(), cap, h.s_cnt.as<int32_t>());
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

int tga_decode_all(tga_graph* gp, int64_t* offsets, int32_t* dst, int64_t* ts, int64_t cap) {
  if (!gp || !offsets) return fail(TGA_E_ARG, "null argument");
  GraphHandle& h = *gp;
  const int32_t n = h.view.n;
  const int32_t nd = std::min(n, h.view.max_vertex);
  std::vector<int32_t> deg((size_t)nd);
  TGA_CUDA_TRY(cudaMemcpy(deg.data(), h.d_deg.p, (size_t)nd * 4, cudaMemcpyDeviceToHost));
  offsets[0] = 0;
  for (int32_t v = 0; v < n; ++v) offsets[v + 1] = offsets[v] + (v < nd ? deg[(size_t)v] : 0);
  const int64_t m = offsets[n];
  if (!dst || !ts) return TGA_OK;  // size query
  if (cap < m) return fail(TGA_E_ARG, "capacity below the number of edges");
  TGA_TRY(h.s_e.ensure((size_t)(n + 1) * 8));
  TGA_TRY(h.s_f.ensure((size_t)std::max<int64_t>(m, 1) * 4));
  TGA_TRY(h.s_g.ensure((size_t)std::max<int64_t>(m, 1) * 8));
  TGA_CUDA_TRY(cudaMemcpy(h.s_e.p, offsets, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice));
  TGA_TRY(h.begin_call());
  KL(k_decode_csr, grid_for(nd, kBlock))(h.view, nd, h.s_e.as<int64_t>(), h.s_f.as<int32_t>(),
                                                               h.s_g.as<int64_t>(), m);
  cudaMemcpyAsync(dst, h.s_f.p, (size_t)m * 4, cudaMemcpyDeviceToHost, h.stream);
  cudaMemcpyAsync(ts, h.s_g.p, (size_t)m * 8, cudaMemcpyDeviceToHost, h.stream);
  return h.end_call();
}

int tga_bfs(tga_graph* gp, int32_t src, int64_t t_lo, int64_t t_hi, int32_t* arrival_out, int32_t* hops_out) {
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (src < 0) src = h.cfg.bfs_start_vertex;
  if (src < 0 || src >= h.view.max_vertex) return fail(TGA_E_ARG, "source out of range");
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(bfs_buffers(h));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  BfsArgs a{};
  a.tp = h.s_a.as<uint64_t>();
  a.stamp = h.s_b.as<uint32_t>();
  a.ncnt = h.s_cnt.as<int32_t>();
  a.lo = t_lo;
  a.hi = t_hi;
  a.edges = edges;
  KL(k_fill_u64, grid_for(nv, kBlock))(a.tp, kTpInf, nv);
  cudaMemsetAsync(a.stamp, 0, (size_t)nv * 4, h.stream);
  const uint64_t start = (uint64_t)std::max<int64_t>(t_lo, 0) << 32;
  cudaMemcpyAsync(a.tp + src, &start, 8, cudaMemcpyHostToDevice, h.stream);
  cudaMemcpyAsync(h.s_q0.p, &src, 4, cudaMemcpyHostToDevice, h.stream);
  uint32_t wave = 0;
  int rc = TGA_OK;
  const int levels = run_bfs_levels(h, a, h.s_q0, h.s_q1, 1, wave, rc);
  if (rc) return rc;
  int32_t* arr = h.s_q0.as<int32_t>();
  int32_t* hops = h.s_q1.as<int32_t>();
  KL(k_unpack_tp, grid_for(nv, kBlock))(a.tp, arr, hops, nv);
  if (arrival_out) cudaMemcpyAsync(arrival_out, arr, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (hops_out) cudaMemcpyAsync(hops_out, hops, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = levels;
  return finish(h, edges);
}

int tga_cc(tga_graph* gp, int64_t t_lo, int64_t t_hi, int32_t flags, int32_t* label_out, int32_t* components_out) {
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(bfs_buffers(h));
  TGA_TRY(h.s_d.ensure((size_t)nv * 4));   // labels
  TGA_TRY(h.s_e.ensure((size_t)nv));       // reached
  TGA_TRY(h.s_f.ensure((size_t)nv * 4));   // touched list
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  BfsArgs a{};
  a.tp = h.s_a.as<uint64_t>();
  a.stamp = h.s_b.as<uint32_t>();
  a.ncnt = h.s_cnt.as<int32_t>();
  a.tcnt = h.s_cnt.as<int32_t>() + 4;
  a.touched = h.s_f.as<int32_t>();
  int32_t* best = h.s_cnt.as<int32_t>() + 8;
  a.lo = t_lo;
  a.hi = t_hi;
  a.edges = edges;
  int32_t* label = h.s_d.as<int32_t>();
  uint8_t* reached = h.s_e.as<uint8_t>();
  KL(k_fill_u64, grid_for(nv, kBlock))(a.tp, kTpInf, nv);
  KL(k_fill_i32, grid_for(nv, kBlock))(label, -1, nv);
  cudaMemsetAsync(a.stamp, 0, (size_t)nv * 4, h.stream);
  cudaMemsetAsync(reached, 0, (size_t)nv, h.stream);
  const int32_t limit = (int32_t)(0.8 * h.view.max_label);
  const int32_t end = std::min(h.view.max_label, nv);
  int64_t total = 0;
  int small_run = 0, comp = 0, levels = 0;
  uint32_t wave = 0;
  int32_t v = std::max(h.cfg.cc_vertex_begin, 0);
  const uint64_t start = (uint64_t)std::max<int64_t>(t_lo, 0) << 32;
  while (v < end) {
    if ((flags & TGA_CC_EARLY_EXIT) && total > limit) break;
    // Next seed: smallest unreached vertex >= v with outdegree > 9, searched in growing chunks.
    int32_t seed = INT32_MAX;
    for (int32_t from = v, chunk = 4096; from < end && seed == INT32_MAX; from += chunk, chunk *= 2) {
      const int32_t to = (int32_t)std::min<int64_t>((int64_t)from + chunk, end);
      h.h_pinned[20] = INT32_MAX;
      cudaMemcpyAsync(best, &h.h_pinned[20], 4, cudaMemcpyHostToDevice, h.stream);
      KL(k_cc_find_seed, grid_for(to - from, kBlock))(reached, h.d_deg.as<int32_t>(), from, to, best);
      cudaMemcpyAsync(&h.h_pinned[21], best, 4, cudaMemcpyDeviceToHost, h.stream);
      TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
      seed = (int32_t)h.h_pinned[21];
    }
    if (seed == INT32_MAX) break;
    h.h_pinned[22] = 0;
    cudaMemcpyAsync(a.tcnt, &h.h_pinned[22], 4, cudaMemcpyHostToDevice, h.stream);
    cudaMemcpyAsync(a.tp + seed, &start, 8, cudaMemcpyHostToDevice, h.stream);
    cudaMemcpyAsync(h.s_q0.p, &seed, 4, cudaMemcpyHostToDevice, h.stream);
    int rc = TGA_OK;
    levels += run_bfs_levels(h, a, h.s_q0, h.s_q1, 1, wave, rc);
    if (rc) return rc;
    cudaMemcpyAsync(&h.h_pinned[23], a.tcnt, 4, cudaMemcpyDeviceToHost, h.stream);
    TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
    const int32_t reach = (int32_t)h.h_pinned[23];
    KL(k_cc_label, grid_for(std::max(reach, 1), kBlock))(a.touched, a.tcnt, seed, comp, a.tp,
                                                                             label, reached);
    ++comp;
    total += reach + 1;
    if (reach + 1 < 5) ++small_run;
    else small_run = 0;
    if ((flags & TGA_CC_EARLY_EXIT) && small_run > 50) break;
    v = seed + 1;
  }
  if (label_out) cudaMemcpyAsync(label_out, label, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (components_out) *components_out = comp;
  h.timing.iterations = levels;
  return finish(h, edges);
}

int tga_pagerank(tga_graph* gp, int32_t iters, float damping, float alpha, int64_t t_lo, int64_t t_hi, float* rank_out) {
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (iters <= 0) iters = h.cfg.pr_iters;
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  const bool windowed = !(t_lo <= 0 && t_hi == TGA_T_MAX);
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));
  TGA_TRY(h.s_b.ensure((size_t)nv * 4));
  TGA_TRY(h.s_c.ensure((size_t)nv * 4));
  TGA_TRY(h.s_g.ensure((size_t)(iters + 1) * 8));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  const float base = (1.0f - damping) / (float)h.view.max_label;
  float* bufs[2] = {h.s_a.as<float>(), h.s_b.as<float>()};
  double* sums = h.s_g.as<double>();
  KL(k_fill_f32, grid_for(nv, kBlock))(bufs[0], 1.0f / (float)nv, nv);
  KL(k_fill_f32, grid_for(nv, kBlock))(bufs[1], base, nv);
  KL(k_pr_init_sums, grid_for(iters, kBlock))(sums, iters, (double)base * (double)nv);
  float* invdeg = nullptr;
  if (windowed) {
    invdeg = h.s_c.as<float>();
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_window_invdeg, grid_for(nv, kBlock))(h.view, t_lo, t_hi, invdeg, edges);
    h.kernel_end(ev);
  }
  for (int k = 0; k < iters; ++k) {
    PrArgs a{invdeg, h.d_deg.as<int32_t>(), bufs[k & 1], bufs[(k + 1) & 1], sums, k, damping, alpha, base, t_lo, t_hi, edges};
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_pr_iter, grid_for(nv, kBlock))(h.view, a);
    h.kernel_end(ev);
  }
  float* out = bufs[iters & 1];
  float* fin = h.s_c.as<float>();
  KL(k_pr_final, grid_for(nv, kBlock))(out, sums, iters - 1, fin, nv);
  if (rank_out) cudaMemcpyAsync(rank_out, fin, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = iters;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(iters + (windowed ? 1 : 0)) * (h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes);
  return rc;
}

int tga_hits(tga_graph* gp, int32_t iters, int32_t mode, int64_t t_lo, int64_t t_hi, float* hub_out, float* auth_out) {
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  if (iters <= 0) iters = h.cfg.hits_iters;
  if (mode != TGA_HITS_GPU && mode != TGA_HITS_JAVA) return fail(TGA_E_ARG, "unknown HITS mode");
  if (t_lo >= t_hi) return fail(TGA_E_ARG, "empty time window");
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));
  TGA_TRY(h.s_b.ensure((size_t)nv * 4));
  TGA_TRY(h.s_c.ensure((size_t)nv * 4));
  TGA_TRY(h.s_g.ensure((size_t)(2 * iters + 2) * 8));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  float* hub = h.s_a.as<float>();
  float* auth[2] = {h.s_b.as<float>(), h.s_c.as<float>()};
  double* sums = h.s_g.as<double>();
  KL(k_fill_f32, grid_for(nv, kBlock))(hub, 1.0f, nv);
  KL(k_fill_f32, grid_for(nv, kBlock))(auth[0], 1.0f, nv);
  cudaMemsetAsync(sums, 0, (size_t)(2 * iters + 2) * 8, h.stream);
  // sums[2k] = sum hub^2 of iteration k, sums[2k+1] = sum auth^2 of iteration k.
  for (int k = 0; k < iters; ++k) {
    HitsArgs a{};
    a.hub = hub;
    a.auth_in = auth[k & 1];
    a.auth_next = auth[(k + 1) & 1];
    a.hsum = sums + 2 * k;
    a.aprev = k == 0 ? nullptr : sums + 2 * k - 1;
    a.java = mode == TGA_HITS_JAVA;
    a.lo = t_lo;
    a.hi = t_hi;
    a.edges = edges;
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_hits_hub, grid_for(nv, kBlock))(h.view, a);
    h.kernel_end(ev);
    ev = h.kernel_begin();
    KL(k_hits_auth, grid_for(nv, kBlock))(h.view, a);
    h.kernel_end(ev);
    KL(k_sumsq, grid_for(nv, kBlock))(a.auth_next, nv, sums + 2 * k + 1);
  }
  float* hub_fin = hub;
  float* auth_fin = auth[iters & 1];
  float* out_auth = auth[(iters + 1) & 1];
  KL(k_scale, grid_for(nv, kBlock))(auth_fin, sums + 2 * iters - 1, out_auth, nv);
  if (hub_out) cudaMemcpyAsync(hub_out, hub_fin, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (auth_out) cudaMemcpyAsync(auth_out, out_auth, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = iters;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = (uint64_t)(2 * iters) * (h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes);
  return rc;
}

int tga_degree(tga_graph* gp, int64_t t_start, int64_t t_end, int32_t* degree_out, int64_t* avg_out) {
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));
  TGA_TRY(h.s_b.ensure((size_t)nv * 8));
  TGA_TRY(h.begin_call());
  unsigned long long* edges = edge_counter(h);
  cudaEvent_t* ev = h.kernel_begin();
  KL(k_degree, grid_for(nv, kBlock))(h.view, t_start, t_end, h.s_a.as<int32_t>(),
                                                          h.s_b.as<int64_t>(), edges);
  h.kernel_end(ev);
  if (degree_out) cudaMemcpyAsync(degree_out, h.s_a.p, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (avg_out) cudaMemcpyAsync(avg_out, h.s_b.p, (size_t)nv * 8, cudaMemcpyDeviceToHost, h.stream);
  h.timing.iterations = 1;
  const int rc = finish(h, edges);
  h.timing.compressed_bytes = h.info.graph_bytes + h.info.timestamp_bytes + h.info.index_bytes;
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
  if (!gp) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *gp;
  const int32_t nv = h.view.max_vertex;
  if (prio_mode == 2 && !prio_in) return fail(TGA_E_ARG, "priorities required for mode 2");
  if (prio_mode < 0 || prio_mode > 2) return fail(TGA_E_ARG, "unknown priority mode");
  TGA_TRY(h.s_a.ensure((size_t)nv * 4));  // colours
  TGA_TRY(h.s_b.ensure((size_t)nv * 4));  // priorities
  TGA_TRY(h.s_q0.ensure((size_t)nv * 4));
  TGA_TRY(h.s_q1.ensure((size_t)nv * 4));
  TGA_TRY(h.s_cnt.ensure(64));
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
  if (prio_mode == 0) KL(k_gc_prio_curand, grid_for(nv, kBlock))(prio, nv);
  else cudaMemcpyAsync(prio, prio_in, (size_t)nv * 4, cudaMemcpyHostToDevice, h.stream);
  cudaMemsetAsync(color, 0xFF, (size_t)nv * 4, h.stream);
  KL(k_iota, grid_for(nv, kBlock))(h.s_q0.as<int32_t>(), nv);
  int32_t* cnt = h.s_cnt.as<int32_t>();
  DevBuf* cur = &h.s_q0;
  DevBuf* nxt = &h.s_q1;
  int32_t wn = nv;
  int round = 0;
  while (wn != 0 && round < 512) {
    cudaMemsetAsync(cnt, 0, 4, h.stream);
    cudaEvent_t* ev = h.kernel_begin();
    KL(k_gc_round, grid_for(wn, kBlock))(h.view, cur->as<int32_t>(), wn, nxt->as<int32_t>(), cnt,
                                                              color, prio, (uint32_t)round, flags & TGA_GC_JAVA_ISOLATED,
                                                              edges);
    h.kernel_end(ev);
    cudaMemcpyAsync(&h.h_pinned[24], cnt, 4, cudaMemcpyDeviceToHost, h.stream);
    TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
    wn = (int32_t)h.h_pinned[24];
    std::swap(cur, nxt);
    ++round;
  }
  if (color_out) cudaMemcpyAsync(color_out, color, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (prio_out) cudaMemcpyAsync(prio_out, prio, (size_t)nv * 4, cudaMemcpyDeviceToHost, h.stream);
  if (rounds_out) *rounds_out = round;
  h.timing.iterations = round;
  return finish(h, edges);
}

}  // extern "C"
