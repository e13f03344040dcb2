// Host-side state of one resident compressed graph (the object behind tga_graph*).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/tga.h"
#include "slices.cuh"

namespace tga {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

#define TGA_CUDA_TRY(expr)                                                                    \
  do {                                                                                        \
    cudaError_t e_ = (expr);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return ::tga::fail(e_ == cudaErrorMemoryAllocation ? TGA_E_OOM : TGA_E_CUDA,           \
                         std::string(#expr " failed: ") + cudaGetErrorString(e_));            \
  } while (0)

// Growable device buffer owned by a handle.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t n);  // keeps contents only when no growth is needed
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct KernelTimer {
  cudaEvent_t a = nullptr, b = nullptr;
};

// An instantiated CUDA graph of an iteration loop (sweep.cuh, run_loop), kept on the handle and
// replayed while everything baked into its launches (its key) stays the same.
struct LoopGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;
  size_t timers = 0;      // kernel timer pairs the loop records
  int64_t launches = 0;   // kernels the loop launches
  int64_t decodes = 0;    // of those, decode launches (timing.decode_launches)
};

struct CcJobDeleter {
  void operator()(tga_cc_job* j) const;
};

struct GraphHandle {
  tga_dataset_cfg cfg{};
  std::string name, storage;
  tga_info info{};
  GraphView view{};
  cudaStream_t stream = nullptr;
  int device = 0;
  int sm_count = 1;
  // resident format data
  DevBuf d_graph, d_ts, d_gl, d_gu, d_gs, d_tl, d_tu, d_ts_samples, d_err;
  // per-vertex outdegrees (int32, filled once at load by a decode kernel)
  DevBuf d_deg;
  // division by a running count d in [2, max outdegree + 1] by multiplication: (M, l - 1) per d
  // (k_degree_long in algos.cu, degree centrality); built at load
  DevBuf d_divtab;
  // edge-balanced work decomposition (slices.cuh): slices of long lists, work items, and
  // slice_first[v]..slice_first[v+1] = slices of vertex v (empty for short lists)
  DevBuf d_slices, d_items, d_slice_first, d_slice_deep;
  uint64_t work_bytes = 0;           // device bytes of the work decomposition (slices, schedule, runs)
  // decode order of the sweeps (vertex ids >= 0 and -(slice+1)), grouped by work class
  DevBuf d_order;
  // lean sweep schedule (lean.cuh): LeanEntry[nlean], the sweep order with short lists (copying
  // ones included) as whole-list entries
  DevBuf d_lean;
  int32_t nlean = 0;
  // copied values of every list resolved at load (GraphView::copies / copy_base)
  DevBuf d_copies, d_copy_base;
  DevBuf d_hot;  // hot scatter targets (GraphView::hot)
  int32_t nhot = 0;
  // runs of equal successors cut by slices: RunInfo[nruns], (run, slice) pairs of the per-call
  // pre-pass, and the per-call list index of each run's first in-window edge
  DevBuf d_runs, d_run_pairs, d_run_first;
  int32_t nruns = 0, nrun_pairs = 0;
  // sliced (long) lists: LongList[nlong] with the base of each list's segment in a buffer of one
  // entry per edge of all long lists (long_edges entries), and that base + first for each slice
  DevBuf d_long, d_slice_ebase;
  int32_t nlong = 0;
  int64_t long_edges = 0;
  DevBuf d_view;                     // device-global copy of `view` (GraphView::self)
  int32_t norder = 0;
  int32_t dense_min = 1;             // traversal levels with at least this many entries sweep all lists
  int32_t dense_div = 0;             // dense_min = schedule entries / dense_div (0: $TGA_DENSE_DIV or 1)
  std::vector<uint8_t> chain_host;   // list copies from a reference chain
  int32_t nitems = 0, nslice_items = 0;
  int64_t nslices = 0;
  int32_t slice_len = 0, item_edges = 0;
  std::vector<int32_t> slice_first_host;
  // scratch used by the algorithms
  DevBuf s_a, s_b, s_c, s_d, s_e, s_f, s_g, s_q0, s_q1, s_cnt, s_sum, s_edges;
  // multi-source traversal state kept between calls (batch.cu): arrivals | last-enqueued arrivals
  // ([max_vertex][m_cap] each), the wide queues, frontier masks, dirty bits, per-vertex epoch stamps and the list of
  // vertices the last traversal touched.  With m_clean, everything is "unreached"/zero except the
  // m_pending sources' entries at the touched vertices, which the next traversal resets first.
  DevBuf m_state, m_mask, m_dirty, m_stamp, m_touched, m_dq;
  // connected-components job reused by tga_cc / tga_cc_batch (batch.cu); dropped by build_work,
  // since its run table is sized for the decomposition's cut runs
  std::unique_ptr<tga_cc_job, CcJobDeleter> cc_cache;
  uint32_t work_gen = 0;             // bumped by every build_work (jobs made earlier refuse to run)
  int32_t m_cap = 0, m_pending = 0;
  uint32_t m_epoch = 0;
  bool m_clean = false;
  uint32_t* h_pinned = nullptr;  // small pinned readback area
  // timing of the last call
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
  std::vector<KernelTimer> ktimers;
  size_t ktimer_used = 0;
  tga_timing timing{};
  bool time_kernels = true;
  bool capturing = false;            // a loop is being captured into a CUDA graph (run_loop)
  LoopGraph pr_loop, hits_loop, prm_loop;
  int64_t info_edges = 0;            // total temporal edges (sum of outdegrees)
  int64_t max_ts = INT64_MAX;        // largest timestamp of the graph (computed at load)
  int64_t min_ts_data = INT64_MIN;   // smallest timestamp of the graph (same pass)
  std::vector<int32_t> degrees;      // host copy of the outdegrees

  int begin_call();                 // resets timing, records the start event
  int end_call();                   // records the end event, syncs, checks the device error word
  cudaEvent_t* kernel_begin();      // event pair around one decode launch (nullptr if disabled)
  int reserve_timers(size_t n);     // creates event pairs so that n more kernel_begin calls find them
  void kernel_end(cudaEvent_t* pair);
  int check_device_error();
  ~GraphHandle();
};

// Default slice length: short enough that a frontier level holding one slice of a hub is not
// bound by a single thread's sequential decode, long enough that checkpoints stay a fraction of
// the compressed bytes.
constexpr int32_t kDefaultSliceEdges = 24;

int load_graph(GraphHandle& h, const std::string& dir, const std::string& base, const tga_dataset_cfg& cfg);
// (Re)builds slices and work items: lists longer than slice_len edges are cut into slices,
// the others grouped into items of about item_edges edges.
int build_work(GraphHandle& h, int32_t slice_len, int32_t item_edges);
// Uploads the current view to its device-global copy (after any change of `view`).
int publish_view(GraphHandle& h);

// Computes h.max_ts with one timestamp-only pass (after the work decomposition exists).
int compute_max_timestamp(GraphHandle& h);
int build_hot(GraphHandle& h);
// True when [lo, hi) contains every timestamp of the graph.
inline bool window_covers_all(const GraphHandle& h, int64_t lo, int64_t hi) {
  return lo <= h.view.min_ts && hi > h.max_ts;
}

// Device bytes held by the handle's cached connected-components job (batch.cu).
size_t cc_cache_bytes(const GraphHandle& h);

// Connected components with seeds run as speculative batches of a multi-source traversal
// (batch.cu); same results as the one-seed-at-a-time loop.
int cc_seed_batches(GraphHandle& h, int64_t t_lo, int64_t t_hi, int32_t flags, int32_t* label_out,
                    int32_t* components_out);

// Returns the status of expr from the calling function when it is not TGA_OK.
#define TGA_TRY(expr)            \
  do {                           \
    int rc_ = (expr);            \
    if (rc_) return rc_;         \
  } while (0)

// Launch helpers shared by the algorithm files.
inline unsigned grid_for(int64_t items, int block) { return (unsigned)((items + block - 1) / block); }

// Fixed device scratch of tga_pagerank_noalloc (noalloc.cu), one per device: three rank vectors,
// the in-window outdegree and its inverse (kPrNoAllocMaxVertices entries each), the per-iteration
// rank sums (kPrNoAllocMaxIters) and a 256-byte block of counters that each call zeroes.
constexpr int32_t kPrNoAllocMaxVertices = 1 << 20;
constexpr int32_t kPrNoAllocMaxIters = 1024;
constexpr size_t kPrNoAllocVec = (size_t)kPrNoAllocMaxVertices * 4;
constexpr size_t kPrNoAllocSumsOff = 5 * kPrNoAllocVec;
constexpr size_t kPrNoAllocCountersOff = kPrNoAllocSumsOff + (size_t)kPrNoAllocMaxIters * 8;
constexpr size_t kPrNoAllocScratchBytes = kPrNoAllocCountersOff + 256;
// Device address of that scratch on `device`, looked up once per device (with the device made
// current) and cached.
int pr_noalloc_scratch(int device, unsigned char** out);

}  // namespace tga

struct tga_graph : tga::GraphHandle {};
