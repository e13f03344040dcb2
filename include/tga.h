/*
 * tga.h - C ABI of the B200 engine for temporal-graph analytics on the compressed
 * WebGraph/ChronoGraph-style format of Yukun-Cui/CompressTemporalGraph.
 *
 * The reference has no library: every workload is a standalone CUDA executable per dataset
 * (gpu_cuda/<DS>/<alg>.cu -> gpu_cuda/shared/<alg>.cu main()) configured by compile-time
 * macros (gpu_cuda/shared/dataset_config_base.cuh:1-67).  Each entry point below replaces one
 * of those main() bodies, or the host loader they share; the comment on each one names the
 * reference lines it stands in for.  All pointers are host pointers unless stated otherwise,
 * every result buffer is owned by the caller, the graph handle owns all device memory, and a
 * handle must not be used from two threads at once.  Every function returns a tga_status and
 * leaves a message in tga_last_error() (per thread) when it fails; nothing calls exit().
 */
#ifndef TGA_H
#define TGA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TGA_OK = 0,
  TGA_E_IO = 1,        /* missing / unreadable file (reference: tgaOpenFile -> exit, shared/path_config.cuh:26-36) */
  TGA_E_FORMAT = 2,    /* malformed or inconsistent files, unsupported format parameters */
  TGA_E_OOM = 3,       /* device allocation failed or the admission budget is exceeded */
  TGA_E_DECODE = 4,    /* device decode error (cursor past a stream, id out of range, chain too deep) */
  TGA_E_TIMEOUT = 5,   /* an iteration cap or a bounded wait ran out */
  TGA_E_ARG = 6,       /* invalid argument */
  TGA_E_CUDA = 7,      /* CUDA runtime error (reference: CHECK -> exit(1), shared/bfs.cu:23-32) */
  TGA_E_AGAIN = 8      /* served form: request not finished yet */
} tga_status;

/* Runtime form of the per-dataset macros of shared/dataset_config_base.cuh:11-45 and
 * gpu_cuda/<DS>/dataset_config.cuh (same names, same defaults). */
typedef struct {
  const char* name;               /* DATASET_NAME */
  const char* storage_name;       /* DATASET_STORAGE_NAME (NULL -> name) */
  int32_t max_label;              /* MAX_LABEL: largest vertex id processed */
  int32_t max_vertex;             /* MAX_Vertex: length of per-vertex result arrays */
  int64_t min_timestamp;          /* minTimestamp; TGA_UNSET_TS -> taken from the .timestamps header */
  int32_t min_graph_vertex;       /* MIN_GRAPH_VERTEX (diagnostics only) */
  int32_t active_vertex_begin;    /* ACTIVE_VERTEX_BEGIN */
  int32_t bfs_start_vertex;       /* BFS_START_VERTEX (default 1) */
  int32_t cc_vertex_begin;        /* CONNECTED_COMPONENTS_VERTEX_BEGIN (default 1) */
  int32_t multiple_initial_value; /* MULTIPLE_INITIAL_VALUE; accepted for compatibility, the
                                     decoder needs no multiples sentinel */
  int32_t pr_iters;               /* PAGERANK_ITERATIONS (default 10) */
  int32_t hits_iters;             /* HITS_ITERATIONS (default 10) */
} tga_dataset_cfg;

#define TGA_UNSET_TS ((int64_t)INT64_MIN)
#define TGA_T_MIN ((int64_t)0)
#define TGA_T_MAX ((int64_t)INT64_MAX)

typedef struct tga_graph tga_graph;

typedef struct {
  int32_t n;                      /* vertices in the files */
  int32_t max_label, max_vertex, active_vertex_begin;
  int64_t min_timestamp;          /* from the .timestamps header */
  uint64_t graph_bytes, timestamp_bytes, index_bytes;   /* bytes of .graph, .timestamps, 4 EF files */
  uint64_t device_bytes;          /* device memory held by the handle */
  int32_t graph_ef_low_bits, timestamp_ef_low_bits;
} tga_info;

/* Device-timed figures of the last algorithm call on a handle (CUDA events on its stream). */
typedef struct {
  double total_ms;                /* whole call, device side */
  double decode_ms;               /* sum over the launches of the fused decode kernels */
  int64_t decode_launches;
  int64_t edges_decoded;          /* temporal edges decoded (multi-edges included, all passes) */
  uint64_t compressed_bytes;      /* algorithmic bytes: stream + index bytes of the lists decoded */
  int32_t iterations;             /* levels / rounds / iterations executed */
  int64_t launches;               /* kernels of this library launched by the call */
} tga_timing;

/* Fills *cfg with the defaults of shared/dataset_config_base.cuh. */
void tga_cfg_default(tga_dataset_cfg* cfg);

/* Last error message of the calling thread ("" if none). */
const char* tga_last_error(void);

/* Replaces the loader part of every gpu_cuda/shared/<alg>.cu main() (bfs.cu:1694-1935): reads
 * <root>/data/compressed/<STORAGE>/<STORAGE>.{graph,timestamps}, graph_{lower,upper}_bits.bin
 * and timestamp_{lower,upper}_bits.bin (dataset_config_base.cuh:46-67).  root NULL or "" ->
 * $TGA_COMPRESS_ROOT, else "../.." (path_config.cuh:10-24, dataset_config_base.cuh:39-41).
 * The select structure of the EF index is built here (bfs.cu:1643-1654 builds it with one
 * device thread); the decode tables are not needed. */
int tga_open(const char* root, const tga_dataset_cfg* cfg, tga_graph** out);

/* Same as tga_open for files <dir>/<basename>.* and the four EF files in <dir>. */
int tga_open_dir(const char* dir, const char* basename, const tga_dataset_cfg* cfg, tga_graph** out);

int tga_close(tga_graph* g);
int tga_get_info(tga_graph* g, tga_info* out);
int tga_get_timing(tga_graph* g, tga_timing* out);
/* Work decomposition of the sweeps and traversals: lists longer than slice_edges are cut into
 * resumable slices (decoder checkpoints built once), shorter lists are grouped into work items of
 * about item_edges edges.  Defaults 24 / 256, or $TGA_SLICE_EDGES / $TGA_ITEM_EDGES at open.
 * The reference has no counterpart (one thread per vertex, shared/neighbor_access.cu:1599-1642). */
int tga_set_work_params(tga_graph* g, int32_t slice_edges, int32_t item_edges);
int tga_get_work_params(tga_graph* g, int32_t* slice_edges, int32_t* item_edges, int64_t* slices, int32_t* items);

/* Project autotuner (no reference counterpart): times the workloads whose speed depends on the
 * work decomposition (one PageRank and one HITS iteration, a full-window BFS, a full-window CC and
 * a CC over the middle half of the timestamp span) for slice lengths {16, 24, 32, 48} x item sizes {128, 256, 512}, then the
 * dense-level divisor {1, 2, 4} (a traversal level sweeps every list once its queue holds
 * 1/dense_div of the schedule), and leaves the graph configured with the fastest.  Results of
 * every call are independent of the choice.  CC jobs made before it refuse to run afterwards. */
typedef struct {
  int32_t slice_edges, item_edges, dense_div;  /* chosen */
  int32_t candidates;                          /* configurations timed */
  double best_ms, default_ms;                  /* probe time of the chosen and of the starting one */
} tga_tune_result;
int tga_autotune(tga_graph* g, tga_tune_result* out);

/* cudaStream_t of the handle, as an opaque pointer (all work of the handle runs on it). */
void* tga_stream(tga_graph* g);

/* Neighbour access / "RA" (neighbor_access.cu:1438-1642, main 1909-1930): decodes every list of
 * [active_vertex_begin, max_label) with its timestamps.  small_out[v] = outdegree(v) < 4 (the
 * reference's dv2), checksum_out[v] = order-sensitive hash of v's (successor, timestamp)
 * sequence (sum mod 2^64 of a 64-bit mix of (v, edge index, successor, timestamp)), degree_out[v] = outdegree.  Any output may be NULL (then it stays on the device). */
int tga_neighbor_access(tga_graph* g, uint8_t* small_out, uint64_t* checksum_out, int32_t* degree_out);

/* Successors and timestamps of one vertex in list order (EvolvingMultiGraph.successors,
 * EvolvingMultiGraph.java:391-443).  Writes min(count, cap) entries; *count = outdegree. */
int tga_neighbors(tga_graph* g, int32_t v, int32_t* dst, int64_t* ts, int32_t cap, int32_t* count);

/* Windowed point queries (EvolvingMultiGraph.isNeighbor(node, neighbor, from, to),
 * cpu_java/src/main/java/gr/uoa/di/networkanalysis/EvolvingMultiGraph.java:343-389): out[i] = 1 when
 * some edge node[i] -> neighbor[i] has a timestamp in [t_from[i], t_to[i]] (both ends inclusive, as
 * the reference), else 0.  t_from / t_to may be NULL (no bound), which is isNeighbor(node, neighbor)
 * (EvolvingMultiGraph.java:328-341).  nq queries in one launch, one thread each. */
int tga_is_neighbor(tga_graph* g, int32_t nq, const int32_t* node, const int32_t* neighbor, const int64_t* t_from,
                    const int64_t* t_to, uint8_t* out);

/* Whole graph as CSR: offsets[n+1], dst[m], ts[m] (cap = capacity of dst/ts). */
int tga_decode_all(tga_graph* g, int64_t* offsets, int32_t* dst, int64_t* ts, int64_t cap);

/* Failure-detection self-test (no reference counterpart): launches a two-block cooperative grid
 * whose second block never reaches the grid barrier, so the first block's wait runs out after
 * limit_ms (<= 10 s; the traversals use 10 s).  *status_out = 1 when the wait ended with the
 * timeout status, as every traversal's barriers do; the context stays usable. */
int tga_barrier_selftest(double limit_ms, int32_t* status_out);

/* Temporal BFS (bfs.cu:1218-1692, host loop 1999-2038).  Edge (x->y,t) with t in [t_lo, t_hi)
 * relaxes y when arrival(x) <= t; only the first in-window occurrence of consecutive equal
 * successors counts.  arrival_out[v] = earliest arrival (INT32_MAX unreached, source = max(t_lo,0));
 * hops_out[v] = fewest edges of a path from the source that reaches every vertex on it at that
 * vertex's earliest arrival (a BFS over edges with arrival(x) <= t == arrival(y)); this is the
 * deterministic form of the reference's racy d_Ca level.  src < 0 -> bfs_start_vertex. */
int tga_bfs(tga_graph* g, int32_t src, int64_t t_lo, int64_t t_hi, int32_t* arrival_out, int32_t* hops_out);

/* Connected components by temporal reach (connected_components.cu:1210-1233,1679-1776, seed loop
 * 2091-2149): seeds ascend from cc_vertex_begin below max_label, need outdegree > 9 and must be
 * unreached; every vertex a seed reaches gets that seed's component number (last seed wins).
 * flags & 1: apply the reference's early exits (stop once > 0.8*max_label vertices were reached,
 * or after more than 50 consecutive components smaller than 5) on exact reach counts.
 * label_out[v] = -1 when never reached.  Seeds run as speculative batches of one multi-source
 * traversal (the next K candidates at once, validated in seed order; same labels as one seed per
 * traversal); flags & 2 runs one seed per traversal instead, the plain form batching is measured
 * against. */
#define TGA_CC_EARLY_EXIT 1
#define TGA_CC_ONE_SEED 2
int tga_cc(tga_graph* g, int64_t t_lo, int64_t t_hi, int32_t flags, int32_t* label_out, int32_t* components_out);

/* Temporal PageRank (pagerank.cu:1221-1660, loop 1956-2007) in FP32: rank starts at 1/max_vertex;
 * each iteration new[u] = (1-d)/max_label, then every source x in [active, max_label) adds
 * d*R[x]*(1-exp(-alpha*t))/deg(x) to each deduplicated in-window successor, then new is divided
 * by its sum.  deg(x) = in-window outdegree (= outdegree without a window).  iters <= 0 ->
 * pr_iters of the configuration; alpha is TEMPORAL_ALPHA (0.1 in the reference). */
int tga_pagerank(tga_graph* g, int32_t iters, float damping, float alpha, int64_t t_lo, int64_t t_hi, float* rank_out);

/* tga_pagerank that allocates no device memory (no counterpart in the reference).  For callers
 * that cannot allocate in the middle of their work: a server that reserved its device memory up
 * front and must not grow it per request, or a pipeline whose other streams must not be stalled
 * by cudaMalloc/cudaFree (they synchronise the device).  Same kernels and result as tga_pagerank;
 * the working vectors live in one fixed file-scope device array per device (about 20 MiB), and
 * the result goes to rank_out_dev, a caller-owned device buffer of max_vertex floats on the
 * graph's device.
 *   Limits: max_vertex <= 1048576 and iters <= 1024 (after iters <= 0 -> pr_iters); larger
 *   requests fail with TGA_E_ARG and a message naming the limit (use tga_pagerank).
 *   First call on a device: looks the array up with cudaGetSymbolAddress (this loads the module
 *   holding it); make one call before capturing a stream or starting latency-critical work.
 *   Under eager module loading (CUDA_MODULE_LOADING=EAGER) the array is reserved when the
 *   context is created instead, whether or not this entry point is ever called.  The address
 *   belongs to the primary context; it is looked up again after a cudaDeviceReset.
 *   rank_out_dev must be plain device memory (cudaMalloc), not managed memory.
 *   Concurrency: the array is shared by all handles on a device; overlapping calls race, so
 *   serialise them (one call at a time per device).
 *   Timing: only total_ms, iterations and edges_decoded are recorded (no per-kernel timers). */
int tga_pagerank_noalloc(tga_graph* g, int32_t iters, float damping, float alpha, int64_t t_lo, int64_t t_hi,
                         float* rank_out_dev);

/* HITS (hits.cu:1428-1987, loop 2284-2349) in FP32.  mode 0 = reference GPU semantics (hub and
 * authority accumulate without reset, L2-normalised each half step); mode 1 = Java semantics
 * (reset before each half step, BaselineRunner.java:493-549). */
#define TGA_HITS_GPU 0
#define TGA_HITS_JAVA 1
int tga_hits(tga_graph* g, int32_t iters, int32_t mode, int64_t t_lo, int64_t t_hi, float* hub_out, float* auth_out);

/* Windowed degree centrality with Java semantics (BaselineRunner.java:316-346; the GPU version
 * is degree_centrality.cu:1211-1680): for x in [active, max_label] count out-edges to active
 * successors with t_start <= t <= t_end ((0,0) = all edges), keep the running integer mean
 * time, and when t_start != t_end replace the count by (int)(0.85*c + 0.15*c*(avg-start)/(end-start) + 1). */
int tga_degree(tga_graph* g, int64_t t_start, int64_t t_end, int32_t* degree_out, int64_t* avg_out);

/* Jones-Plassmann greedy colouring (graph_coloring.cu:1475-1734): round c colours every worklist
 * vertex that has no deduplicated out-neighbour with higher (priority, lower id) still
 * uncoloured at the start of the round; at most 512 rounds.
 * prio_mode 0 = cuRAND XORWOW curand_init(123, v, 0), curand() % 256 (the reference's
 *               initialize_randlist, graph_coloring.cu:1624-1632, generated by cuRAND on device);
 *           1 = java.util.Random(123).nextInt(256) per vertex (BaselineRunner.java:392-396);
 *           2 = caller-provided prio_in[max_vertex].
 * flags & 1 = Java semantics for vertices without out-edges (coloured in round 0; the reference
 * GPU never colours them).  color_out[v] = round, UINT32_MAX if uncoloured.  prio_out optional. */
#define TGA_GC_JAVA_ISOLATED 1
int tga_color(tga_graph* g, int32_t prio_mode, const uint32_t* prio_in, int32_t flags, uint32_t* color_out,
              uint32_t* prio_out, int32_t* rounds_out);

/* ---- batched form ---------------------------------------------------------------------------
 * No counterpart in the reference (one query per executable run).
 * Many temporal BFS queries in one traversal: up to 256 sources per launch, packed 64 per 64-bit
 * word of a bitmask frontier, each with its own window [t_lo[i], t_hi[i]); larger batches run as
 * several launches.  arrival_out is nsrc x max_vertex (row i = query i), same semantics as
 * tga_bfs; hops are not produced. */
int tga_bfs_batch(tga_graph* g, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                  int32_t* arrival_out);

/* Fastest temporal paths from one source (temporal_ligra apps/temporal/Fastest-Compute.C, whose
 * edges have a start and an end time; here an edge happens at one instant, and paths follow
 * tga_bfs's edge rule).  A path's duration is the time of its last edge minus the time of its
 * first.  duration_out[v] = least duration of a path src -> v over edges with t in [t_lo, t_hi)
 * (0 for src, -1 when unreachable); departure_out[v] = the earliest first-edge time achieving it
 * (-1 for src and unreachable vertices).  Computed as the minimum over the distinct in-window
 * timestamps d of src's out-edges of (earliest arrival over [d, t_hi)) - d, the departures running
 * as rows of tga_bfs_batch's traversal.  Either output may be NULL.  The earliest-arrival query of
 * the same project (EarliestArrival-Compute.C) is tga_bfs's arrival_out. */
int tga_fastest(tga_graph* g, int32_t src, int64_t t_lo, int64_t t_hi, int64_t* duration_out,
                int64_t* departure_out);

/* Fewest-hop temporal paths (temporal_ligra apps/temporal/Shortest-Compute.C, whose update keeps a
 * label only when it is both earlier and shorter and so depends on the visiting order; here the
 * value is exact): hops_out[v] = the fewest edges on a time-respecting path from src to v within
 * [t_lo, t_hi) under tga_bfs's edge rule (INT32_MAX when unreached), arrival_out[v] = the earliest
 * arrival (equal to tga_bfs's).  Computed by level-synchronous relaxation: level k expands only the
 * vertices whose earliest arrival over at most k-1 edges dropped at level k-1.  Either output may
 * be NULL. */
int tga_shortest(tga_graph* g, int32_t src, int64_t t_lo, int64_t t_hi, int32_t* hops_out, int32_t* arrival_out);

/* Latest departures towards one target (temporal_ligra apps/temporal/LatestDeparture-Compute.C,
 * "reverse foremost", which transposes the graph).  tga_reverse writes a time-reversed copy of g to
 * <dir>/<base>.* with its index files: edge (x -> y, t) becomes (y -> x, pivot - t); pivot < 0 ->
 * the largest timestamp of g, returned in *pivot_out.  Open the copy with g's configuration.
 * tga_latest_departure(copy, pivot, target, ...) then gives out[v] = the latest first-edge time of
 * a path v -> target over edges with t in [t_lo, t_hi) (paths follow tga_bfs's edge rule on the
 * copy), -1 when there is none; out[target] = min(t_hi - 1, pivot).  One traversal from the target
 * on the copy over the window [pivot - t_hi + 1, pivot - t_lo + 1); pivot minus the timestamps must
 * stay below 2^31, as tga_bfs's arrivals are 32-bit. */
int tga_reverse(tga_graph* g, int64_t pivot, const char* dir, const char* base, int64_t* pivot_out);
int tga_latest_departure(tga_graph* reversed, int64_t pivot, int32_t target, int64_t t_lo, int64_t t_hi,
                         int64_t* out);

/* Many connected-components queries (one per window [t_lo[i], t_hi[i])) in one launch: up to 32
 * windows share the 256 source slots of each speculative seed batch, every window keeping its own
 * candidates, validation, early exits and labels; larger counts run as several launches.
 * label_out is nq x max_vertex (row i = window i), components_out[nq]; each row equals tga_cc's
 * result for that window.  flags: TGA_CC_EARLY_EXIT only. */
int tga_cc_batch(tga_graph* g, int32_t nq, const int64_t* t_lo, const int64_t* t_hi, int32_t flags,
                 int32_t* label_out, int32_t* components_out);

/* Resumable connected components for continuous batching: a job holds up to `capacity` (<= 32)
 * windows in flight, each in a slot.  tga_cc_job_add puts a window in a free slot (TGA_E_AGAIN when
 * none is free); tga_cc_job_step runs speculative seed batches for every window in flight until
 * all are finished or about budget_ms of device time has passed (budget_ms <= 0: until finished),
 * always stopping between batches, so other calls on the same graph may run between steps;
 * *finished gets bit s set for each slot whose window is finished; tga_cc_job_take copies a
 * finished window's labels (max_vertex entries, may be NULL) and component count and frees the
 * slot.  A window's result equals tga_cc's.  The job owns its device memory and uses the graph's
 * stream; destroy it before closing the graph.  After tga_set_work_params the job's add and step
 * return TGA_E_ARG (its per-run table belongs to the old decomposition): make a new job. */
typedef struct tga_cc_job tga_cc_job;
int tga_cc_job_create(tga_graph* g, int32_t capacity, int32_t flags, tga_cc_job** out);
int tga_cc_job_add(tga_cc_job* job, int64_t t_lo, int64_t t_hi, int32_t* slot);
int tga_cc_job_step(tga_cc_job* job, double budget_ms, uint32_t* finished);
int tga_cc_job_take(tga_cc_job* job, int32_t slot, int32_t* label_out, int32_t* components_out);
int tga_cc_job_destroy(tga_cc_job* job);

/* Many windowed PageRanks as one strided vector: up to 32 queries per launch (more run as several
 * launches), each list decoded once per iteration; rank_out is nq x max_vertex (row i = query i),
 * same semantics as tga_pagerank with that window. */
int tga_pagerank_batch(tga_graph* g, int32_t nq, int32_t iters, float damping, float alpha, const int64_t* t_lo,
                       const int64_t* t_hi, float* rank_out);

/* As tga_pagerank_batch with a per-query iteration count (iters[i] <= 0: the graph's pr_iters):
 * the batch runs the largest count and takes each query's result after its own last iteration, so
 * row i equals tga_pagerank(iters[i], ...) for that window. */
int tga_pagerank_batch_iters(tga_graph* g, int32_t nq, const int32_t* iters, float damping, float alpha,
                             const int64_t* t_lo, const int64_t* t_hi, float* rank_out);

/* ---- served form ---------------------------------------------------------------------------
 * No counterpart in the reference.  A server keeps several graphs resident and answers a stream
 * of queries.  One worker thread per graph repeatedly takes the queries that arrived since its
 * last round, admits them while their device working memory fits the server's budget, and runs
 * them together: BFS queries as one multi-source traversal, PageRank queries as one strided vector
 * (each with its own iteration count), point queries in one launch; CC queries join the graph's
 * resumable CC job (tga_cc_job_*), which each round advances by a time slice sized by the age of
 * its oldest window against the oldest other waiting query.  Rounds of different graphs take the
 * device one at a time, the graph with the oldest outstanding query first.  While a graph is
 * attached to a running server, only the server may use its handle. */
typedef struct tga_server tga_server;

#define TGA_Q_BFS 0
#define TGA_Q_PAGERANK 1
#define TGA_Q_CC 2
#define TGA_Q_NEIGHBOR 3

typedef struct {
  int32_t kind;        /* TGA_Q_BFS, TGA_Q_PAGERANK, TGA_Q_CC or TGA_Q_NEIGHBOR */
  int32_t graph;       /* id from tga_server_add_graph */
  int32_t src;         /* BFS source; point query: node */
  int32_t iters;       /* PageRank iterations (<= 0: pr_iters of the graph's configuration) */
  int32_t dst;         /* point query: neighbor */
  int32_t reserved;
  int64_t t_lo, t_hi;  /* time window [t_lo, t_hi); point query: [t_lo, t_hi], both ends inclusive
                          (tga_is_neighbor) */
  void* out;           /* caller-owned host buffer: max_vertex entries of BFS int32 arrivals, PageRank
                          float ranks (damping 0.85, alpha 0.1) or CC int32 labels; one uint8 for a
                          point query; NULL: results dropped */
} tga_query;

typedef struct {
  int64_t submitted, completed, failed, rounds;
  double p50_ms, p99_ms, mean_ms;  /* latency from tga_submit to completion */
  double queries_per_s;            /* completed / (last completion - first submission) */
} tga_server_stats;

/* budget_bytes: device working memory that admitted queries may hold at once (BFS about
 * 12 bytes, PageRank about 20 bytes, CC about 40 bytes per vertex of their graph; a point query
 * 64 bytes). */
int tga_server_create(int64_t budget_bytes, tga_server** out);
int tga_server_add_graph(tga_server* s, tga_graph* g, int32_t* graph_id);
/* Queues q; *ticket identifies it.  A query larger than the whole budget fails with TGA_E_OOM. */
int tga_submit(tga_server* s, const tga_query* q, int64_t* ticket);
/* TGA_OK when the query finished (its result is in q.out; *latency_ms if not NULL), TGA_E_AGAIN
 * while it is queued or running, or the query's own error code. */
int tga_poll(tga_server* s, int64_t ticket, double* latency_ms);
/* Blocks until every query submitted so far has finished. */
int tga_server_drain(tga_server* s);
int tga_server_get_stats(tga_server* s, tga_server_stats* out);
/* Stops the workers after the queued queries and frees the server (not the graphs). */
int tga_server_destroy(tga_server* s);

/* ---- format layer (host only, no GPU needed) ----------------------------------------------- */

typedef struct {
  int64_t n, m;
  double deg_exponent;
  int64_t max_degree;
  double repeat_frac, local_frac;
  int32_t local_radius;
  double pref_frac, copy_frac;
  int32_t ts_kind;                /* 0 uniform, 1 Poisson process, 2 bursty */
  int64_t ts_span, min_timestamp;
  uint64_t seed;
  int32_t ref_safe;               /* no in-edges to vertex 0 and n-1 */
  int32_t hub_count;              /* hubs: this many vertices, spread over the id range, get */
  int64_t hub_degree;             /* exactly hub_degree out-edges each (0: none) */
} tga_gen_params;

typedef struct {
  int64_t n, m, max_degree;
  uint64_t graph_bytes, timestamp_bytes, index_bytes;
  int64_t copied_arcs, intervalised_arcs, residual_arcs, multiples_arcs, max_chain;
} tga_gen_summary;

/* Seeded synthetic dataset written in the reference layout under dir (base.* plus the 4 EF
 * files); raw_path (optional) receives the 4-column text edge list. */
int tga_generate(const tga_gen_params* p, const char* dir, const char* base, const char* raw_path,
                 tga_gen_summary* out);

/* Compresses a 4-column raw text edge list ("src dst w ts", sources sorted) the way
 * EvolvingMultiGraph.store does (EvolvingMultiGraph.java:147-275), plus the 4 EF index files.
 * A path ending in ".gz" is read through gzip, as the reference's data/raw/<DS>.raw.txt.gz.
 * max_label < 0 -> n-1. */
int tga_encode_raw(const char* raw_path, const char* dir, const char* base, int64_t max_label, tga_gen_summary* out);

/* Host-only writer behind tga_reverse: writes the time-reversed graph of a CSR (offsets[n+1],
 * dst[m], ts[m], every ts in [0, pivot]) as a dataset <dir>/<base>.* with its index files.  Each
 * new list is ordered by successor, and repeated successors by reversed time. */
int tga_write_reversed(const int64_t* offsets, const int32_t* dst, const int64_t* ts, int64_t n, int64_t pivot,
                       const char* dir, const char* base, tga_gen_summary* out);

/* Realised backward-reference chain depth (cpu_java ReferenceDepthScanner.java:18-110), host only:
 * reads <dir>/<base>.graph, .offsets and .properties; a list that copies from the list `ref`
 * positions back has depth one more than that list, other lists depth 0.  depth_out (n entries,
 * may be NULL) gets every list's depth; depth_counts[d] counts lists of depth d < 16, deeper ones
 * are truncated_nodes, as the reference counts them. */
typedef struct {
  int64_t nodes, referenced_nodes, truncated_nodes;
  int32_t maximum_depth, configured_max_ref_count;
  int64_t depth_counts[16];
} tga_ref_depths;
int tga_reference_depths(const char* dir, const char* base, tga_ref_depths* out, int32_t* depth_out);

/* Producer of the four GPU index files (graph_{lower,upper}_bits.bin, timestamp_{lower,upper}_bits.bin,
 * the layout read by sh/bfs.cu:543-565,1785-1789, for which the reference ships no producer) for a
 * directory the Java encoder wrote: graph offsets from <base>.offsets (gamma deltas,
 * BVMultiGraph.java:1913-1922), timestamp offsets by walking <base>.timestamps with each record's
 * outdegree (EvolvingMultiGraph.java:131-275); needs the nodes property of <base>.properties.
 * tga_open does the same in memory when the index files are missing. */
int tga_build_index(const char* dir, const char* base, int64_t max_label);
/* The same files with the two walks run on the GPU: the offsets and timestamp streams decoded
 * speculatively in 4096-bit chunks, each chunk redecoded from its predecessor's exit until the
 * chunks fall into step, then every offset written in parallel.  TGA_E_TIMEOUT if the chunks do
 * not settle in 64 rounds (tga_build_index then gives the files). */
int tga_build_index_device(const char* dir, const char* base, int64_t max_label);

/* 65536-entry 16-bit look-ahead decode table, (length << 16) | value, 0 if the code does not fit;
 * kind 0 = gamma (gpu_cuda/decode_tables/gammaInA.txt), 3 = zeta_3 (zetaInA.txt). */
int tga_decode_table(int32_t kind, int32_t* out);

/* Writes n values with one code into out (MSB-first, zero-padded), as dsiutils' OutputBitStream
 * does for the reference encoder: kind 0 = gamma, 1 = zeta_k, 2 = unary, 3 = 64-bit fixed width
 * (writeLong(x, 64), the .timestamps header).  *nbits = bits written; TGA_E_ARG if cap is short. */
int tga_encode_codes(int32_t kind, int32_t k, const uint64_t* values, int64_t n, uint8_t* out, int64_t cap,
                     int64_t* nbits);

/* Elias-Fano index of a non-decreasing sequence in the GPU layout of the four *_bits.bin files
 * (read by gpu_cuda/shared/bfs.cu:543-565).  l < 0 -> l = (int)log2(stream_bytes*8/max_label) is
 * the caller's job; here l must be given.  Sizes are returned in *lower_bytes / *upper_bytes; a
 * NULL buffer is a size query. */
int tga_ef_encode(const uint64_t* values, int64_t n, int32_t l, uint8_t* lower, int64_t lower_cap, uint8_t* upper,
                  int64_t upper_cap, int64_t* lower_bytes, int64_t* upper_bytes);

#ifdef __cplusplus
}
#endif
#endif /* TGA_H */
