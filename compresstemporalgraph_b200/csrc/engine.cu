// Loader and handle management: reads the reference's on-disk files, builds the EF select
// samples, uploads everything into HBM in the layout documented in dview.cuh, and computes the
// per-vertex outdegrees once.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "decoder.cuh"
#include "engine.hpp"
#include "format.hpp"
#include "lean.cuh"
#include "trace.cuh"

namespace tga {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int DevBuf::ensure(size_t n) {
  if (n <= bytes && p) return TGA_OK;
  release();
  if (n == 0) n = 8;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    cudaGetLastError();
    return fail(TGA_E_OOM, "device allocation of " + std::to_string(n) + " bytes failed: " + cudaGetErrorString(e));
  }
  bytes = n;
  return TGA_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

GraphHandle::~GraphHandle() {
  if (stream) cudaStreamSynchronize(stream);
  for (DevBuf* b : {&d_graph, &d_ts, &d_gl, &d_gu, &d_gs, &d_tl, &d_tu, &d_ts_samples, &d_err, &d_deg, &d_slices,
                    &d_items, &d_slice_first, &d_slice_deep, &d_order, &d_lean, &d_copies, &d_copy_base, &d_hot, &d_runs, &d_run_pairs, &d_run_first, &d_long, &d_slice_ebase,
                    &d_view, &s_edges, &s_a, &s_b, &s_c, &s_d, &s_e, &s_f, &s_g, &s_q0, &s_q1, &s_cnt, &s_sum,
                    &m_state, &m_mask, &m_dirty, &m_stamp, &m_touched, &m_dq, &d_divtab})
    b->release();
  for (auto& k : ktimers) {
    if (k.a) cudaEventDestroy(k.a);
    if (k.b) cudaEventDestroy(k.b);
  }
  for (LoopGraph* lg : {&pr_loop, &hits_loop, &prm_loop})
    if (lg->exec) cudaGraphExecDestroy(lg->exec);
  if (ev_begin) cudaEventDestroy(ev_begin);
  if (ev_end) cudaEventDestroy(ev_end);
  if (h_pinned) cudaFreeHost(h_pinned);
  if (stream) cudaStreamDestroy(stream);
}

int GraphHandle::begin_call() {
  timing = tga_timing{};
  ktimer_used = 0;
  if (int rc = s_sum.ensure(4096)) return rc;  // work and edge counters
  TGA_CUDA_TRY(cudaMemsetAsync(d_err.p, 0, sizeof(uint32_t), stream));
  TGA_CUDA_TRY(cudaEventRecord(ev_begin, stream));
  return TGA_OK;
}

int GraphHandle::reserve_timers(size_t n) {
  while (ktimers.size() < ktimer_used + n) {
    KernelTimer k;
    if (cudaEventCreate(&k.a) != cudaSuccess || cudaEventCreate(&k.b) != cudaSuccess)
      return fail(TGA_E_CUDA, "cannot create timing events");
    ktimers.push_back(k);
  }
  return TGA_OK;
}

cudaEvent_t* GraphHandle::kernel_begin() {
  if (!time_kernels) return nullptr;
  if (ktimer_used == ktimers.size()) {
    KernelTimer k;
    if (cudaEventCreate(&k.a) != cudaSuccess || cudaEventCreate(&k.b) != cudaSuccess) return nullptr;
    ktimers.push_back(k);
  }
  KernelTimer& k = ktimers[ktimer_used++];
  // Inside a capture the record must be a graph node of its own (an external record), so the
  // replayed graph still times the kernel.
  if (capturing) cudaEventRecordWithFlags(k.a, stream, cudaEventRecordExternal);
  else cudaEventRecord(k.a, stream);
  return &k.a;
}

void GraphHandle::kernel_end(cudaEvent_t* pair) {
  if (!pair) return;
  KernelTimer* k = reinterpret_cast<KernelTimer*>(pair);
  if (capturing) cudaEventRecordWithFlags(k->b, stream, cudaEventRecordExternal);
  else cudaEventRecord(k->b, stream);
  timing.decode_launches++;
}

int GraphHandle::check_device_error() {
  uint32_t err = 0;
  TGA_CUDA_TRY(cudaMemcpyAsync(h_pinned, d_err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(stream));
  err = h_pinned[0];
  if (err) {
    std::string what;
    if (err & kErrCursor) what += " cursor-past-stream";
    if (err & kErrCode) what += " code-too-long";
    if (err & kErrChain) what += " reference-chain-too-deep";
    if (err & kErrId) what += " vertex-id-out-of-range";
    if (err & kErrCount) what += " list-shorter-than-outdegree";
    if (err & kErrIndex) what += " index-lookup-out-of-range";
    if (err & kErrTimeout) return fail(TGA_E_TIMEOUT, "iteration cap reached on the device");
    return fail(TGA_E_DECODE, "device decode error:" + what);
  }
  return TGA_OK;
}

int GraphHandle::end_call() {
  TGA_CUDA_TRY(cudaEventRecord(ev_end, stream));
  TGA_CUDA_TRY(cudaGetLastError());
  int rc = check_device_error();
  float ms = 0;
  cudaEventElapsedTime(&ms, ev_begin, ev_end);
  timing.total_ms = ms;
  double dk = 0;
  for (size_t i = 0; i < ktimer_used; ++i) {
    float t = 0;
    if (cudaEventElapsedTime(&t, ktimers[i].a, ktimers[i].b) == cudaSuccess) dk += t;
  }
  timing.decode_ms = dk;
  return rc;
}

// ---------------------------------------------------------------------------------------------
// Loading

#if defined(__BYTE_ORDER__) && __BYTE_ORDER__ != __ORDER_LITTLE_ENDIAN__
#error "the stream words are built by byte-swapping little-endian host loads"
#endif

// Byte i of the stream becomes bits 63-8(i%8) .. 56-8(i%8) of word i/8 (the device reads the
// streams as big-endian 64-bit words); bytes past the end are zero.
static void to_be_words(const std::vector<uint8_t>& bytes, std::vector<uint64_t>& words, size_t pad_words) {
  const size_t nw = (bytes.size() + 7) / 8;
  words.assign(nw + pad_words, 0);
  if (!bytes.empty()) std::memcpy(words.data(), bytes.data(), bytes.size());
  for (size_t i = 0; i < nw; ++i) words[i] = __builtin_bswap64(words[i]);
}

static void to_le_words(const std::vector<uint8_t>& bytes, std::vector<uint64_t>& words, size_t pad_words) {
  const size_t nw = (bytes.size() + 7) / 8;
  words.assign(nw + pad_words, 0);
  std::memcpy(words.data(), bytes.data(), bytes.size());
}

// samples[k] = position of the (64k)-th one; returns the number of ones.
static uint64_t build_select_samples(const std::vector<uint64_t>& upper, std::vector<uint64_t>& samples) {
  samples.clear();
  uint64_t ones = 0;
  for (size_t wi = 0; wi < upper.size(); ++wi) {
    uint64_t w = upper[wi];
    while (w) {
      const int b = __builtin_ctzll(w);
      if ((ones & 63) == 0) samples.push_back(wi * 64 + (uint64_t)b);
      ++ones;
      w &= w - 1;
    }
  }
  samples.push_back(upper.size() * 64);  // guard
  return ones;
}

template <class T>
static int upload(GraphHandle& h, DevBuf& b, const std::vector<T>& v) {
  int rc = b.ensure(v.size() * sizeof(T));
  if (rc) return rc;
  TGA_CUDA_TRY(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  h.info.device_bytes += v.size() * sizeof(T);
  return TGA_OK;
}

// Outdegree of every list and whether it copies from a reference chain.
__global__ void k_outdegrees(GraphView g, int32_t* deg, uint8_t* chain, int32_t count) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= count) return;
  uint64_t pos = ef_get(g, g.gef, (uint64_t)x);
  const int d = (int)read_gamma(g, g.g, pos);
  deg[x] = d;
  chain[x] = d > 0 && read_unary(g, g.g, pos) > 0;
}

// Resolves the copy mask of every list with a reference into GraphView::copies (two passes of
// k_resolve_copies: counts, then values at their prefix-sum bases).
static int resolve_copies(GraphHandle& h) {
  // The chain walk reads the device-global copy of the view (max_list has been set since it was
  // last published).
  TGA_TRY(publish_view(h));
  std::vector<int32_t> ids;
  for (size_t x = 0; x < h.chain_host.size(); ++x)
    if (h.chain_host[x]) ids.push_back((int32_t)x);
  const size_t nb = h.degrees.size() + 1;
  std::vector<uint32_t> base(nb, 0);
  int rc;
  DevBuf d_ids, d_cnt;
  std::vector<uint32_t> cnt(ids.size(), 0);
  if (!ids.empty()) {
    if ((rc = d_ids.ensure(ids.size() * 4)) || (rc = d_cnt.ensure(ids.size() * 4))) return rc;
    TGA_CUDA_TRY(cudaMemcpy(d_ids.p, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice));
    k_resolve_copies<<<grid_for((int64_t)ids.size(), 128), 128, 0, h.stream>>>(h.view, d_ids.as<int32_t>(),
                                                                              (int32_t)ids.size(), d_cnt.as<uint32_t>(),
                                                                              nullptr, nullptr);
    TGA_CUDA_TRY(cudaGetLastError());
    TGA_CUDA_TRY(cudaMemcpyAsync(cnt.data(), d_cnt.p, ids.size() * 4, cudaMemcpyDeviceToHost, h.stream));
    if ((rc = h.check_device_error())) return rc;
  }
  uint64_t total = 0;
  {
    size_t k = 0;
    for (size_t x = 0; x + 1 < nb; ++x) {
      base[x] = (uint32_t)total;
      if (k < ids.size() && (size_t)ids[k] == x) total += cnt[k++];
      if (total >= (1ull << 32)) return fail(TGA_E_FORMAT, "more than 2^32 copied values");
    }
    base[nb - 1] = (uint32_t)total;
  }
  if ((rc = h.d_copy_base.ensure(nb * 4)) || (rc = h.d_copies.ensure(std::max<uint64_t>(total, 1) * 4))) return rc;
  TGA_CUDA_TRY(cudaMemcpy(h.d_copy_base.p, base.data(), nb * 4, cudaMemcpyHostToDevice));
  h.info.device_bytes += nb * 4 + std::max<uint64_t>(total, 1) * 4;
  if (!ids.empty()) {
    k_resolve_copies<<<grid_for((int64_t)ids.size(), 128), 128, 0, h.stream>>>(
        h.view, d_ids.as<int32_t>(), (int32_t)ids.size(), nullptr, h.d_copy_base.as<uint32_t>(), h.d_copies.as<int32_t>());
    TGA_CUDA_TRY(cudaGetLastError());
    TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
    if ((rc = h.check_device_error())) return rc;
  }
  h.view.copies = h.d_copies.as<int32_t>();
  h.view.copy_base = h.d_copy_base.as<uint32_t>();
  return publish_view(h);
}

int load_graph(GraphHandle& h, const std::string& dir, const std::string& base, const tga_dataset_cfg& cfg) {
  h.cfg = cfg;
  if (cfg.max_label < 0 || cfg.max_vertex <= cfg.max_label)
    return fail(TGA_E_ARG, "max_vertex must exceed max_label >= 0");
  const std::string bp = dir + "/" + base;
  std::vector<uint8_t> graph, ts, gl, gu, tl, tu;
  const std::pair<const char*, std::vector<uint8_t>*> files[] = {
      {".graph", &graph}, {".timestamps", &ts}};
  for (const auto& f : files)
    if (!read_file(bp + f.first, *f.second))
      return fail(TGA_E_IO, "Cannot open required file: " + bp + f.first + " (set TGA_COMPRESS_ROOT if needed)");
  const std::pair<const char*, std::vector<uint8_t>*> idx[] = {
      {"/graph_lower_bits.bin", &gl}, {"/graph_upper_bits.bin", &gu},
      {"/timestamp_lower_bits.bin", &tl}, {"/timestamp_upper_bits.bin", &tu}};
  std::string missing;
  for (const auto& f : idx)
    if (missing.empty() && !read_file(dir + f.first, *f.second)) missing = dir + f.first;
  if (ts.size() < 8) return fail(TGA_E_FORMAT, "timestamps file shorter than its 64-bit header");
  if (!missing.empty()) {
    // No GPU index files (a directory written by the Java encoder): rebuild their content from
    // <base>.offsets and the streams, walked on the GPU (offsets_on_device; the host walk
    // index_from_offsets only if its speculative chunks did not fall into step).
    std::vector<uint8_t> offsets;
    if (!read_file(bp + ".offsets", offsets))
      return fail(TGA_E_IO, "Cannot open required file: " + missing + " (nor " + bp +
                                ".offsets to rebuild it; set TGA_COMPRESS_ROOT if needed)");
    const auto pr = read_properties(bp + ".properties");
    const auto it = pr.find("nodes");
    if (it == pr.end()) return fail(TGA_E_FORMAT, "rebuilding the index needs the nodes property of " + bp + ".properties");
    try {
      EFIndex ge, te;
      const int64_t nodes = std::atoll(it->second.c_str());
      std::vector<uint64_t> goff, toff;
      const int drc = offsets_on_device(graph, offsets, ts, nodes, goff, toff);
      if (drc == TGA_OK) {
        ge = ef_build(goff, ef_low_bits(graph.size(), cfg.max_label));
        te = ef_build(toff, ef_low_bits(ts.size(), cfg.max_label));
      } else if (drc == TGA_E_TIMEOUT) {
        index_from_offsets(graph, offsets, ts, nodes, 2, cfg.max_label, &ge, &te);
      } else {
        return drc;
      }
      gl = std::move(ge.lower);
      gu = std::move(ge.upper);
      tl = std::move(te.lower);
      tu = std::move(te.upper);
    } catch (const std::exception& e) {
      return fail(TGA_E_FORMAT, std::string("rebuilding the index from .offsets: ") + e.what());
    }
  }
  int64_t header = 0;
  for (int i = 0; i < 8; ++i) header = (int64_t)(((uint64_t)header << 8) | ts[(size_t)i]);
  if (cfg.min_timestamp != TGA_UNSET_TS && cfg.min_timestamp != header)
    return fail(TGA_E_FORMAT, "minTimestamp " + std::to_string(cfg.min_timestamp) +
                                  " of the configuration differs from the .timestamps header " +
                                  std::to_string(header));

  const auto props = read_properties(bp + ".properties");
  auto prop_int = [&](const char* k, long long dflt) -> long long {
    auto it = props.find(k);
    return it == props.end() ? dflt : std::atoll(it->second.c_str());
  };
  if (prop_int("windowsize", 7) <= 0) return fail(TGA_E_FORMAT, "graphs stored without references (windowsize 0) are not supported");
  if (prop_int("zetak", 3) != 3) return fail(TGA_E_FORMAT, "only zeta_3 residual coding is supported");
  const int min_interval = (int)prop_int("minintervallength", 4);
  if (min_interval < 1) return fail(TGA_E_FORMAT, "minimum interval length must be positive");
  if (prop_int("maxrefcount", 3) > kMaxLevels - 1)
    return fail(TGA_E_FORMAT, "reference chains deeper than " + std::to_string(kMaxLevels - 1) + " are not supported");

  std::vector<uint64_t> wg, wt, wgl, wgu, wtl, wtu, sg, st;
  to_be_words(graph, wg, 2);
  to_be_words(ts, wt, 2);
  to_be_words(gl, wgl, 2);
  to_be_words(tl, wtl, 2);
  to_le_words(gu, wgu, 1);
  to_le_words(tu, wtu, 1);
  const uint64_t gcount = build_select_samples(wgu, sg);
  const uint64_t tcount = build_select_samples(wtu, st);
  const int lg = ef_low_bits(graph.size(), cfg.max_label);
  const int lt = ef_low_bits(ts.size(), cfg.max_label);
  if (gcount < (uint64_t)cfg.max_label + 1 || tcount < (uint64_t)cfg.max_label + 1)
    return fail(TGA_E_FORMAT, "EF index holds " + std::to_string(gcount) + "/" + std::to_string(tcount) +
                                  " entries, fewer than max_label+1 = " + std::to_string(cfg.max_label + 1));
  if (gl.size() * 8 < gcount * (uint64_t)lg || tl.size() * 8 < tcount * (uint64_t)lt)
    return fail(TGA_E_FORMAT, "EF lower-bits file too short for its entry count");
  int64_t n = prop_int("nodes", -1);
  if (n <= 0) n = (int64_t)std::min<uint64_t>(gcount, tcount);
  if (n > INT32_MAX) return fail(TGA_E_FORMAT, "more than 2^31-1 vertices");

  h.info.n = (int32_t)n;
  h.info.max_label = cfg.max_label;
  h.info.max_vertex = cfg.max_vertex;
  h.info.active_vertex_begin = cfg.active_vertex_begin;
  h.info.min_timestamp = header;
  h.info.graph_bytes = graph.size();
  h.info.timestamp_bytes = ts.size();
  h.info.index_bytes = gl.size() + gu.size() + tl.size() + tu.size();
  h.info.graph_ef_low_bits = lg;
  h.info.timestamp_ef_low_bits = lt;

  TGA_CUDA_TRY(cudaGetDevice(&h.device));
  TGA_CUDA_TRY(cudaDeviceGetAttribute(&h.sm_count, cudaDevAttrMultiProcessorCount, h.device));
  TGA_CUDA_TRY(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
  TGA_CUDA_TRY(cudaEventCreate(&h.ev_begin));
  TGA_CUDA_TRY(cudaEventCreate(&h.ev_end));
  TGA_CUDA_TRY(cudaMallocHost((void**)&h.h_pinned, 4096));
  int rc;
  if ((rc = upload(h, h.d_graph, wg)) || (rc = upload(h, h.d_ts, wt)) || (rc = upload(h, h.d_gl, wgl)) ||
      (rc = upload(h, h.d_gu, wgu)) || (rc = upload(h, h.d_gs, sg)) || (rc = upload(h, h.d_tl, wtl)) ||
      (rc = upload(h, h.d_tu, wtu)) || (rc = upload(h, h.d_ts_samples, st)))
    return rc;
  if ((rc = h.d_err.ensure(256))) return rc;
  TGA_CUDA_TRY(cudaMemset(h.d_err.p, 0, 256));

  GraphView& v = h.view;
  v.g = Stream{h.d_graph.as<uint64_t>(), graph.size() * 8, wg.size()};
  v.t = Stream{h.d_ts.as<uint64_t>(), ts.size() * 8, wt.size()};
  v.gef = EFView{h.d_gl.as<uint64_t>(), h.d_gu.as<uint64_t>(), h.d_gs.as<uint64_t>(), wgu.size(), gcount, lg};
  v.tef = EFView{h.d_tl.as<uint64_t>(), h.d_tu.as<uint64_t>(), h.d_ts_samples.as<uint64_t>(), wtu.size(), tcount, lt};
  v.n = (int32_t)n;
  v.max_label = cfg.max_label;
  v.max_vertex = cfg.max_vertex;
  v.active_begin = cfg.active_vertex_begin;
  v.min_interval = min_interval;
  v.min_ts = header;
  v.err = h.d_err.as<uint32_t>();
  if ((rc = publish_view(h))) return rc;

  const int32_t ndeg = (int32_t)std::min<int64_t>(n, (int64_t)cfg.max_vertex);
  if ((rc = h.d_deg.ensure((size_t)cfg.max_vertex * sizeof(int32_t)))) return rc;
  h.info.device_bytes += (size_t)cfg.max_vertex * sizeof(int32_t);
  TGA_CUDA_TRY(cudaMemsetAsync(h.d_deg.p, 0, (size_t)cfg.max_vertex * sizeof(int32_t), h.stream));
  DevBuf chain_dev;
  if ((rc = chain_dev.ensure((size_t)std::max(ndeg, 1)))) return rc;
  k_outdegrees<<<grid_for(ndeg, 256), 256, 0, h.stream>>>(v, h.d_deg.as<int32_t>(), chain_dev.as<uint8_t>(), ndeg);
  TGA_CUDA_TRY(cudaGetLastError());
  std::vector<int32_t> deg((size_t)ndeg);
  h.chain_host.assign((size_t)ndeg, 0);
  TGA_CUDA_TRY(cudaMemcpyAsync(deg.data(), h.d_deg.p, (size_t)ndeg * 4, cudaMemcpyDeviceToHost, h.stream));
  TGA_CUDA_TRY(cudaMemcpyAsync(h.chain_host.data(), chain_dev.p, (size_t)ndeg, cudaMemcpyDeviceToHost, h.stream));
  if ((rc = h.check_device_error())) return rc;
  int64_t maxd = 0, m = 0;
  for (int32_t d : deg) {
    if (d < 0) return fail(TGA_E_FORMAT, "negative outdegree");
    maxd = std::max<int64_t>(maxd, d);
    m += d;
  }
  // Every temporal edge owns a zeta_2 timestamp code of at least 2 bits.
  if ((uint64_t)m > (uint64_t)(ts.size() - 8) * 4)
    return fail(TGA_E_FORMAT, "outdegrees sum to " + std::to_string(m) + " edges, more than the .timestamps stream can hold");
  // The largest outdegree caps every header-driven loop of the decoder on damaged streams.
  v.max_list = (int32_t)std::min<int64_t>(INT32_MAX / 4, std::max<int64_t>(maxd, 1));
  {
    // Per count d >= 2: l = ceil(log2 d) and M = ceil(2^(31 + l) / d), which is below 2^32, so that
    // for every n < 2^31, n / d = mulhi(M, n) >> (l - 1) (Granlund and Montgomery, "Division by
    // Invariant Integers using Multiplication", PLDI 1994: with M d - 2^(31+l) = e < d <= 2^l,
    // n e < 2^(31+l) keeps the rounding error below one step).  Stored as (M, l - 1); d = 1
    // divides trivially and entry 0 is unused.
    std::vector<uint32_t> tab(2 * ((size_t)v.max_list + 2), 0);
    for (uint64_t d = 2; d < (uint64_t)v.max_list + 2; ++d) {
      int l = 0;
      while ((1ull << l) < d) ++l;
      tab[2 * d] = (uint32_t)(((1ull << (31 + l)) + d - 1) / d);
      tab[2 * d + 1] = (uint32_t)(l - 1);
    }
    if ((rc = upload(h, h.d_divtab, tab))) return rc;
  }
  h.info_edges = m;
  h.degrees = std::move(deg);
  if ((rc = resolve_copies(h))) return rc;
  const char* env_slice = std::getenv("TGA_SLICE_EDGES");
  const char* env_item = std::getenv("TGA_ITEM_EDGES");
  if (int rc = build_work(h, env_slice ? std::atoi(env_slice) : kDefaultSliceEdges, env_item ? std::atoi(env_item) : 256))
    return rc;
  if (int rc = build_hot(h)) return rc;
  return compute_max_timestamp(h);
}

int publish_view(GraphHandle& h) {
  if (int rc = h.d_view.ensure(sizeof(GraphView))) return rc;
  h.view.self = h.d_view.as<GraphView>();
  TGA_CUDA_TRY(cudaMemcpyAsync(h.d_view.p, &h.view, sizeof(GraphView), cudaMemcpyHostToDevice, h.stream));
  TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return TGA_OK;
}

int build_work(GraphHandle& h, int32_t slice_len, int32_t item_edges) {
  if (slice_len < 16 || item_edges < 1) return fail(TGA_E_ARG, "slice length must be >= 16 and item size >= 1");
  // State sized for the old decomposition (the cached CC job's run table) goes; CC jobs made by
  // callers see the new generation and refuse to run.
  h.cc_cache.reset();
  ++h.work_gen;
  GraphView& v = h.view;
  // The build walks the lists without seeking (checkpoints are being made).
  v.slices = nullptr;
  v.slice_deep = nullptr;
  v.slice_first = nullptr;
  v.deg = nullptr;
  v.seek_min = INT32_MAX;
  if (int rc = publish_view(h)) return rc;
  const int32_t nd = (int32_t)h.degrees.size();
  std::vector<int32_t> big_v;
  std::vector<int64_t> slot_base{0}, deep_base{0};
  for (int32_t x = 0; x < nd; ++x) {
    const int32_t d = h.degrees[(size_t)x];
    // Long lists are sliced; so is every list that copies from a reference chain, whatever its
    // length: opening one parses the records along its chain (and walks the referenced lists to
    // the first copied value), which costs more than decoding a short list, so its state after
    // opening is kept as a checkpoint (a single slice when the list is short).
    if (d > slice_len || (d > 0 && h.chain_host[(size_t)x])) {
      big_v.push_back(x);
      const int64_t nslot = (d + slice_len - 1) / slice_len;
      slot_base.push_back(slot_base.back() + nslot);
      // Chain levels only for the slices of lists that copy from a chain.
      deep_base.push_back(deep_base.back() + (h.chain_host[(size_t)x] ? nslot : 0));
    }
  }
  const int32_t nbig = (int32_t)big_v.size();
  std::vector<int32_t> nsl((size_t)nbig, 0);
  std::vector<SliceState> slices;
  std::vector<DeepState> slice_deep_tmp;
  if (nbig) {
    DevBuf bv, sb, db, ns, tmp, tmpd;
    int rc;
    if ((rc = bv.ensure((size_t)nbig * 4)) || (rc = sb.ensure(slot_base.size() * 8)) || (rc = db.ensure(deep_base.size() * 8)) ||
        (rc = ns.ensure((size_t)nbig * 4)) || (rc = tmp.ensure((size_t)slot_base.back() * sizeof(SliceState))) ||
        (rc = tmpd.ensure((size_t)std::max<int64_t>(1, deep_base.back()) * sizeof(DeepState))))
      return rc;
    TGA_CUDA_TRY(cudaMemcpyAsync(db.p, deep_base.data(), deep_base.size() * 8, cudaMemcpyHostToDevice, h.stream));
    TGA_CUDA_TRY(cudaMemcpyAsync(bv.p, big_v.data(), (size_t)nbig * 4, cudaMemcpyHostToDevice, h.stream));
    TGA_CUDA_TRY(cudaMemcpyAsync(sb.p, slot_base.data(), slot_base.size() * 8, cudaMemcpyHostToDevice, h.stream));
    k_build_slices<<<grid_for(nbig, 64), 64, 0, h.stream>>>(v, bv.as<int32_t>(), sb.as<int64_t>(), db.as<int64_t>(), nbig, slice_len,
                                                           tmp.as<SliceState>(), tmpd.as<DeepState>(), ns.as<int32_t>());
    TGA_CUDA_TRY(cudaGetLastError());
    slices.resize((size_t)slot_base.back());
    TGA_CUDA_TRY(cudaMemcpyAsync(nsl.data(), ns.p, (size_t)nbig * 4, cudaMemcpyDeviceToHost, h.stream));
    TGA_CUDA_TRY(cudaMemcpyAsync(slices.data(), tmp.p, slices.size() * sizeof(SliceState), cudaMemcpyDeviceToHost,
                                 h.stream));
    slice_deep_tmp.resize((size_t)deep_base.back());
    TGA_CUDA_TRY(cudaMemcpyAsync(slice_deep_tmp.data(), tmpd.p, slice_deep_tmp.size() * sizeof(DeepState),
                                 cudaMemcpyDeviceToHost, h.stream));
    if ((rc = h.check_device_error())) return rc;
    bv.release(); sb.release(); db.release(); ns.release(); tmp.release(); tmpd.release();
  }
  // Compact the slices, build slice_first and the work items (slices first, then short lists).
  std::vector<SliceState> packed;
  std::vector<DeepState> packed_deep;
  std::vector<int32_t> slice_first((size_t)nd + 1, 0);
  std::vector<WorkItem> items;
  {
    int32_t b = 0;
    for (int32_t x = 0; x < nd; ++x) {
      slice_first[(size_t)x] = (int32_t)packed.size();
      if (b < nbig && big_v[(size_t)b] == x) {
        for (int32_t j = 0; j < nsl[(size_t)b]; ++j) {
          items.push_back(WorkItem{x, x + 1, (int32_t)packed.size()});
          const size_t slot = (size_t)(slot_base[(size_t)b] + j);
          const size_t dslot = (size_t)(deep_base[(size_t)b] + j);
          SliceState sl = slices[slot];
          if (sl.chain) {
            sl.deep = (int32_t)packed_deep.size();
            packed_deep.push_back(slice_deep_tmp[dslot]);
          }
          packed.push_back(sl);
        }
        ++b;
      }
    }
    slice_first[(size_t)nd] = (int32_t)packed.size();
  }
  // Runs of equal successors that slices cut: consecutive slices of a list that start inside the
  // same run (the builder left the run's start index in `run`) form one run, which begins in the
  // slice before the first of them.
  std::vector<RunInfo> runs;
  std::vector<int2> run_pairs;
  for (int32_t x = 0; x < nd; ++x) {
    const int32_t a = slice_first[(size_t)x], b = slice_first[(size_t)x + 1];
    for (int32_t j = a; j < b; ++j) {
      SliceState& sl = packed[(size_t)j];
      const int32_t rs = sl.run;
      if (rs < 0 || j == a) {
        sl.run = -1;
        continue;
      }
      if (!runs.empty() && runs.back().v == x && runs.back().start == rs &&
          runs.back().first_slice + runs.back().nslices == j) {
        ++runs.back().nslices;
      } else {
        runs.push_back(RunInfo{x, rs, j - 1, 2});
      }
      sl.run = (int32_t)runs.size() - 1;
    }
  }
  for (size_t r = 0; r < runs.size(); ++r)
    for (int32_t k = 0; k < runs[r].nslices; ++k) run_pairs.push_back(make_int2((int)r, runs[r].first_slice + k));
  h.nruns = (int32_t)runs.size();
  h.nrun_pairs = (int32_t)run_pairs.size();
  // Per-edge segments of the sliced lists (for workloads that are sequential per list).
  std::vector<LongList> longs;
  std::vector<int64_t> slice_ebase(packed.size(), 0);
  int64_t long_edges = 0;
  for (int32_t x = 0; x < nd; ++x) {
    const int32_t a = slice_first[(size_t)x], b = slice_first[(size_t)x + 1];
    if (a == b) continue;
    longs.push_back(LongList{x, 0, long_edges});
    for (int32_t j = a; j < b; ++j) slice_ebase[(size_t)j] = long_edges + packed[(size_t)j].first;
    long_edges += h.degrees[(size_t)x];
  }
  h.nlong = (int32_t)longs.size();
  h.long_edges = long_edges;
  h.nslice_items = (int32_t)items.size();
  {
    constexpr int32_t kVertexCost = 4, kMaxRange = 4096;
    int32_t start = -1, cost = 0;
    for (int32_t x = 0; x < nd; ++x) {
      const bool big = slice_first[(size_t)x + 1] != slice_first[(size_t)x];
      if (big) {
        if (start >= 0) items.push_back(WorkItem{start, x, -1});
        start = -1;
        cost = 0;
        continue;
      }
      if (start < 0) start = x;
      cost += h.degrees[(size_t)x] + kVertexCost;
      if (cost >= item_edges || x + 1 - start >= kMaxRange) {
        items.push_back(WorkItem{start, x + 1, -1});
        start = -1;
        cost = 0;
      }
    }
    if (start >= 0) items.push_back(WorkItem{start, nd, -1});
  }
  h.nitems = (int32_t)items.size();
  // Decode order for the sweeps: every slice, then every non-empty short list, grouped by work
  // class (quarter-octave of the outdegree) from the largest class down, so the 32 lanes of a warp
  // open their lists together and decode lists of nearly equal length.
  std::vector<int32_t> order;
  order.reserve(packed.size() + (size_t)nd);
  // Slices and lists that do not copy from a reference chain come first, those that do last:
  // only the latter run the (large) chain decoder, and keeping them together keeps the two code
  // paths from competing for the instruction cache.
  for (int c = 0; c < 2; ++c) {
    std::vector<int32_t> grp;
    for (size_t j = 0; j < packed.size(); ++j)
      if ((packed[j].chain != 0) == (c == 1)) grp.push_back((int32_t)j);
    // longest slices first, so the lanes of a warp decode slices of equal length
    std::stable_sort(grp.begin(), grp.end(),
                     [&](int32_t a, int32_t b) { return packed[(size_t)a].count > packed[(size_t)b].count; });
    for (int32_t j : grp) order.push_back(-j - 1);
  }
  {
    auto cls = [&](int32_t d) { return (int)std::floor(4.0 * std::log2((double)d)); };
    const int ncls = cls(std::max(slice_len, 1)) + 2;
    std::vector<std::vector<int32_t>> bins((size_t)ncls * 2);
    for (int32_t x = 0; x < nd; ++x) {
      const int32_t d = h.degrees[(size_t)x];
      if (d <= 0 || slice_first[(size_t)x + 1] != slice_first[(size_t)x]) continue;
      bins[(size_t)(std::min(cls(d), ncls - 1) * 2 + (h.chain_host[(size_t)x] ? 1 : 0))].push_back(x);
    }
    for (int c = 0; c < 2; ++c)
      for (int b = (int)bins.size() - 2 + c; b >= 0; b -= 2) order.insert(order.end(), bins[(size_t)b].begin(), bins[(size_t)b].end());
  }
  h.norder = (int32_t)order.size();
  // Lean schedule: the order above, with a short copying list (a single slice from edge 0) as a
  // whole-list entry (the lean decoder opens it from its record and the resolved copies).
  {
    std::vector<int32_t> ids;
    ids.reserve(order.size());
    for (int32_t e : order) {
      if (e < 0) {
        const SliceState& sl = packed[(size_t)(-e - 1)];
        if (sl.chain && sl.first == 0 && sl.count == h.degrees[(size_t)sl.v]) {
          ids.push_back(sl.v);
          continue;
        }
      }
      ids.push_back(e);
    }
    h.nlean = (int32_t)ids.size();
    if (h.info.graph_bytes * 8 >= (1ull << 48) || h.info.timestamp_bytes * 8 >= (1ull << 48))
      return fail(TGA_E_FORMAT, "stream longer than 2^48 bits");
    DevBuf tmp_ids;
    int rc;
    if ((rc = tmp_ids.ensure(std::max<size_t>(1, ids.size()) * 4)) ||
        (rc = h.d_lean.ensure(std::max<size_t>(1, ids.size()) * sizeof(LeanEntry))))
      return rc;
    if (!ids.empty()) {
      TGA_CUDA_TRY(cudaMemcpy(tmp_ids.p, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice));
      k_lean_entries<<<grid_for((int64_t)ids.size(), 256), 256, 0, h.stream>>>(v, tmp_ids.as<int32_t>(), (int32_t)ids.size(),
                                                                          h.d_lean.as<LeanEntry>());
      TGA_CUDA_TRY(cudaGetLastError());
      TGA_CUDA_TRY(cudaStreamSynchronize(h.stream));
      if ((rc = h.check_device_error())) return rc;
    }
    tmp_ids.release();
  }
  // A traversal level sweeps all lists instead of its queue once the queue holds at least
  // 1/TGA_DENSE_DIV of the schedule's entries.  Default 1 (a sweep only when every entry is in the
  // frontier): with the lean decoder the queue is the faster form at every level size measured
  // (2M/40M graph: BFS 11.3 ms with divisor 16, 7.5 with 4, 7.1 with 2 or 1; CC 39.6 / 37.3 /
  // 35.8 / 35.8 ms).
  const char* env_dense = std::getenv("TGA_DENSE_DIV");
  const int dense_div = h.dense_div > 0 ? h.dense_div : env_dense ? std::max(1, std::atoi(env_dense)) : 1;
  h.dense_min = std::max<int32_t>(1, h.norder / dense_div);
  h.nslices = (int64_t)packed.size();
  h.slice_len = slice_len;
  h.item_edges = item_edges;
  int rc;
  if ((rc = h.d_order.ensure(std::max<size_t>(1, order.size()) * 4))) return rc;
  if (!order.empty())
    TGA_CUDA_TRY(cudaMemcpy(h.d_order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
  if ((rc = h.d_long.ensure(std::max<size_t>(1, longs.size()) * sizeof(LongList))) ||
      (rc = h.d_slice_ebase.ensure(std::max<size_t>(1, slice_ebase.size()) * 8)))
    return rc;
  if (!longs.empty()) {
    TGA_CUDA_TRY(cudaMemcpy(h.d_long.p, longs.data(), longs.size() * sizeof(LongList), cudaMemcpyHostToDevice));
    TGA_CUDA_TRY(cudaMemcpy(h.d_slice_ebase.p, slice_ebase.data(), slice_ebase.size() * 8, cudaMemcpyHostToDevice));
  }
  if ((rc = h.d_runs.ensure(std::max<size_t>(1, runs.size()) * sizeof(RunInfo))) ||
      (rc = h.d_run_pairs.ensure(std::max<size_t>(1, run_pairs.size()) * sizeof(int2))) ||
      (rc = h.d_run_first.ensure(std::max<size_t>(1, runs.size()) * 4)))
    return rc;
  if (!runs.empty()) {
    TGA_CUDA_TRY(cudaMemcpy(h.d_runs.p, runs.data(), runs.size() * sizeof(RunInfo), cudaMemcpyHostToDevice));
    TGA_CUDA_TRY(cudaMemcpy(h.d_run_pairs.p, run_pairs.data(), run_pairs.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  if ((rc = h.d_items.ensure(std::max<size_t>(1, items.size()) * sizeof(WorkItem))) ||
      (rc = h.d_slices.ensure(std::max<size_t>(1, packed.size()) * sizeof(SliceState))) ||
      (rc = h.d_slice_deep.ensure(std::max<size_t>(1, packed_deep.size()) * sizeof(DeepState))) ||
      (rc = h.d_slice_first.ensure(slice_first.size() * 4)))
    return rc;
  if (!items.empty())
    TGA_CUDA_TRY(cudaMemcpy(h.d_items.p, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice));
  if (!packed.empty())
    TGA_CUDA_TRY(cudaMemcpy(h.d_slices.p, packed.data(), packed.size() * sizeof(SliceState), cudaMemcpyHostToDevice));
  if (!packed_deep.empty())
    TGA_CUDA_TRY(cudaMemcpy(h.d_slice_deep.p, packed_deep.data(), packed_deep.size() * sizeof(DeepState),
                            cudaMemcpyHostToDevice));
  TGA_CUDA_TRY(cudaMemcpy(h.d_slice_first.p, slice_first.data(), slice_first.size() * 4, cudaMemcpyHostToDevice));
  h.slice_first_host = std::move(slice_first);
  v.slices = h.d_slices.as<SliceState>();
  v.slice_deep = h.d_slice_deep.as<DeepState>();
  v.slice_first = h.d_slice_first.as<int32_t>();
  v.deg = h.d_deg.as<int32_t>();
  h.work_bytes = h.d_slices.bytes + h.d_slice_deep.bytes + h.d_slice_first.bytes + h.d_items.bytes + h.d_order.bytes +
                 h.d_lean.bytes +
                 h.d_runs.bytes + h.d_run_pairs.bytes + h.d_run_first.bytes + h.d_long.bytes + h.d_slice_ebase.bytes;
  v.seek_min = std::max(16, slice_len / 2);
  return publish_view(h);
}

}  // namespace tga

using namespace tga;

extern "C" {

void tga_cfg_default(tga_dataset_cfg* c) {
  if (!c) return;
  std::memset(c, 0, sizeof *c);
  c->name = "";
  c->storage_name = nullptr;
  c->max_label = 0;
  c->max_vertex = 0;
  c->min_timestamp = TGA_UNSET_TS;
  c->min_graph_vertex = 0;
  c->active_vertex_begin = 0;
  c->bfs_start_vertex = 1;
  c->cc_vertex_begin = 1;
  c->multiple_initial_value = -1;
  c->pr_iters = 10;
  c->hits_iters = 10;
}

const char* tga_last_error(void) { return g_last_error.c_str(); }

static int open_common(const std::string& dir, const std::string& base, const tga_dataset_cfg* cfg, tga_graph** out) {
  if (!cfg || !out) return fail(TGA_E_ARG, "null argument");
  *out = nullptr;
  tga_graph* g = new (std::nothrow) tga_graph();
  if (!g) return fail(TGA_E_OOM, "host allocation failed");
  g->name = cfg->name ? cfg->name : "";
  g->storage = cfg->storage_name ? cfg->storage_name : g->name;
  const int rc = load_graph(*g, dir, base, *cfg);
  if (rc) {
    const std::string msg = tga_last_error();
    delete g;
    set_error(msg);
    return rc;
  }
  *out = g;
  return TGA_OK;
}

int tga_open(const char* root, const tga_dataset_cfg* cfg, tga_graph** out) {
  TGA_TRACE("tga_open");
  if (!cfg) return fail(TGA_E_ARG, "null configuration");
  std::string r = root ? root : "";
  if (r.empty()) {
    const char* env = std::getenv("TGA_COMPRESS_ROOT");
    r = (env && env[0]) ? env : "../..";
  }
  while (!r.empty() && (r.back() == '/' || r.back() == '\\')) r.pop_back();
  const std::string name = cfg->name ? cfg->name : "";
  const std::string storage = cfg->storage_name ? cfg->storage_name : name;
  if (storage.empty()) return fail(TGA_E_ARG, "dataset name is empty");
  return open_common(r + "/data/compressed/" + storage, storage, cfg, out);
}

int tga_open_dir(const char* dir, const char* basename, const tga_dataset_cfg* cfg, tga_graph** out) {
  TGA_TRACE("tga_open_dir");
  if (!dir || !basename) return fail(TGA_E_ARG, "null path");
  return open_common(dir, basename, cfg, out);
}

int tga_close(tga_graph* g) {
  delete g;
  return TGA_OK;
}

int tga_get_info(tga_graph* g, tga_info* out) {
  if (!g || !out) return fail(TGA_E_ARG, "null argument");
  *out = g->info;
  // streams and index (counted at load) + work decomposition + scratch grown by the calls so far
  out->device_bytes += g->work_bytes;
  for (const DevBuf* b : {&g->s_a, &g->s_b, &g->s_c, &g->s_d, &g->s_e, &g->s_f, &g->s_g, &g->s_q0, &g->s_q1, &g->s_cnt,
                          &g->s_sum, &g->s_edges, &g->m_state, &g->m_mask, &g->m_dirty, &g->m_stamp, &g->m_touched, &g->m_dq})
    out->device_bytes += b->bytes;
  out->device_bytes += cc_cache_bytes(*g);
  return TGA_OK;
}

int tga_get_timing(tga_graph* g, tga_timing* out) {
  if (!g || !out) return fail(TGA_E_ARG, "null argument");
  *out = g->timing;
  return TGA_OK;
}

void* tga_stream(tga_graph* g) { return g ? (void*)g->stream : nullptr; }

int tga_set_work_params(tga_graph* g, int32_t slice_edges, int32_t item_edges) {
  if (!g) return fail(TGA_E_ARG, "null graph");
  if (cudaStreamSynchronize(g->stream) != cudaSuccess) return fail(TGA_E_CUDA, "stream synchronisation failed");
  return build_work(*g, slice_edges, item_edges);
}

// Autotuner: times the workloads whose speed depends on the work decomposition (one PageRank and
// one HITS iteration, a full-window BFS, a full-window CC and a CC over the middle half of the
// timestamp span; each run twice, the second timed) for each candidate and keeps the fastest
// total.  Slice length and item size are tried as a grid, then the dense-level divisor at the
// best of those.
int tga_autotune(tga_graph* g, tga_tune_result* out) {
  TGA_TRACE("tga_autotune");
  if (!g) return fail(TGA_E_ARG, "null graph");
  GraphHandle& h = *g;
  const int64_t span = h.max_ts - h.view.min_ts;
  const int64_t wlo = h.view.min_ts + span / 4, whi = h.view.min_ts + 3 * (span / 4) + 1;
  auto probe = [&](double* ms) -> int {
    double total = 0;
    for (int w = 0; w < 5; ++w)
      for (int rep = 0; rep < 2; ++rep) {
        int rc;
        if (w == 0) rc = tga_pagerank(g, 1, 0.85f, 0.1f, TGA_T_MIN, TGA_T_MAX, nullptr);
        else if (w == 1) rc = tga_hits(g, 1, TGA_HITS_GPU, TGA_T_MIN, TGA_T_MAX, nullptr, nullptr);
        else if (w == 2) rc = tga_bfs(g, -1, TGA_T_MIN, TGA_T_MAX, nullptr, nullptr);
        else if (w == 3) rc = tga_cc(g, TGA_T_MIN, TGA_T_MAX, TGA_CC_EARLY_EXIT, nullptr, nullptr);
        else rc = tga_cc(g, wlo, whi, TGA_CC_EARLY_EXIT, nullptr, nullptr);
        if (rc) return rc;
        if (rep == 1) total += h.timing.total_ms;
      }
    *ms = total;
    return TGA_OK;
  };
  if (cudaStreamSynchronize(h.stream) != cudaSuccess) return fail(TGA_E_CUDA, "stream synchronisation failed");
  tga_tune_result r{};
  r.slice_edges = h.slice_len;
  r.item_edges = h.item_edges;
  r.dense_div = h.dense_div > 0 ? h.dense_div : 1;
  TGA_TRY(probe(&r.default_ms));
  r.best_ms = r.default_ms;
  r.candidates = 1;
  for (int32_t sl : {16, 24, 32, 48})
    for (int32_t it : {128, 256, 512}) {
      if (sl == r.slice_edges && it == r.item_edges) continue;
      TGA_TRY(build_work(h, sl, it));
      double ms = 0;
      TGA_TRY(probe(&ms));
      ++r.candidates;
      if (ms < r.best_ms) {
        r.best_ms = ms;
        r.slice_edges = sl;
        r.item_edges = it;
      }
    }
  const int32_t base_div = r.dense_div;
  for (int32_t dd : {1, 2, 4}) {
    if (dd == base_div) continue;
    h.dense_div = dd;
    TGA_TRY(build_work(h, r.slice_edges, r.item_edges));
    double ms = 0;
    TGA_TRY(probe(&ms));
    ++r.candidates;
    if (ms < r.best_ms) {
      r.best_ms = ms;
      r.dense_div = dd;
    }
  }
  h.dense_div = r.dense_div;
  TGA_TRY(build_work(h, r.slice_edges, r.item_edges));
  if (out) *out = r;
  return TGA_OK;
}

int tga_get_work_params(tga_graph* g, int32_t* slice_edges, int32_t* item_edges, int64_t* slices, int32_t* items) {
  if (!g) return fail(TGA_E_ARG, "null graph");
  if (slice_edges) *slice_edges = g->slice_len;
  if (item_edges) *item_edges = g->item_edges;
  if (slices) *slices = g->nslices;
  if (items) *items = g->nitems;
  return TGA_OK;
}

}  // extern "C"
