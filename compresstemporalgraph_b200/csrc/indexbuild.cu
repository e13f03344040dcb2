// Device-side rebuild of the offset index from what the Java encoder writes (BVMultiGraph.java's
// store: <base>.offsets holds the gamma-coded gaps between the bit offsets of consecutive graph
// records; the timestamp stream holds, after its 64-bit header, each list's outdegree-many zeta_2
// codes with no per-list header): the bit offset of every graph record and of every list's first
// timestamp code, from which the host packs the Elias-Fano files.  The host form of the same walk
// is index_from_offsets (format.cpp); this one runs the two sequential walks in parallel.
//
// Both walks read one long stream of self-delimiting codes with no synchronisation points, so
// they are decoded speculatively in chunks of kChunkBits bits (Klein and Wiseman's parallel
// decoding of prefix codes; Weissenberger and Schmidt, "Massively Parallel Huffman Decoding on
// GPUs", ICPP 2018):
//   1. every chunk is decoded by one thread from its first bit as if a code started there, up to
//      the first code boundary at or past its end (its exit), counting codes and summing values;
//   2. a chunk whose assumed entry differs from its predecessor's exit is decoded again from that
//      exit; a wrong entry parses garbage for a few codes and then falls into step with the true
//      boundaries (the codes resynchronise), so its exit is right, and this repeats until no entry
//      changes (two or three rounds in practice; bounded, after which the caller uses the host walk);
//   3. with every entry right, prefix sums of the counts and values give each chunk its first code
//      index and running sum, and every chunk is decoded once more to write its offsets.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"

namespace tga {

namespace {

constexpr uint64_t kChunkBits = 4096;
constexpr int kMaxSyncRounds = 64;

struct ChunkRun {
  uint64_t exit;  // first code boundary at or past the chunk's end
  uint64_t sum;   // sum of the values decoded (gamma walk)
  uint32_t count; // codes that start inside the chunk
  uint32_t pad;
};

// One code at bit pos of s (kZeta: zeta_2, else gamma): its value, and its length in len.  A
// window that holds no valid code (a speculative position that is not a code start) counts as a
// one-bit code.
template <bool kZeta>
__device__ __forceinline__ uint64_t code_at(const Stream& s, uint64_t pos, int& len) {
  const uint64_t w = peek64(s, pos);
  len = 0;
  bool bad = false;
  const uint64_t v = kZeta ? win_zeta<2>(w, &len, &bad) : win_gamma(w, &len, &bad);
  if (bad || len <= 0) len = 1;
  return bad ? 0 : v;
}

template <bool kZeta>
__global__ void k_chunk_runs(Stream s, uint64_t start, uint64_t end, uint32_t nchunks, const uint64_t* entry,
                             const uint8_t* redo, ChunkRun* out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks || (redo && !redo[c])) return;
  uint64_t pos = entry[c];
  const uint64_t stop = min(start + (uint64_t)(c + 1) * kChunkBits, end);
  uint64_t sum = 0;
  uint32_t count = 0;
  // every step advances pos by at least one bit, so at most kChunkBits + 64 steps
  while (pos < stop) {
    int len;
    sum += code_at<kZeta>(s, pos, len);
    pos += (uint64_t)len;
    ++count;
  }
  out[c] = ChunkRun{pos, sum, count, 0};
}

// Entries from the predecessors' exits; redo[c] = 1 (and *changed) where an entry moved.
__global__ void k_chunk_sync(uint32_t nchunks, uint64_t* entry, const ChunkRun* out, uint8_t* redo, uint32_t* changed) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint8_t r = 0;
  if (c > 0 && entry[c] != out[c - 1].exit) {
    entry[c] = out[c - 1].exit;
    r = 1;
    atomicOr(changed, 1u);
  }
  redo[c] = r;
}

// Graph record offsets: code k of the offsets stream is the gap to record k's offset, so
// offset[k] = (sum of codes 0..k).
__global__ void k_emit_graph(Stream s, uint64_t start, uint64_t end, uint32_t nchunks, const uint64_t* entry,
                             const uint64_t* kbase, const uint64_t* sbase, uint64_t total, uint64_t* goff) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint64_t pos = entry[c], k = kbase[c], acc = sbase[c];
  const uint64_t stop = min(start + (uint64_t)(c + 1) * kChunkBits, end);
  while (pos < stop && k < total) {
    int len;
    acc += code_at<false>(s, pos, len);
    goff[k++] = acc;
    pos += (uint64_t)len;
  }
}

// Outdegree of every record: the first gamma code of record v (empty records have degree 0).
__global__ void k_record_degrees(Stream g, const uint64_t* goff, int64_t n, int64_t* deg) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  int64_t d = 0;
  if (goff[v + 1] > goff[v]) {
    int len = 0;
    bool bad = false;
    d = (int64_t)win_gamma(peek64(g, goff[v]), &len, &bad);
    if (bad) d = -1;
  }
  deg[v] = d;
}

// Timestamp offsets: list v starts at code D[v] (D: exclusive prefix of the outdegrees, D[n] =
// total), so toff[v] is the position of code D[v], or the stream's final position for D[v] = total.
__global__ void k_emit_ts(Stream s, uint64_t start, uint64_t end, uint32_t nchunks, const uint64_t* entry,
                          const uint64_t* kbase, const int64_t* D, int64_t n, uint64_t total, uint64_t* toff) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint64_t pos = entry[c], k = kbase[c];
  if (k >= total && c > 0) return;
  const uint64_t stop = min(start + (uint64_t)(c + 1) * kChunkBits, end);
  // first list whose first code is k or later
  int64_t lo = 0, hi = n + 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((uint64_t)D[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  int64_t v = lo;
  while (pos < stop && k < total) {
    while (v <= n && (uint64_t)D[v] == k) toff[v++] = pos;
    int len;
    code_at<true>(s, pos, len);
    pos += (uint64_t)len;
    ++k;
  }
  if (k == total)
    while (v <= n) toff[v++] = pos;
}

struct DeviceStream {
  DevBuf buf;
  Stream s{};
  int up(const std::vector<uint8_t>& bytes, cudaStream_t st) {
    // big-endian 64-bit words, as the loader uploads the streams (two words of zero padding;
    // the host is little-endian, which engine.cu checks)
    const size_t nw = (bytes.size() + 7) / 8 + 2;
    std::vector<uint64_t> w(nw, 0);
    if (!bytes.empty()) std::memcpy(w.data(), bytes.data(), bytes.size());
    for (size_t i = 0; i + 2 < nw; ++i) w[i] = __builtin_bswap64(w[i]);
    if (int rc = buf.ensure(nw * 8)) return rc;
    TGA_CUDA_TRY(cudaMemcpyAsync(buf.p, w.data(), nw * 8, cudaMemcpyHostToDevice, st));
    TGA_CUDA_TRY(cudaStreamSynchronize(st));
    s = Stream{buf.as<uint64_t>(), (uint64_t)bytes.size() * 8, nw};
    return TGA_OK;
  }
};

// Steps 1 and 2 over [start, end) of s: the true entry of every chunk (entry), with the runs
// decoded from it (out).  Returns TGA_E_TIMEOUT when the entries have not settled after
// kMaxSyncRounds rounds.
template <bool kZeta>
int settle_chunks(const Stream& s, uint64_t start, uint64_t end, uint32_t nchunks, DevBuf& entry, DevBuf& out,
                  DevBuf& redo, DevBuf& flag, cudaStream_t st) {
  if (int rc = entry.ensure((size_t)nchunks * 8)) return rc;
  if (int rc = out.ensure((size_t)nchunks * sizeof(ChunkRun))) return rc;
  if (int rc = redo.ensure(nchunks)) return rc;
  if (int rc = flag.ensure(8)) return rc;
  std::vector<uint64_t> e0(nchunks);
  for (uint32_t c = 0; c < nchunks; ++c) e0[c] = start + (uint64_t)c * kChunkBits;
  TGA_CUDA_TRY(cudaMemcpyAsync(entry.p, e0.data(), (size_t)nchunks * 8, cudaMemcpyHostToDevice, st));
  const unsigned grid = (unsigned)((nchunks + 255) / 256);
  k_chunk_runs<kZeta><<<grid, 256, 0, st>>>(s, start, end, nchunks, entry.as<uint64_t>(), nullptr, out.as<ChunkRun>());
  TGA_CUDA_TRY(cudaGetLastError());
  for (int round = 0; round < kMaxSyncRounds; ++round) {
    TGA_CUDA_TRY(cudaMemsetAsync(flag.p, 0, 4, st));
    k_chunk_sync<<<grid, 256, 0, st>>>(nchunks, entry.as<uint64_t>(), out.as<ChunkRun>(), redo.as<uint8_t>(),
                                        flag.as<uint32_t>());
    uint32_t changed = 0;
    TGA_CUDA_TRY(cudaMemcpyAsync(&changed, flag.p, 4, cudaMemcpyDeviceToHost, st));
    TGA_CUDA_TRY(cudaStreamSynchronize(st));
    if (!changed) return TGA_OK;
    k_chunk_runs<kZeta><<<grid, 256, 0, st>>>(s, start, end, nchunks, entry.as<uint64_t>(), redo.as<uint8_t>(),
                                              out.as<ChunkRun>());
    TGA_CUDA_TRY(cudaGetLastError());
  }
  return fail(TGA_E_TIMEOUT, "speculative index walk did not settle");
}

}  // namespace

// goff[0..n] and toff[0..n] as index_from_offsets computes them (toff from bit 64 of the
// timestamp stream, after its header).  Errors leave the vectors unspecified.
int offsets_on_device(const std::vector<uint8_t>& graph, const std::vector<uint8_t>& offsets,
                      const std::vector<uint8_t>& timestamps, int64_t n, std::vector<uint64_t>& goff,
                      std::vector<uint64_t>& toff) {
  if (n <= 0) return fail(TGA_E_FORMAT, "vertex count needed (the nodes property)");
  if (timestamps.size() < 8) return fail(TGA_E_FORMAT, "timestamps file shorter than its 64-bit header");
  cudaStream_t st = nullptr;
  TGA_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{st};
  DeviceStream ds_off, ds_g, ds_t;
  DevBuf entry, out, redo, flag, d_goff, d_deg, d_D, d_toff, d_kb, d_sb;
  int rc;
  if ((rc = ds_off.up(offsets, st)) || (rc = ds_g.up(graph, st)) || (rc = ds_t.up(timestamps, st))) return rc;

  // Graph record offsets: n + 1 gamma codes from bit 0 of the offsets stream.
  const uint64_t oend = ds_off.s.nbits;
  const uint32_t ochunks = (uint32_t)std::max<uint64_t>(1, (oend + kChunkBits - 1) / kChunkBits);
  if ((rc = settle_chunks<false>(ds_off.s, 0, oend, ochunks, entry, out, redo, flag, st))) return rc;
  std::vector<ChunkRun> runs(ochunks);
  TGA_CUDA_TRY(cudaMemcpyAsync(runs.data(), out.p, (size_t)ochunks * sizeof(ChunkRun), cudaMemcpyDeviceToHost, st));
  TGA_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<uint64_t> kb(ochunks), sb(ochunks);
  uint64_t k = 0, acc = 0;
  for (uint32_t c = 0; c < ochunks; ++c) {
    kb[c] = k;
    sb[c] = acc;
    k += runs[c].count;
    acc += runs[c].sum;
  }
  const uint64_t ncodes = (uint64_t)n + 1;
  if (k < ncodes) return fail(TGA_E_FORMAT, "offsets stream holds fewer codes than nodes + 1");
  if ((rc = d_kb.ensure((size_t)ochunks * 8)) || (rc = d_sb.ensure((size_t)ochunks * 8)) ||
      (rc = d_goff.ensure((size_t)ncodes * 8)))
    return rc;
  TGA_CUDA_TRY(cudaMemcpyAsync(d_kb.p, kb.data(), (size_t)ochunks * 8, cudaMemcpyHostToDevice, st));
  TGA_CUDA_TRY(cudaMemcpyAsync(d_sb.p, sb.data(), (size_t)ochunks * 8, cudaMemcpyHostToDevice, st));
  k_emit_graph<<<(ochunks + 255) / 256, 256, 0, st>>>(ds_off.s, 0, oend, ochunks, entry.as<uint64_t>(),
                                                      d_kb.as<uint64_t>(), d_sb.as<uint64_t>(), ncodes,
                                                      d_goff.as<uint64_t>());
  TGA_CUDA_TRY(cudaGetLastError());
  goff.assign((size_t)ncodes, 0);
  TGA_CUDA_TRY(cudaMemcpyAsync(goff.data(), d_goff.p, (size_t)ncodes * 8, cudaMemcpyDeviceToHost, st));
  TGA_CUDA_TRY(cudaStreamSynchronize(st));
  for (uint64_t v = 1; v < ncodes; ++v)
    if (goff[v] < goff[v - 1]) return fail(TGA_E_FORMAT, "offsets decrease");
  if (goff.back() > (uint64_t)graph.size() * 8) return fail(TGA_E_FORMAT, "offsets point past the end of the graph stream");

  // Outdegrees, their exclusive prefix (the first timestamp code of every list).
  if ((rc = d_deg.ensure((size_t)n * 8))) return rc;
  k_record_degrees<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ds_g.s, d_goff.as<uint64_t>(), n, d_deg.as<int64_t>());
  TGA_CUDA_TRY(cudaGetLastError());
  std::vector<int64_t> D((size_t)n + 1);
  TGA_CUDA_TRY(cudaMemcpyAsync(D.data(), d_deg.p, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
  TGA_CUDA_TRY(cudaStreamSynchronize(st));
  int64_t total = 0;
  for (int64_t v = 0; v < n; ++v) {
    const int64_t d = D[(size_t)v];
    if (d < 0) return fail(TGA_E_FORMAT, "bad outdegree code in record " + std::to_string(v));
    D[(size_t)v] = total;
    total += d;
  }
  D[(size_t)n] = total;

  // Timestamp offsets: `total` zeta_2 codes from bit 64.
  const uint64_t tstart = 64, tend = ds_t.s.nbits;
  const uint32_t tchunks = (uint32_t)std::max<uint64_t>(1, (tend - tstart + kChunkBits - 1) / kChunkBits);
  if ((rc = settle_chunks<true>(ds_t.s, tstart, tend, tchunks, entry, out, redo, flag, st))) return rc;
  runs.resize(tchunks);
  TGA_CUDA_TRY(cudaMemcpyAsync(runs.data(), out.p, (size_t)tchunks * sizeof(ChunkRun), cudaMemcpyDeviceToHost, st));
  TGA_CUDA_TRY(cudaStreamSynchronize(st));
  kb.resize(tchunks);
  k = 0;
  for (uint32_t c = 0; c < tchunks; ++c) {
    kb[c] = k;
    k += runs[c].count;
  }
  if (k < (uint64_t)total) return fail(TGA_E_FORMAT, "timestamp stream holds fewer codes than the outdegrees sum to");
  if ((rc = d_kb.ensure((size_t)tchunks * 8)) || (rc = d_D.ensure(((size_t)n + 1) * 8)) ||
      (rc = d_toff.ensure(((size_t)n + 1) * 8)))
    return rc;
  TGA_CUDA_TRY(cudaMemcpyAsync(d_kb.p, kb.data(), (size_t)tchunks * 8, cudaMemcpyHostToDevice, st));
  TGA_CUDA_TRY(cudaMemcpyAsync(d_D.p, D.data(), ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, st));
  if (total == 0) {
    toff.assign((size_t)n + 1, tstart);
    return TGA_OK;
  }
  k_emit_ts<<<(tchunks + 255) / 256, 256, 0, st>>>(ds_t.s, tstart, tend, tchunks, entry.as<uint64_t>(),
                                                   d_kb.as<uint64_t>(), d_D.as<int64_t>(), n, (uint64_t)total,
                                                   d_toff.as<uint64_t>());
  TGA_CUDA_TRY(cudaGetLastError());
  toff.assign((size_t)n + 1, 0);
  TGA_CUDA_TRY(cudaMemcpyAsync(toff.data(), d_toff.p, ((size_t)n + 1) * 8, cudaMemcpyDeviceToHost, st));
  TGA_CUDA_TRY(cudaStreamSynchronize(st));
  return TGA_OK;
}

}  // namespace tga
