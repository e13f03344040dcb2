// Device views of a resident compressed temporal graph: bit streams, Elias-Fano offset
// indexes and the word-level code decoders shared by every kernel.
//
// Layout in HBM (built once by the loader):
//   * .graph and .timestamps bytes are stored as 64-bit words in big-endian word order
//     (word i holds stream bytes 8i..8i+7, first byte in the top 8 bits), so bit p of a stream
//     is bit 63-(p&63) of word p>>6 and a 64-bit look-ahead is one funnel shift of two words.
//     Two zero words of padding follow each stream.
//   * EF lower bits are stored the same way (they are MSB-first in the files); EF upper bits
//     keep the files' little-endian word order (LSB-first, as read by the reference's select).
//   * select samples: samples[k] = bit position of the (64k)-th one of the upper bits.
#pragma once
#include <cstdint>

namespace tga {

constexpr int kInf = 0x7fffffff;       // exhausted-iterator marker (never a valid vertex id)
constexpr int kMaxLevels = 4;          // reference chains of depth <= 3 (maxrefcount 3)

// Device error bits (OR-ed into GraphView::err, read back by the host after each call).
enum : uint32_t {
  kErrCursor = 1u,      // a read ran past the end of a stream
  kErrCode = 2u,        // a code longer than the supported window (corrupt stream)
  kErrChain = 4u,       // reference chain deeper than kMaxLevels-1
  kErrId = 8u,          // decoded vertex id outside [0, n)
  kErrCount = 16u,      // a successor list ended before its outdegree was reached
  kErrIndex = 32u,      // EF index lookup outside the index
  kErrTimeout = 64u,    // an iteration cap was reached
};

struct Stream {
  const uint64_t* w;   // big-endian-ordered words
  uint64_t nbits;      // valid bits (file bytes * 8)
  uint64_t nwords;     // words allocated (>= ceil(nbits/64) + 2)
};

struct EFView {
  const uint64_t* lower;    // big-endian-ordered words
  const uint64_t* upper;    // little-endian words
  const uint64_t* samples;  // select samples, one per 64 ones
  uint64_t upper_words;
  uint64_t count;           // number of values
  int l;
};

struct GraphView {
  Stream g, t;
  EFView gef, tef;
  int32_t n;             // vertices in the files (max id + 1)
  int32_t max_label;     // MAX_LABEL of the dataset configuration
  int32_t max_vertex;    // MAX_Vertex (size of per-vertex result arrays)
  int32_t active_begin;  // ACTIVE_VERTEX_BEGIN
  int32_t min_interval;  // minintervallength of the successor format
  int32_t max_list;      // largest outdegree in the graph (bounds every header-driven loop)
  // Slice checkpoints of long lists (slices.cuh), used by the decoder to seek over long skip
  // blocks of a referenced list; null until the work decomposition is built.
  const struct SliceState* slices;
  const struct DeepState* slice_deep;  // chain levels of the checkpoints that have some
  const int32_t* slice_first;
  const int32_t* deg;    // outdegrees (set with the slices)
  int32_t seek_min;      // skip blocks longer than this seek through a checkpoint
  // Device-global copy of this view.  Out-of-line decoder routines take it instead of the kernel
  // parameter, whose address would otherwise force a local-memory copy read by the hot loop.
  const struct GraphView* self;
  int64_t min_ts;        // header of the .timestamps stream
  uint32_t* err;         // device error word
  // Copied values resolved at load: the values that the copy mask of list x selects from its
  // referenced list, in order, are copies[copy_base[x] .. copy_base[x+1]) (empty for a list without
  // a reference).  Read by the lean sweep decoder (lean.cuh) instead of walking the chain.
  const int32_t* copies;
  const uint32_t* copy_base;
  // Hot scatter targets (hot.cuh): a direct-mapped table of kHotSlots vertex ids (-1 empty) and
  // their kHotSlots compact indexes, or null when no vertex qualifies.
  const int32_t* hot;
};

__device__ __forceinline__ void set_err(const GraphView& g, uint32_t bit) { atomicOr(g.err, bit); }

// 64 bits of a stream starting at bit p (MSB-aligned).  Out-of-range word indexes are
// clamped to the zero padding so a corrupt cursor never leaves the allocation.
__device__ __forceinline__ uint64_t peek64(const Stream& s, uint64_t p) {
  uint64_t i = p >> 6;
  const uint64_t last = s.nwords - 2;
  if (i > last) i = last;
  const uint64_t w0 = __ldg(s.w + i), w1 = __ldg(s.w + i + 1);
  const int sh = (int)(p & 63);
  return sh ? (w0 << sh) | (w1 >> (64 - sh)) : w0;
}

// ---- codes on an MSB-aligned 64-bit window ------------------------------------------------
// Each returns the value and adds the code length to *len.  A window of all zeros or a code
// that does not fit in 64 bits flags kErrCode and yields 0.

__device__ __forceinline__ uint64_t win_unary(uint64_t w, int* len) {
  const int z = __clzll(w);
  *len += z + 1;
  return (uint64_t)z;
}

__device__ __forceinline__ uint64_t win_gamma(uint64_t w, int* len, bool* bad) {
  const int m = __clzll(w);          // value+1 has m+1 significant bits
  if (m >= 32) { *bad = true; *len += 1; return 0; }
  const uint64_t v1 = w >> (63 - 2 * m);   // the 2m+1-bit code read as an integer = value + 1
  *len += 2 * m + 1;
  return v1 - 1;
}

template <int K>
__device__ __forceinline__ uint64_t win_zeta(uint64_t w, int* len, bool* bad) {
  const int h = __clzll(w);
  const int nb = h * K + K - 1;
  if (h + 1 + nb + 1 > 64) { *bad = true; *len += 1; return 0; }
  const uint64_t pay = w << (h + 1);       // payload at the top
  const uint64_t left = 1ull << (h * K);
  const uint64_t val = pay >> (64 - nb);   // nb >= K-1 >= 1
  if (val < left) { *len += h + 1 + nb; return val + left - 1; }
  *len += h + 2 + nb;
  return (pay >> (63 - nb)) - 1;
}

__device__ __forceinline__ int64_t d_nat2int(uint64_t x) { return (x & 1) ? -(int64_t)(x >> 1) - 1 : (int64_t)(x >> 1); }

// Random-access readers (two word loads per code).
__device__ __forceinline__ uint64_t read_gamma(const GraphView& g, const Stream& s, uint64_t& p) {
  int len = 0;
  bool bad = false;
  const uint64_t v = win_gamma(peek64(s, p), &len, &bad);
  if (bad) set_err(g, kErrCode);
  p += (uint64_t)len;
  return v;
}
__device__ __forceinline__ uint64_t read_unary(const GraphView& g, const Stream& s, uint64_t& p) {
  const uint64_t w = peek64(s, p);
  if (w == 0) { set_err(g, kErrCode); p += 64; return 0; }
  int len = 0;
  const uint64_t v = win_unary(w, &len);
  p += (uint64_t)len;
  return v;
}
template <int K>
__device__ __forceinline__ uint64_t read_zeta(const GraphView& g, const Stream& s, uint64_t& p) {
  int len = 0;
  bool bad = false;
  const uint64_t v = win_zeta<K>(peek64(s, p), &len, &bad);
  if (bad) set_err(g, kErrCode);
  p += (uint64_t)len;
  return v;
}

// ---- Elias-Fano access ---------------------------------------------------------------------

// Position of the (r+1)-th set bit of w (r < popcount(w)), by halving with population counts.
__device__ __forceinline__ int nth_set_bit64(uint64_t w, int r) {
  int pos = 0;
  uint32_t x = (uint32_t)w;
  int c = __popc(x);
  if (r >= c) {
    r -= c;
    pos = 32;
    x = (uint32_t)(w >> 32);
  }
  for (int half = 16; half >= 2; half >>= 1) {
    c = __popc(x & ((1u << half) - 1u));
    if (r >= c) {
      r -= c;
      pos += half;
      x >>= half;
    }
  }
  return pos + (r >= (int)(x & 1u));
}

// Position of the i-th one (0-based) of the upper bits.  The scan from the sample is bounded by
// the bitmap's end, not by a fixed word count: after a hub's record (5M edges, 190M bits of
// timestamps) the next one lies thousands of words further on.
__device__ __forceinline__ uint64_t ef_select(const GraphView& g, const EFView& e, uint64_t i) {
  uint64_t p = __ldg(e.samples + (i >> 6));
  int r = (int)(i & 63);
  uint64_t wi = p >> 6;
  if (wi >= e.upper_words) {
    set_err(g, kErrIndex);
    return 0;
  }
  uint64_t w = __ldg(e.upper + wi) & (~0ull << (p & 63));
#pragma unroll 1
  for (;;) {
    const int c = __popcll(w);
    if (r < c) return wi * 64 + (uint64_t)nth_set_bit64(w, r);
    r -= c;
    if (++wi >= e.upper_words) break;
    w = __ldg(e.upper + wi);
  }
  set_err(g, kErrIndex);
  return 0;
}

__device__ __forceinline__ uint64_t ef_get(const GraphView& g, const EFView& e, uint64_t i) {
  if (i >= e.count) { set_err(g, kErrIndex); return 0; }
  uint64_t low = 0;
  if (e.l) {
    const uint64_t p = i * (uint64_t)e.l;
    const uint64_t wi = p >> 6;
    const int sh = (int)(p & 63);
    const uint64_t w0 = __ldg(e.lower + wi), w1 = __ldg(e.lower + wi + 1);
    const uint64_t win = sh ? (w0 << sh) | (w1 >> (64 - sh)) : w0;
    low = win >> (64 - e.l);
  }
  const uint64_t high = ef_select(g, e, i) - i;
  return (high << e.l) | low;
}

// Sequential reader with a two-word register window, for streams consumed front to back
// (the timestamps of one list, the residuals of a list).
struct SeqReader {
  const uint64_t* next;  // next word to load
  const uint64_t* end;   // one past the last loadable word
  uint64_t hi, lo;
  int sh;                // bits of hi already consumed
  uint64_t base;         // absolute bit position of hi's first bit

  __device__ __forceinline__ void init(const Stream& s, uint64_t p) {
    uint64_t i = p >> 6;
    const uint64_t last = s.nwords - 2;
    if (i > last) i = last;
    end = s.w + s.nwords;
    hi = __ldg(s.w + i);
    lo = __ldg(s.w + i + 1);
    next = s.w + i + 2;
    sh = (int)(p & 63);
    base = i * 64;
  }
  __device__ __forceinline__ uint64_t window() const { return sh ? (hi << sh) | (lo >> (64 - sh)) : hi; }
  __device__ __forceinline__ void skip(int n) {
    sh += n;
    if (sh >= 64) {
      sh -= 64;
      hi = lo;
      lo = next < end ? __ldg(next) : 0ull;
      ++next;
      base += 64;
    }
  }
  __device__ __forceinline__ uint64_t pos() const { return base + (uint64_t)sh; }
};

}  // namespace tga
