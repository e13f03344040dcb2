// Host-side MSB-first bit streams and the instantaneous codes of the compressed
// temporal-graph format (unary, Elias gamma, zeta_k, minimal binary, int2nat).
//
// The on-disk streams are written exactly like dsiutils' OutputBitStream, which the
// reference encoder uses (BVMultiGraph.java:485-563 write/readResidual, writeBlock;
// EvolvingMultiGraph.java:131-144 writeLongZeta of int2nat(delta)):
//   * bits are packed MSB-first inside each byte, the last byte is zero-padded;
//   * unary(x)   = x zeros followed by a one                      (x+1 bits);
//   * gamma(x)   = unary(msb(x+1)) then the low msb(x+1) bits of x+1;
//   * zeta_k(x)  = unary(h), h = msb(x+1)/k, then x+1-2^(hk) in minimal binary
//                  over [0, 2^(hk)(2^k-1)): hk+k-1 bits if the value is < 2^(hk),
//                  else (value + 2^(hk)) in hk+k bits;
//   * int2nat(x) = 2x for x >= 0, -2x-1 for x < 0 (nat2int is its inverse).
// The decode tables shipped with the reference (gpu_cuda/decode_tables/gammaInA.txt,
// zetaInA.txt) are regenerated from these definitions by table16() and match entry
// for entry.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace tga {

inline int msb64(uint64_t v) { return v ? 63 - __builtin_clzll(v) : -1; }

inline uint64_t int2nat(int64_t x) { return x >= 0 ? (uint64_t)x << 1 : ((uint64_t)(-(x + 1)) << 1) | 1u; }
inline int64_t nat2int(uint64_t n) { return (n & 1) ? -(int64_t)(n >> 1) - 1 : (int64_t)(n >> 1); }

class WordWriter;

class BitWriter {
 public:
  std::vector<uint8_t> bytes;
  uint64_t nbits = 0;

  void reserve_bits(uint64_t b) { bytes.reserve((b + 7) / 8); }

  // Appends the low `len` bits of `v`, most significant first (len <= 64).
  void write_bits(uint64_t v, int len) {
    while (len > 0) {
      const int used = (int)(nbits & 7);
      if (used == 0) bytes.push_back(0);
      const int room = 8 - used;
      const int take = len < room ? len : room;
      const uint64_t chunk = (len == 64 && take == 64) ? v : (v >> (len - take)) & ((1ull << take) - 1);
      bytes.back() |= (uint8_t)(chunk << (room - take));
      nbits += take;
      len -= take;
    }
  }
  int write_unary(uint64_t x) {
    uint64_t z = x;
    while (z >= 32) { write_bits(0, 32); z -= 32; }
    write_bits(1, (int)z + 1);
    return (int)x + 1;
  }
  int write_gamma(uint64_t x) {
    const uint64_t v = x + 1;
    const int m = msb64(v);
    write_unary((uint64_t)m);
    if (m) write_bits(v, m);
    return 2 * m + 1;
  }
  int write_minimal_binary(uint64_t x, uint64_t b) {
    const int lb = msb64(b);
    const uint64_t m = (lb + 1 >= 64 ? 0ull : (1ull << (lb + 1))) - b;
    if (x < m) { if (lb) write_bits(x, lb); return lb; }
    write_bits(x + m, lb + 1);
    return lb + 1;
  }
  int write_zeta(uint64_t x, int k) {
    const uint64_t v = x + 1;
    const int h = msb64(v) / k;
    const int u = write_unary((uint64_t)h);
    const uint64_t left = 1ull << (h * k);
    return u + write_minimal_binary(v - left, (left << k) - left);
  }
  int write_long(uint64_t x, int len) { write_bits(x, len); return len; }
  // Appends all bits of a finished WordWriter.
  inline void append_words(const WordWriter& o);
};

// The same codes written a 64-bit word at a time (MSB-first within each word), for the encoders'
// per-thread streams, which BitWriter::append_words joins into the byte stream; the bits are the
// ones BitWriter writes for the same calls.  finish() before the words are read.
class WordWriter {
 public:
  std::vector<uint64_t> words;  // complete words (after finish(): every bit written)
  uint64_t nbits = 0;

  // Appends the low `len` bits of `v`, most significant first (len <= 64).
  void write_bits(uint64_t v, int len) {
    if (len <= 0) return;
    if (len < 64) v &= (1ull << len) - 1;
    nbits += (uint64_t)len;
    const int room = 64 - pend_;
    if (len < room) {
      acc_ |= v << (room - len);
      pend_ += len;
      return;
    }
    const int rest = len - room;  // bits of v that do not fit in the current word
    acc_ |= rest ? v >> rest : v;
    words.push_back(acc_);
    acc_ = rest ? v << (64 - rest) : 0;
    pend_ = rest;
  }
  int write_unary(uint64_t x) {
    uint64_t z = x;
    while (z >= 32) { write_bits(0, 32); z -= 32; }
    write_bits(1, (int)z + 1);
    return (int)x + 1;
  }
  int write_gamma(uint64_t x) {
    const uint64_t v = x + 1;
    const int m = msb64(v);
    write_unary((uint64_t)m);
    if (m) write_bits(v, m);
    return 2 * m + 1;
  }
  int write_minimal_binary(uint64_t x, uint64_t b) {
    const int lb = msb64(b);
    const uint64_t m = (lb + 1 >= 64 ? 0ull : (1ull << (lb + 1))) - b;
    if (x < m) { if (lb) write_bits(x, lb); return lb; }
    write_bits(x + m, lb + 1);
    return lb + 1;
  }
  int write_zeta(uint64_t x, int k) {
    const uint64_t v = x + 1;
    const int h = msb64(v) / k;
    const int u = write_unary((uint64_t)h);
    const uint64_t left = 1ull << (h * k);
    return u + write_minimal_binary(v - left, (left << k) - left);
  }
  // Moves the pending bits into words (zero-padded); nothing may be written afterwards.
  void finish() {
    if (pend_ > 0) words.push_back(acc_);
    acc_ = 0;
    pend_ = 0;
  }

 private:
  uint64_t acc_ = 0;  // pending bits, in the top pend_ bits
  int pend_ = 0;      // < 64
};

inline void BitWriter::append_words(const WordWriter& o) {
  if (o.nbits == 0) return;
  const int used = (int)(nbits & 7);
  const size_t first = (size_t)(nbits >> 3);  // byte holding bit nbits
  nbits += o.nbits;
  bytes.resize((size_t)((nbits + 7) >> 3), 0);
  uint8_t* d = bytes.data() + first;
  const size_t avail = bytes.size() - first;  // bytes from d on
  const size_t nw = (size_t)((o.nbits + 63) >> 6);
  for (size_t i = 0; i < nw; ++i) {
    const uint64_t x = o.words[i];
    const uint64_t hi = x >> used;                                    // bytes 8i .. 8i+7
    const uint8_t lo = used ? (uint8_t)(x << (8 - used)) : (uint8_t)0;  // top of byte 8i+8
    const size_t at = 8 * i;
    if (at + 9 <= avail) {
      for (int k = 0; k < 8; ++k) d[at + (size_t)k] |= (uint8_t)(hi >> (56 - 8 * k));
      d[at + 8] |= lo;
    } else {
      // The last word: bytes past the end hold only zero padding.
      for (int k = 0; k < 8 && at + (size_t)k < avail; ++k) d[at + (size_t)k] |= (uint8_t)(hi >> (56 - 8 * k));
      if (at + 8 < avail) d[at + 8] |= lo;
    }
  }
}

// Counts bits without storing them (the "NullOutputStream" bit counter of diffComp).
struct BitCounter {
  uint64_t nbits = 0;
  int write_unary(uint64_t x) { nbits += x + 1; return (int)x + 1; }
  int write_gamma(uint64_t x) { const int m = msb64(x + 1); nbits += 2 * m + 1; return 2 * m + 1; }
  int write_zeta(uint64_t x, int k) {
    const uint64_t v = x + 1;
    const int h = msb64(v) / k;
    const uint64_t left = 1ull << (h * k);
    const int len = (v - left < left) ? h * k + k - 1 : h * k + k;
    nbits += h + 1 + len;
    return h + 1 + len;
  }
};

// Sequential MSB-first reader over a byte buffer (host side; used by the loader,
// the EF producer and the index builders, never on the device).
class BitReader {
 public:
  BitReader(const uint8_t* d, uint64_t nbytes, uint64_t pos = 0) : d_(d), nbits_(nbytes * 8), pos_(pos) {}
  uint64_t pos() const { return pos_; }
  void seek(uint64_t p) { pos_ = p; }
  int bit() {
    if (pos_ >= nbits_) throw std::runtime_error("bit stream overrun at bit " + std::to_string(pos_));
    const int b = (d_[pos_ >> 3] >> (7 - (pos_ & 7))) & 1;
    ++pos_;
    return b;
  }
  uint64_t bits(int len) {
    uint64_t v = 0;
    for (int i = 0; i < len; ++i) v = (v << 1) | (uint64_t)bit();
    return v;
  }
  uint64_t unary() {
    uint64_t n = 0;
    while (bit() == 0) ++n;
    return n;
  }
  uint64_t gamma() {
    const uint64_t m = unary();
    if (m > 63) throw std::runtime_error("gamma code too long");
    return ((1ull << m) | bits((int)m)) - 1;
  }
  uint64_t zeta(int k) {
    const uint64_t h = unary();
    if (h * k + k > 64) throw std::runtime_error("zeta code too long");
    const uint64_t left = 1ull << (h * k);
    const uint64_t val = bits((int)(h * k + k - 1));
    if (val < left) return val + left - 1;
    return ((val << 1) | (uint64_t)bit()) - 1;
  }

 private:
  const uint8_t* d_;
  uint64_t nbits_;
  uint64_t pos_;
};

// Word-at-a-time MSB-first reader for long host-side walks (same codes as BitReader): a 64-bit
// look-ahead from any bit, clz for unary prefixes.  The buffer is read through a copy padded with
// 16 zero bytes, so look-ahead past the end reads zeros; running past the end throws.
class FastBitReader {
 public:
  FastBitReader(const std::vector<uint8_t>& d, uint64_t pos = 0) : d_(d), nbits_((uint64_t)d.size() * 8), pos_(pos) {
    d_.resize(d.size() + 16, 0);
  }
  uint64_t pos() const { return pos_; }
  void seek(uint64_t p) { pos_ = p; }
  uint64_t peek64() const {
    const uint64_t byte = pos_ >> 3;
    const int sh = (int)(pos_ & 7);
    uint64_t w = 0;
    for (int i = 0; i < 8; ++i) w = (w << 8) | d_[byte + (uint64_t)i];
    return sh ? (w << sh) | (uint64_t)(d_[byte + 8] >> (8 - sh)) : w;
  }
  void skip(uint64_t n) {
    pos_ += n;
    if (pos_ > nbits_) throw std::runtime_error("bit stream overrun at bit " + std::to_string(pos_));
  }
  uint64_t bits(int len) {
    if (len == 0) return 0;
    const uint64_t v = peek64() >> (64 - len);
    skip((uint64_t)len);
    return v;
  }
  uint64_t unary() {
    uint64_t n = 0;
    for (;;) {
      if (pos_ >= nbits_) throw std::runtime_error("bit stream overrun at bit " + std::to_string(pos_));
      const uint64_t w = peek64();
      if (w) {
        const int z = __builtin_clzll(w);
        skip((uint64_t)z + 1);
        return n + (uint64_t)z;
      }
      n += 64;
      skip(64);
    }
  }
  uint64_t gamma() {
    const uint64_t m = unary();
    if (m > 63) throw std::runtime_error("gamma code too long");
    return ((1ull << m) | bits((int)m)) - 1;
  }
  uint64_t zeta(int k) {
    const uint64_t h = unary();
    if (h * k + k > 64) throw std::runtime_error("zeta code too long");
    const uint64_t left = 1ull << (h * k);
    const uint64_t val = bits((int)(h * k + k - 1));
    if (val < left) return val + left - 1;
    return ((val << 1) | bits(1)) - 1;
  }

 private:
  std::vector<uint8_t> d_;
  uint64_t nbits_;
  uint64_t pos_;
};

// 16-bit look-ahead table in the reference's layout: entry w = (code length << 16) |
// value for the code that starts at the top of the 16-bit window w, 0 when the code
// does not fit in 16 bits.  kind 0 = gamma, kind 3 = zeta_3.
inline std::vector<int32_t> table16(int kind) {
  std::vector<int32_t> t(65536, 0);
  for (uint32_t w = 0; w < 65536; ++w) {
    uint8_t buf[4] = {(uint8_t)(w >> 8), (uint8_t)w, 0, 0};
    BitReader r(buf, 4);
    uint64_t v;
    try { v = kind == 0 ? r.gamma() : r.zeta(kind); } catch (...) { continue; }
    if (r.pos() <= 16 && v < 65536) t[w] = (int32_t)((r.pos() << 16) | v);
  }
  return t;
}

}  // namespace tga
