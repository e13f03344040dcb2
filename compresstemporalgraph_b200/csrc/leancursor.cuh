// Register-only decoder of one successor list (or one slice of it) with its timestamps, shared by
// every sweep and traversal kernel:
//   * the two sequential streams of a list -- its residual gaps (zeta-3) and its timestamp deltas
//     (zeta-2) -- are read through register windows (BitWin) that advance one word load at a
//     time; multiples and intervals, read once per run, use random reads (peek64);
//   * the record's multiples and intervals sections are walked once at open through the same
//     window that then reads the residuals (their lengths give the residual count);
//   * the values a list copies from its reference chain (2.4% of the arcs of the 2M/40M graph, 1.7
//     per copying list on average) are resolved once at load into a side array
//     (GraphView::copies), read in order like a fourth sub-list, so no reference chain is decoded
//     and the decoder keeps no state in local memory.
// Results are those of EdgeCursor (decoder.cuh), which stays for the checkpoint builder and the
// copy resolution: the same successor order and timestamps, MergedIntIterator's rule (equal heads
// emitted once), kInf in exhausted sub-iterators.
#pragma once
#include "decoder.cuh"

namespace tga {

// Sequential reader over a big-endian word stream (the graph stream, or the timestamps with
// kTs): the next 64 bits at any point are one funnel shift of two registers, and a third register
// holds the word after them, so the load that refills the window is issued a whole word (a code
// or two) before its bits are needed.  Loads are clamped to the stream's allocation, whose two
// trailing words are zero padding.
template <bool kTs>
struct BitWin {
  const uint64_t* p;  // next word to load
  uint64_t a, b, c;   // current word and the two after it
  int sh;             // bits of a already consumed (0..63)

  __device__ __forceinline__ static const Stream& st(const GraphView& g) { return kTs ? g.t : g.g; }
  __device__ __forceinline__ static uint64_t load(const GraphView& g, const uint64_t* q) {
    const Stream& s = st(g);
    return q < s.w + s.nwords ? __ldg(q) : 0ull;
  }
  __device__ __forceinline__ void init(const GraphView& g, uint64_t pos) {
    const Stream& s = st(g);
    uint64_t i = pos >> 6;
    const uint64_t last = s.nwords - 2;
    if (i > last) i = last;
    const uint64_t* q = s.w + i;
    a = __ldg(q);
    b = __ldg(q + 1);
    c = load(g, q + 2);
    p = q + 3;
    sh = (int)(pos & 63);
  }
  __device__ __forceinline__ uint64_t window() const {
    // (b >> 1) >> (63 - sh) is b >> (64 - sh) for sh > 0 and 0 for sh == 0, with no branch.
    return (a << sh) | ((b >> 1) >> (63 - sh));
  }
  __device__ __forceinline__ void skip(const GraphView& g, int n) {  // n <= 64
    sh += n;
    if (sh >= 64) {
      sh -= 64;
      a = b;
      b = c;
      c = load(g, p);
      ++p;
    }
  }
  // Absolute bit position of the next unread bit.
  __device__ __forceinline__ uint64_t pos(const GraphView& g) const {
    return ((uint64_t)(p - st(g).w) - 3) * 64 + (uint64_t)sh;
  }
  __device__ __forceinline__ uint64_t gamma(const GraphView& g) {
    int len = 0;
    bool bad = false;
    const uint64_t v = win_gamma(window(), &len, &bad);
    if (bad) set_err(g, kErrCode);
    skip(g, len);
    return v;
  }
  __device__ __forceinline__ uint64_t unary(const GraphView& g) {
    const uint64_t w = window();
    if (w == 0) {
      set_err(g, kErrCode);
      skip(g, 64);
      return 0;
    }
    int len = 0;
    const uint64_t v = win_unary(w, &len);
    skip(g, len);
    return v;
  }
  template <int K>
  __device__ __forceinline__ uint64_t zeta(const GraphView& g) {
    int len = 0;
    bool bad = false;
    const uint64_t v = win_zeta<K>(window(), &len, &bad);
    if (bad) set_err(g, kErrCode);
    skip(g, len);
    return v;
  }
};

// One list (or slice) being decoded: merge of multiples, intervals, residuals and the values its
// copy mask selects from the referenced list, read from the copies resolved at load
// (GraphView::copies), so no reference chain is walked.
struct LeanCursor {
  int hm, mrem, mleft;
  int hi, iend, ileft;
  int hr, rleft;
  int hc;              // copied-values head
  uint32_t cnext, cend;// next copied value to load, end of the list's copied values
  uint64_t mpos, ipos; // next multiples / intervals codes
  BitWin<false> rr;    // residual gaps
  BitWin<true> tr;     // timestamp deltas
  int64_t prev;
  int remaining;

  // Whole list x from its record at gbit and its timestamps at tbit; returns the outdegree.
  __device__ __forceinline__ int open(const GraphView& g, int x, uint64_t gbit, uint64_t tbit) {
    hm = hi = hr = hc = kInf;
    remaining = 0;
    rr.init(g, gbit);
    const int d = (int)rr.gamma(g);
    if (d <= 0) return 0;
    if (d > g.max_list) {
      set_err(g, kErrCode);
      return 0;
    }
    int extra = d;
    if (rr.unary(g) != 0) {
      // Copy blocks: skipped here (their selection is resolved in GraphView::copies).
      const int bc = (int)rr.gamma(g);
      if (bc < 0 || bc > 2 * d + 2 * g.max_list + 1) {
        set_err(g, kErrCode);
        return 0;
      }
#pragma unroll 1
      for (int i = 0; i < bc; ++i) rr.gamma(g);
      const uint32_t c0 = __ldg(g.copy_base + x), c1 = __ldg(g.copy_base + x + 1);
      cend = c1;
      cnext = c0 + 1;
      if (c0 < c1) hc = __ldg(g.copies + c0);
      extra = d - (int)(c1 - c0);
    }
    if (extra > 0) {
      const int mc = (int)rr.gamma(g);
      if (mc < 0 || mc > d) {
        set_err(g, kErrCode);
        return 0;
      }
      if (mc) {
        hm = x + (int)d_nat2int(rr.gamma(g));
        mrem = (int)rr.gamma(g) + 2;
        mleft = mc - 1;
        extra -= mrem;
        mpos = rr.pos(g);
#pragma unroll 1
        for (int i = 1; i < mc; ++i) {
          rr.gamma(g);
          extra -= (int)rr.gamma(g) + 2;
        }
      }
    }
    if (extra > 0) {
      const int ic = (int)rr.gamma(g);
      if (ic < 0 || ic > d) {
        set_err(g, kErrCode);
        return 0;
      }
      if (ic) {
        hi = x + (int)d_nat2int(rr.gamma(g));
        const int len = (int)rr.gamma(g) + g.min_interval;
        iend = hi + len;
        ileft = ic - 1;
        extra -= len;
        ipos = rr.pos(g);
#pragma unroll 1
        for (int i = 1; i < ic; ++i) {
          rr.gamma(g);
          extra -= (int)rr.gamma(g) + g.min_interval;
        }
      }
    }
    if (extra > 0) {
      rleft = extra;
      hr = x + (int)d_nat2int(rr.template zeta<3>(g));
    }
    tr.init(g, tbit);
    prev = g.min_ts;
    remaining = d;
    return d;
  }

  // Slice s (its checkpoint holds the complete state at its first edge; at level 0 its `emitted`
  // counts the copied values consumed before it).
  // count >= 0: decode that many edges from the checkpoint (the whole list from its first slice).
  __device__ __forceinline__ int restore(const GraphView& g, const SliceState& s, int count = -1) {
    const ListState& t = s.top;
    hm = t.hm;
    mrem = t.mrem;
    mleft = t.mleft;
    mpos = t.mpos;
    hi = t.hi;
    iend = t.iend;
    ileft = t.ileft;
    ipos = t.ipos;
    hr = t.hr;
    rleft = t.rleft;
    hc = t.hc;
    if (s.chain) {
      cnext = __ldg(g.copy_base + s.v) + (uint32_t)t.emitted + 1;
      cend = __ldg(g.copy_base + s.v + 1);
    }
    if (hr != kInf) rr.init(g, t.rpos);
    tr.init(g, s.tpos);
    prev = s.prev;
    remaining = count >= 0 ? count : s.count;
    return remaining;
  }

  // Whole list of vertex x (ids past the files' vertex count have empty lists): a sliced list from
  // its first checkpoint (walking a hub's record would read its whole multiples section), any
  // other from its record, located through the Elias-Fano indexes.
  __device__ __forceinline__ int open_vertex(const GraphView& g, int x) {
    remaining = 0;
    if (x < 0 || x >= g.n) {
      if (x < 0) set_err(g, kErrId);
      return 0;
    }
    if (const SliceState* cp = first_checkpoint(g, x)) return restore(g, *cp, __ldg(g.deg + x));
    return open(g, x, ef_get(g, g.gef, (uint64_t)x), ef_get(g, g.tef, (uint64_t)x));
  }

  __device__ __forceinline__ void next_multiples_run(const GraphView& g) {
    if (mleft > 0) {
      hm += (int)read_gamma(g, g.g, mpos) + 1;
      mrem = (int)read_gamma(g, g.g, mpos) + 2;
      --mleft;
    } else {
      hm = kInf;
    }
  }

  __device__ __forceinline__ int next_successor(const GraphView& g) {
    const int v = min(min(hm, hi), min(hr, hc));
    if (v == kInf) return kInf;
    if (hm == v && --mrem == 0) next_multiples_run(g);
    if (hi == v && ++hi == iend) {
      if (ileft > 0) {
        hi = iend + (int)read_gamma(g, g.g, ipos) + 1;
        iend = hi + (int)read_gamma(g, g.g, ipos) + g.min_interval;
        --ileft;
      } else {
        hi = kInf;
      }
    }
    if (hr == v) {
      if (--rleft > 0) hr += (int)rr.template zeta<3>(g) + 1;
      else hr = kInf;
    }
    if (hc == v) hc = cnext < cend ? __ldg(g.copies + cnext++) : kInf;
    return v;
  }

  // After next() returned y: when the edges that follow repeat y from its multiples run (hm == y
  // with mrem copies left; intervals and residuals are strictly increasing, so only a copied value
  // equal to y could interleave), consumes them (at most the entry's remaining edges) and returns
  // how many.  For sweeps that read no timestamps.
  __device__ __forceinline__ int skip_repeats(const GraphView& g, int y) {
    if (hm != y || hc == y) return 0;
    const int k = min(mrem, remaining);
    remaining -= k;
    mrem -= k;
    if (mrem == 0) next_multiples_run(g);
    return k;
  }

  // Successor-only state (no timestamp window) for a later resume_successors(): the heads and
  // stream positions in t, the copied-values cursor in cn / ce.
  __device__ __forceinline__ void save_successors(const GraphView& g, ListState& t, uint32_t& cn, uint32_t& ce) const {
    t.mpos = mpos;
    t.ipos = ipos;
    t.rpos = hr != kInf ? rr.pos(g) : 0;
    t.hm = hm;
    t.hi = hi;
    t.hr = hr;
    t.hc = hc;
    t.mleft = mleft;
    t.mrem = mrem;
    t.ileft = ileft;
    t.iend = iend;
    t.rleft = rleft;
    cn = cnext;
    ce = cend;
  }
  __device__ __forceinline__ void resume_successors(const GraphView& g, const ListState& t, uint32_t cn, uint32_t ce,
                                                    int count) {
    hm = t.hm;
    mrem = t.mrem;
    mleft = t.mleft;
    mpos = t.mpos;
    hi = t.hi;
    iend = t.iend;
    ileft = t.ileft;
    ipos = t.ipos;
    hr = t.hr;
    rleft = t.rleft;
    hc = t.hc;
    cnext = cn;
    cend = ce;
    if (hr != kInf) rr.init(g, t.rpos);
    prev = 0;
    remaining = count;
  }

  // Next (successor, timestamp); false once the entry is exhausted (or on a decode error).
  template <bool kTimes = true>
  __device__ __forceinline__ bool next(const GraphView& g, int& y, int64_t& t) {
    if (remaining <= 0) return false;
    --remaining;
    y = next_successor(g);
    if (kTimes) {
      prev += d_nat2int(tr.template zeta<2>(g));
      t = prev;
    } else {
      t = 0;
    }
    if ((unsigned)y >= (unsigned)g.n) {
      set_err(g, y == kInf ? kErrCount : kErrId);
      remaining = 0;
      return false;
    }
    return true;
  }
};

}  // namespace tga
