// Lean decoder for full sweeps: the per-edge state of one list lives in registers only.
//
// The general cursor (decoder.cuh) carries a reference chain's state in local memory and reads
// every code with two random word loads (peek64), and a whole list is located through two
// Elias-Fano selects (several dependent loads each) before its first code is read.  Sweeps over
// every list (neighbour access, PageRank, HITS, window counts) use this leaner form instead:
//   * the two sequential streams of a list -- its residual gaps (zeta-3) and its timestamp deltas
//     (zeta-2) -- are read through register windows of two 64-bit words that advance one word
//     load at a time (BitWin); multiples and intervals, read once per run, keep random reads;
//   * a whole (short) list is opened from a schedule entry that carries the bit positions of its
//     record and of its timestamps (LeanEntry), so opening costs one coalesced 16-byte load and
//     then the list's own words;
//   * the record's multiples and intervals sections are walked once at open through the same
//     window that then reads the residuals (their lengths give the residual count);
//   * the values a list copies from its reference chain (2.4% of the arcs of the 2M/40M graph, 1.7
//     per copying list on average) are resolved once at load into a side array (copies), read in
//     order like a fourth sub-list, so no reference chain is decoded during a sweep.
// Results are those of EdgeCursor (the same successor order and timestamps): the merge keeps
// MergedIntIterator's rule (equal heads emitted once) and exhausted sub-iterators hold kInf.
#pragma once
#include "sweep.cuh"

namespace tga {

// Lean sweeps: 4 blocks of 256 per SM (up to 64 registers, no local memory).
#define TGA_LEAN_BOUNDS __launch_bounds__(kBlock, 4)

// Schedule entry of a lean sweep: v >= 0 a whole list whose record starts at bit gbit of the
// graph stream and whose timestamps start at bit tbit; v < 0 the slice -(v+1) (positions unused).
// Positions are 48-bit: hi16 = (gbit >> 32) << 16 | (tbit >> 32).
struct LeanEntry {
  int32_t v;
  uint32_t hi16;
  uint32_t glo, tlo;
};

__host__ __device__ inline LeanEntry lean_entry(int32_t v, uint64_t gbit, uint64_t tbit) {
  LeanEntry e;
  e.v = v;
  e.hi16 = (uint32_t)(((gbit >> 32) & 0xFFFF) << 16 | ((tbit >> 32) & 0xFFFF));
  e.glo = (uint32_t)gbit;
  e.tlo = (uint32_t)tbit;
  return e;
}

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
  __device__ __forceinline__ int restore(const GraphView& g, const SliceState& s) {
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
    remaining = s.count;
    return s.count;
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

  // Next (successor, timestamp); false once the entry is exhausted (or on a decode error).
  template <bool kTimes>
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

// A lean schedule as kernels take it.
struct LeanWork {
  const LeanEntry* e;
  int32_t count;
  const SliceState* slices;
  const int32_t* run_first;
};

// Sweep driver over a lean schedule: thread i decodes entry i (the schedule groups entries of equal
// length, so the lanes of a warp finish together).  (Measured against a grid of one to two waves in
// which each thread walks the schedule with the grid's stride and prefetches its next entry: that
// hid more load latency but its lanes fell out of step, and the PageRank pass took 1.26-1.41 ms
// against 1.17 ms.)
// Hooks and kRuns / kTimes / kRunArg as in run_order (sweep.cuh).  kSkip (with kTimes = false):
// edge() returns an int -- 0 stop the list, 1 go on, 2 go on and the edges that repeat this
// successor right after it do not matter to the hook: they are consumed without a merge step or a
// hook call, and count as decoded edges.  (With timestamps the repeats' deltas still have to be
// decoded one by one, and a per-lane skip loop only makes the warp diverge.)
template <bool kRuns = false, bool kTimes = true, bool kRunArg = false, bool kSkip = false, class Want, class Begin,
          class Edge, class End>
__device__ __forceinline__ unsigned long long run_lean(const GraphView& g, const LeanEntry* entries, int count,
                                                       const SliceState* slices, const int32_t* run_first, Want want,
                                                       Begin begin, Edge edge, End end) {
  static_assert(!(kSkip && kTimes), "repeats carry their own timestamps");
  unsigned long long edges = 0;
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= count) return 0;
  const LeanEntry e = entries[i];
  LeanCursor c;
  RunFilter rf;
  int x, first = 0, cnt, lead = kNoRunFilter, run = -1;
  if (e.v >= 0) {
    x = e.v;
    if (!want(x)) return 0;
    const uint64_t gbit = ((uint64_t)(e.hi16 >> 16) << 32) | e.glo;
    const uint64_t tbit = ((uint64_t)(e.hi16 & 0xFFFF) << 32) | e.tlo;
    cnt = c.open(g, x, gbit, tbit);
  } else {
    const SliceState& s = slices[-e.v - 1];
    x = s.v;
    if (!want(x)) return 0;
    cnt = c.restore(g, s);
    first = s.first;
    if (kRuns && s.run >= 0) lead = __ldg(run_first + s.run);
    run = s.run;
  }
  bool go;
  if constexpr (kRunArg) go = cnt > 0 && begin(x, first, cnt, run);
  else go = cnt > 0 && begin(x, first, cnt);
  if (!go) return 0;
  if (kRuns) rf.start(lead, first);
  int y;
  int64_t t;
  while (c.template next<kTimes>(g, y, t)) {
    ++edges;
    const bool pass = !kRuns || rf.pass(y);
    if constexpr (kSkip) {
      if (!pass) continue;
      const int r = edge(x, y, t);
      if (r == 0) break;
      // (a slice inside a run whose kept edge is still ahead goes on edge by edge)
      if (r == 2 && (!kRuns || rf.lead == kNoRunFilter || rf.lead < rf.idx)) {
        const int k = c.skip_repeats(g, y);
        edges += (unsigned)k;
        if (kRuns) rf.idx += k;
      }
    } else {
      if (pass && !edge(x, y, t)) break;
    }
  }
  end(x);
  return edges;
}

// Resolution of the copy masks at load: one thread per list x of `ids` (lists with a reference),
// its copy mask run over the referenced chain with the general decoder.  Pass 1 (out == nullptr)
// stores the count in count[i]; pass 2 writes the values at out + base[x].
static __global__ void k_resolve_copies(GraphView g, const int32_t* ids, int32_t n, uint32_t* count,
                                        const uint32_t* base, int32_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = ids[i];
  DeepState deep;
  EdgeCursor c(&deep);
  if (c.open(g, x) <= 0 || !c.chain) {
    if (!out) count[i] = 0;
    return;
  }
  int h = c.top.hc;
  uint32_t k = 0;
  int32_t* dst = out ? out + base[x] : nullptr;
#pragma unroll 1
  while (h != kInf && k <= (uint32_t)g.max_list) {
    if (dst) dst[k] = h;
    ++k;
    h = deep_copy_next(*g.self, deep);
  }
  if (!out) count[i] = k;
}

// Builds the whole-list entries of a lean schedule: entry i of `ids` (a vertex, or -(slice+1))
// becomes a LeanEntry, with the record and timestamp positions of a vertex looked up in the
// Elias-Fano indexes.
static __global__ void k_lean_entries(GraphView g, const int32_t* ids, int32_t n, LeanEntry* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = ids[i];
  if (v < 0) {
    out[i] = lean_entry(v, 0, 0);
    return;
  }
  out[i] = lean_entry(v, ef_get(g, g.gef, (uint64_t)v), ef_get(g, g.tef, (uint64_t)v));
}

}  // namespace tga
