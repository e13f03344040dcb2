// Successor-list decoder for one vertex, bit-exact with the Java iterator stack that defines
// the format:
//   BVMultiGraph.successors (BVMultiGraph.java:738-886): outdegree, reference, copy blocks,
//     multiples, intervals, residuals;
//   webgraph MaskedIntIterator (copy/skip blocks over the referenced list, last block implicit),
//   MergedIntIterator (sorted merge, equal heads emitted once), IntIntervalSequenceIterator,
//   IntMultiplesSequenceIterator (IntMultiplesSequenceIterator.java:106-126),
//   ResidualIntIterator (BVMultiGraph.java:655-707);
//   EvolvingMultiGraph.SuccessorIterator (EvolvingMultiGraph.java:396-443) for timestamps.
//
// A reference chain of depth <= 3 is decoded with one state block per level; levels are
// template parameters so every field access is static.  The referenced lists are decoded only
// as far as the copy mask needs them.  Exhausted sub-iterators hold kInf, which is never a
// vertex id (the reference decoder uses MAX_LABEL and breaks on a successor equal to it,
// gpu_cuda/shared/bfs.cu:763-776).
#pragma once
#include "dview.cuh"

namespace tga {

struct LevelState {
  uint64_t mpos, ipos, rpos, bpos;
  int hm, hi, hr, hc;        // heads of multiples, intervals, residuals, copied values
  int mleft, mrem;           // multiples runs still to read, copies left of the current run
  int ileft, iend;           // intervals still to read, end (exclusive) of the current one
  int rleft;                 // residuals left including the head
  int bleft, cur_left;       // copy blocks still to read, values left in the current copy block
                             // (-1: copy everything that remains)
  int x;                     // vertex whose list this level decodes
  int emitted;               // values of this list returned so far
};

struct ChainState {
  LevelState lv[kMaxLevels];
};

// Complete decoder state at one edge of a long list (see slices.cuh).
struct SliceState {
  ChainState cs;
  uint64_t tpos;    // bit position of the slice's first timestamp code
  int64_t prev;     // timestamp preceding the slice's first edge
  int32_t v;        // vertex
  int32_t count;    // edges in the slice
  int32_t first;    // index of the slice's first edge in the list of v
  int32_t pad;
};

template <int L>
__device__ __forceinline__ int list_next(const GraphView& g, ChainState& s);

// Skips k values of the list decoded at level L.  A long skip over a list that has slice
// checkpoints restores the last checkpoint at or before the target (its levels 0.. become levels
// L.. here: a list referenced at level L has a chain of at most kMaxLevels-1-L further levels),
// so the walk is bounded by one slice instead of the skip length.
template <int L>
__device__ __forceinline__ void skip_values(const GraphView& g, ChainState& s, int k) {
  LevelState& st = s.lv[L];
  if (L > 0 && k > g.seek_min && g.slice_first) {
    const int a = g.slice_first[st.x], b = g.slice_first[st.x + 1];
    const int target = st.emitted + k;
    if (b - a > 1) {
      int lo = a, hi = b - 1;  // last slice with first <= target
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (g.slices[mid].first <= target) lo = mid;
        else hi = mid - 1;
      }
      const SliceState& cp = g.slices[lo];
      if (cp.first > st.emitted) {
        s.lv[L] = cp.cs.lv[0];
        if constexpr (L + 1 < kMaxLevels) s.lv[L + 1] = cp.cs.lv[1];
        if constexpr (L + 2 < kMaxLevels) s.lv[L + 2] = cp.cs.lv[2];
        if constexpr (L + 3 < kMaxLevels) s.lv[L + 3] = cp.cs.lv[3];
        k = target - cp.first;
      }
    }
  }
  for (int i = 0; i < k && i <= g.max_list; ++i)
    if (list_next<L>(g, s) == kInf) break;
}

template <int L>
__device__ __forceinline__ int masked_next(const GraphView& g, ChainState& s) {
  if constexpr (L + 1 < kMaxLevels) {
    LevelState& st = s.lv[L];
    if (st.cur_left == 0) return kInf;
    const int v = list_next<L + 1>(g, s);
    if (v == kInf) return kInf;
    if (st.cur_left > 0) {
      --st.cur_left;
      if (st.cur_left == 0 && st.bleft > 0) {
        const int skip = (int)read_gamma(g, g.g, st.bpos) + 1;
        --st.bleft;
        skip_values<L + 1>(g, s, skip);
        if (st.bleft > 0) {
          st.cur_left = (int)read_gamma(g, g.g, st.bpos) + 1;
          --st.bleft;
        } else {
          st.cur_left = -1;
        }
      }
    }
    return v;
  } else {
    return kInf;
  }
}

template <int L>
__device__ __forceinline__ int list_next(const GraphView& g, ChainState& s) {
  LevelState& st = s.lv[L];
  const int v = min(min(st.hm, st.hi), min(st.hr, st.hc));
  if (v == kInf) return kInf;
  if (st.hm == v) {
    if (--st.mrem == 0) {
      if (st.mleft > 0) {
        st.hm += (int)read_gamma(g, g.g, st.mpos) + 1;
        st.mrem = (int)read_gamma(g, g.g, st.mpos) + 2;
        --st.mleft;
      } else {
        st.hm = kInf;
      }
    }
  }
  if (st.hi == v) {
    if (++st.hi == st.iend) {
      if (st.ileft > 0) {
        st.hi = st.iend + (int)read_gamma(g, g.g, st.ipos) + 1;
        st.iend = st.hi + (int)read_gamma(g, g.g, st.ipos) + g.min_interval;
        --st.ileft;
      } else {
        st.hi = kInf;
      }
    }
  }
  if (st.hr == v) {
    if (--st.rleft > 0) st.hr += (int)read_zeta<3>(g, g.g, st.rpos) + 1;
    else st.hr = kInf;
  }
  if constexpr (L + 1 < kMaxLevels) {
    if (st.hc == v) st.hc = masked_next<L>(g, s);
  }
  ++st.emitted;
  return v;
}

// Parses the record of vertex x into level L; returns its outdegree.
template <int L>
__device__ __forceinline__ int level_init(const GraphView& g, ChainState& s, int x) {
  LevelState& st = s.lv[L];
  st.hm = st.hi = st.hr = st.hc = kInf;
  st.rleft = 0;
  st.x = x;
  st.emitted = 0;
  if (x < 0 || x >= g.n) { set_err(g, kErrId); return 0; }
  uint64_t pos = ef_get(g, g.gef, (uint64_t)x);
  const int d = (int)read_gamma(g, g.g, pos);
  if (d == 0) return 0;
  if (d < 0 || d > g.max_list) { set_err(g, kErrCode); return 0; }
  const int ref = (int)read_unary(g, g.g, pos);
  int extra = d;
  if (ref > 0) {
    if constexpr (L + 1 < kMaxLevels) {
      const int bc = (int)read_gamma(g, g.g, pos);
      // A copy mask alternates copy/skip blocks over the referenced list, so a valid record
      // has at most 2*(its degree + the referenced degree)+1 blocks; anything larger is corrupt.
      if (bc < 0 || bc > 2 * d + 2 * g.max_list + 1) { set_err(g, kErrCode); return 0; }
      st.bpos = pos;
      int total = 0, copied = 0;
      for (int i = 0; i < bc; ++i) {
        const int b = (int)read_gamma(g, g.g, pos) + (i ? 1 : 0);
        total += b;
        if (!(i & 1)) copied += b;
      }
      const int dref = level_init<L + 1>(g, s, x - ref);
      if (!(bc & 1)) copied += dref - total;
      extra = d - copied;
      if (bc == 0) {
        st.cur_left = -1;
        st.bleft = 0;
      } else {
        st.cur_left = (int)read_gamma(g, g.g, st.bpos);
        st.bleft = bc - 1;
        if (st.cur_left == 0 && st.bleft > 0) {
          const int skip = (int)read_gamma(g, g.g, st.bpos) + 1;
          --st.bleft;
          skip_values<L + 1>(g, s, skip);
          if (st.bleft > 0) {
            st.cur_left = (int)read_gamma(g, g.g, st.bpos) + 1;
            --st.bleft;
          } else {
            st.cur_left = -1;
          }
        }
      }
      st.hc = masked_next<L>(g, s);
    } else {
      set_err(g, kErrChain);
      return 0;
    }
  }
  if (extra > 0) {
    const int mc = (int)read_gamma(g, g.g, pos);
    if (mc < 0 || mc > d) { set_err(g, kErrCode); return 0; }
    if (mc) {
      st.mpos = pos;
      for (int i = 0; i < mc; ++i) {
        read_gamma(g, g.g, pos);
        extra -= (int)read_gamma(g, g.g, pos) + 2;
      }
      st.hm = x + (int)d_nat2int(read_gamma(g, g.g, st.mpos));
      st.mrem = (int)read_gamma(g, g.g, st.mpos) + 2;
      st.mleft = mc - 1;
    }
  }
  if (extra > 0) {
    const int ic = (int)read_gamma(g, g.g, pos);
    if (ic < 0 || ic > d) { set_err(g, kErrCode); return 0; }
    if (ic) {
      st.ipos = pos;
      for (int i = 0; i < ic; ++i) {
        read_gamma(g, g.g, pos);
        extra -= (int)read_gamma(g, g.g, pos) + g.min_interval;
      }
      st.hi = x + (int)d_nat2int(read_gamma(g, g.g, st.ipos));
      st.iend = st.hi + (int)read_gamma(g, g.g, st.ipos) + g.min_interval;
      st.ileft = ic - 1;
    }
  }
  if (extra > 0) {
    st.rleft = extra;
    st.rpos = pos;
    st.hr = x + (int)d_nat2int(read_zeta<3>(g, g.g, st.rpos));
  }
  return d;
}

// Temporal edge iterator of one vertex: successor ids in list order with their timestamps.
struct EdgeCursor {
  ChainState cs;
  SeqReader ts;
  int64_t prev;
  int remaining;
  int x;

  // Returns the outdegree.
  __device__ __forceinline__ int open(const GraphView& g, int v) {
    x = v;
    remaining = 0;
    if (v >= g.n) return 0;  // ids past the files' vertex count have empty lists
    remaining = level_init<0>(g, cs, v);
    if (remaining > 0) {
      ts.init(g.t, ef_get(g, g.tef, (uint64_t)v));
      prev = g.min_ts;
    }
    return remaining;
  }
  // Next (successor, timestamp); returns false when the list is exhausted.
  __device__ __forceinline__ bool next(const GraphView& g, int& y, int64_t& t) {
    if (remaining <= 0) return false;
    --remaining;
    y = list_next<0>(g, cs);
    int len = 0;
    bool bad = false;
    const uint64_t z = win_zeta<2>(ts.window(), &len, &bad);
    if (bad) set_err(g, kErrCode);
    ts.skip(len);
    prev += d_nat2int(z);
    t = prev;
    if (y == kInf || y < 0 || y >= g.n) {
      set_err(g, y == kInf ? kErrCount : kErrId);
      remaining = 0;
      return false;
    }
    return true;
  }
};

}  // namespace tga
