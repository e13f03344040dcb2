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
// Layout of the state: the list being decoded (level 0) lives in registers and its merge step is
// inlined into every kernel.  A reference chain (levels 1..3, maxrefcount 3) is only needed for
// the copied successors, so its state sits in a DeepState in local memory and is advanced by a
// few out-of-line routines; this keeps the hot loop small (the whole chain inlined at every call
// site overflowed the instruction cache).  Exhausted sub-iterators hold kInf, which is never a
// vertex id (the reference decoder uses MAX_LABEL and breaks on a successor equal to it,
// gpu_cuda/shared/bfs.cu:763-776).
#pragma once
#include "dview.cuh"

namespace tga {

// One successor list being merged.
struct ListState {
  uint64_t mpos, ipos, rpos;
  int hm, hi, hr, hc;        // heads of multiples, intervals, residuals, copied values
  int mleft, mrem;           // multiples runs still to read, copies left of the current run
  int ileft, iend;           // intervals still to read, end (exclusive) of the current one
  int rleft;                 // residuals left including the head
  int x;                     // vertex whose list this is
  int emitted;               // below level 0: values returned so far; at level 0: copied values
                             // consumed (the index of hc in the list's resolved copies)
};

// Copy mask of one level over the next level's list.
struct MaskState {
  uint64_t bpos;             // next block length in the stream
  int bleft;                 // blocks still to read
  int cur_left;              // values left in the current copy block (-1: copy all that remains)
  int skip;                  // values of the next level to skip before the next copied one
  int pad;
};

// Levels 1..kMaxLevels-1 of a reference chain (lv[j] is level j+1) and the masks of levels
// 0..kMaxLevels-2 (mask[j] selects from lv[j]).
struct DeepState {
  MaskState mask[kMaxLevels - 1];
  ListState lv[kMaxLevels - 1];
};

// Decoder state at the first edge of a slice (see slices.cuh).  The reference-chain levels of a
// list that copies from a chain are kept apart (GraphView::slice_deep[deep]), so a checkpoint of a
// plain list is one cache line.
struct SliceState {
  ListState top;
  uint64_t tpos;    // bit position of the slice's first timestamp code
  int64_t prev;     // timestamp preceding the slice's first edge
  int32_t v;        // vertex
  int32_t count;    // edges in the slice
  int32_t first;    // index of the slice's first edge in the list of v
  int32_t chain;    // the list copies from a reference chain
  int32_t deep;     // its chain levels: index into slice_deep (-1 when chain == 0)
  int32_t run;      // the slice starts inside a run of equal successors: that run's index, else -1
};

// A run of equal successors that slices cut (slices.cuh): list `v`, edges from list index
// `start`, overlapping the slices first_slice .. first_slice + nslices - 1.
struct RunInfo {
  int32_t v, start, first_slice, nslices;
};

// A sliced list and the base of its segment in a per-edge buffer over all sliced lists.
struct LongList {
  int32_t v, pad;
  int64_t base;
};

// ---- merge step shared by all levels ---------------------------------------------------------

// Advances the sub-iterators whose head equals v (equal heads are emitted once, as
// MergedIntIterator does).  Returns true if the copied-values head must advance too.
__device__ __forceinline__ bool merge_advance(const GraphView& g, ListState& st, int v) {
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
  return st.hc == v;
}

// Header of the record of x: outdegree, reference, copy blocks (scanned).  Returns the outdegree
// (0 for an empty list, -1 for a corrupt record); *ref, *bc, *copied, *total describe the copy
// part, mask.bpos points at the first block, pos just past the blocks.
__device__ __forceinline__ int parse_record(const GraphView& g, ListState& st, MaskState& mask, int x, int& ref,
                                            int& bc, int& copied, int& total, uint64_t& pos) {
  st.hm = st.hi = st.hr = st.hc = kInf;
  st.rleft = 0;
  st.x = x;
  st.emitted = 0;
  ref = 0;
  bc = 0;
  copied = total = 0;
  if (x < 0 || x >= g.n) { set_err(g, kErrId); return -1; }
  pos = ef_get(g, g.gef, (uint64_t)x);
  const int d = (int)read_gamma(g, g.g, pos);
  if (d == 0) return 0;
  if (d < 0 || d > g.max_list) { set_err(g, kErrCode); return -1; }
  ref = (int)read_unary(g, g.g, pos);
  if (ref > 0) {
    bc = (int)read_gamma(g, g.g, pos);
    // A copy mask alternates copy/skip blocks over the referenced list, so a valid record has at
    // most 2*(its degree + the largest degree)+1 blocks; anything larger is corrupt.
    if (bc < 0 || bc > 2 * d + 2 * g.max_list + 1) { set_err(g, kErrCode); return -1; }
    mask.bpos = pos;
#pragma unroll 1
    for (int i = 0; i < bc; ++i) {
      const int b = (int)read_gamma(g, g.g, pos) + (i ? 1 : 0);
      total += b;
      if (!(i & 1)) copied += b;
    }
  }
  return d;
}

// Multiples, intervals and residuals of a record; `extra` = outdegree minus copied values.
__device__ __forceinline__ bool parse_extra(const GraphView& g, ListState& st, int x, int d, int extra, uint64_t pos) {
  if (extra > 0) {
    const int mc = (int)read_gamma(g, g.g, pos);
    if (mc < 0 || mc > d) { set_err(g, kErrCode); return false; }
    if (mc) {
      st.mpos = pos;
#pragma unroll 1
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
    if (ic < 0 || ic > d) { set_err(g, kErrCode); return false; }
    if (ic) {
      st.ipos = pos;
#pragma unroll 1
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
  return true;
}

// ---- reference-chain levels (local memory, out of line) ---------------------------------------

template <int L>
__device__ __forceinline__ int deep_next(const GraphView& g, DeepState& d);

// Loads checkpoint cp (list cp.v at its edge cp.first) into level L and its chain into the levels
// below (a list at level L has at most kMaxLevels-1-L further levels).
template <int L>
__device__ __forceinline__ void load_checkpoint(const GraphView& g, DeepState& d, const SliceState& cp) {
  d.lv[L - 1] = cp.top;
  d.lv[L - 1].x = cp.v;
  d.lv[L - 1].emitted = cp.first;
  if (cp.chain) {
    const DeepState& cd = g.slice_deep[cp.deep];
    if constexpr (L < kMaxLevels - 1) {
      d.mask[L] = cd.mask[0];
      d.lv[L] = cd.lv[0];
    }
    if constexpr (L + 1 < kMaxLevels - 1) {
      d.mask[L + 1] = cd.mask[1];
      d.lv[L + 1] = cd.lv[1];
    }
  }
}

// First slice of x (its checkpoint at edge 0 is the state right after parsing the record), or
// null if x is not sliced (or checkpoints are not available yet).
__device__ __forceinline__ const SliceState* first_checkpoint(const GraphView& g, int x) {
  if (!g.slice_first || x < 0 || x >= g.n) return nullptr;
  const int s0 = g.slice_first[x];
  return s0 != g.slice_first[x + 1] ? &g.slices[s0] : nullptr;
}

// Seeks over a pending skip of k values of level L (>= 1) when it is long: the last checkpoint
// of level L's list at or before the target becomes level L, its chain the levels below (a list
// referenced at level L has at most kMaxLevels-1-L further levels), and k shrinks to the values
// still to skip from there, so a skip costs at most one slice of decoding.
template <int L>
__device__ __forceinline__ void deep_seek(const GraphView& g, DeepState& d, int& k) {
  if (k <= g.seek_min || !g.slice_first) return;
  const ListState& st = d.lv[L - 1];
  const int a = g.slice_first[st.x], b = g.slice_first[st.x + 1];
  if (b - a <= 1) return;
  const int target = st.emitted + k;
  int lo = a, hi = b - 1;  // last slice with first <= target
#pragma unroll 1
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g.slices[mid].first <= target) lo = mid;
    else hi = mid - 1;
  }
  const SliceState& cp = g.slices[lo];
  if (cp.first > st.emitted) {
    load_checkpoint<L>(g, d, cp);
    k = target - cp.first;
  }
}

// Next value selected by the copy mask of level M (0..kMaxLevels-2) over level M+1.  The skip
// block after a copy block is left pending in the mask and consumed by the next call, so level
// M+1 is advanced from a single place (one inlined copy of each level's step).
template <int M>
__device__ __forceinline__ int deep_masked(const GraphView& g, DeepState& d) {
  MaskState& mk = d.mask[M];
  if (mk.cur_left == 0) return kInf;
  if (mk.skip > 0) deep_seek<M + 1>(g, d, mk.skip);
#pragma unroll 1
  for (;;) {
    const int v = deep_next<M + 1>(g, d);
    if (v == kInf) return kInf;
    if (mk.skip > 0) {
      --mk.skip;
      continue;
    }
    if (mk.cur_left > 0 && --mk.cur_left == 0 && mk.bleft > 0) {
      mk.skip = (int)read_gamma(g, g.g, mk.bpos) + 1;
      --mk.bleft;
      if (mk.bleft > 0) {
        mk.cur_left = (int)read_gamma(g, g.g, mk.bpos) + 1;
        --mk.bleft;
      } else {
        mk.cur_left = -1;
      }
    }
    return v;
  }
}

template <int L>
__device__ __forceinline__ int deep_next(const GraphView& g, DeepState& d) {
  ListState& st = d.lv[L - 1];
  const int v = min(min(st.hm, st.hi), min(st.hr, st.hc));
  if (v == kInf) return kInf;
  if (merge_advance(g, st, v)) {
    if constexpr (L < kMaxLevels - 1) st.hc = deep_masked<L>(g, d);
    else st.hc = kInf;
  }
  ++st.emitted;
  return v;
}

// Starts the copy mask of level M (bc blocks at mask[M].bpos): first block read; after a leading
// empty copy block the following skip block is left pending.
template <int M>
__device__ __forceinline__ void mask_start(const GraphView& g, DeepState& d, int bc) {
  MaskState& mk = d.mask[M];
  mk.skip = 0;
  if (bc == 0) {
    mk.cur_left = -1;
    mk.bleft = 0;
    return;
  }
  mk.cur_left = (int)read_gamma(g, g.g, mk.bpos);
  mk.bleft = bc - 1;
  if (mk.cur_left == 0 && mk.bleft > 0) {
    mk.skip = (int)read_gamma(g, g.g, mk.bpos) + 1;
    --mk.bleft;
    if (mk.bleft > 0) {
      mk.cur_left = (int)read_gamma(g, g.g, mk.bpos) + 1;
      --mk.bleft;
    } else {
      mk.cur_left = -1;
    }
  }
}

// Opens level L (>= 1) on vertex x; returns its outdegree.  A sliced (long) list is opened from
// its first checkpoint: parsing its record would walk its whole multiples and intervals sections.
template <int L>
__device__ __forceinline__ int deep_open(const GraphView& g, DeepState& d, int x) {
  if (const SliceState* cp = first_checkpoint(g, x)) {
    load_checkpoint<L>(g, d, *cp);
    return g.deg[x];
  }
  ListState& st = d.lv[L - 1];
  int ref, bc, copied, total;
  uint64_t pos;
  MaskState own;
  const int dd = parse_record(g, st, own, x, ref, bc, copied, total, pos);
  if (dd <= 0) return 0;
  int extra = dd;
  if (ref > 0) {
    if constexpr (L < kMaxLevels - 1) {
      const int dref = deep_open<L + 1>(g, d, x - ref);
      if (!(bc & 1)) copied += dref - total;
      extra = dd - copied;
      d.mask[L] = own;
      mask_start<L>(g, d, bc);
      st.hc = deep_masked<L>(g, d);
    } else {
      set_err(g, kErrChain);
      return 0;
    }
  }
  if (!parse_extra(g, st, x, dd, extra, pos)) return 0;
  return dd;
}

// Out-of-line entry points used by level 0.
struct OpenRef {
  int dref;   // outdegree of the referenced list
  int head;   // first copied value (kInf if none)
};

static __device__ __noinline__ int deep_copy_next(const GraphView& g, DeepState& d) { return deep_masked<0>(g, d); }

static __device__ __noinline__ OpenRef deep_open_ref(const GraphView& g, DeepState& d, int xref, int bc, uint64_t bpos) {
  OpenRef r;
  r.dref = deep_open<1>(g, d, xref);
  d.mask[0].bpos = bpos;
  mask_start<0>(g, d, bc);
  r.head = deep_copy_next(g, d);
  return r;
}

// ---- level 0 --------------------------------------------------------------------------------

__device__ __forceinline__ int top_next(const GraphView& g, ListState& st, DeepState* deep) {
  const int v = min(min(st.hm, st.hi), min(st.hr, st.hc));
  if (v == kInf) return kInf;
  if (merge_advance(g, st, v)) {
    st.hc = deep_copy_next(*g.self, *deep);
    ++st.emitted;
  }
  return v;
}

// Parses the record of x into level 0 (and its reference chain); returns the outdegree.
// *chain is set when the list copies from a reference chain.
__device__ __forceinline__ int top_open(const GraphView& g, ListState& st, DeepState* deep, int x, int& chain) {
  int ref, bc, copied, total;
  uint64_t pos;
  MaskState mk;
  const int d = parse_record(g, st, mk, x, ref, bc, copied, total, pos);
  chain = 0;
  if (d <= 0) return 0;
  int extra = d;
  if (ref > 0) {
    chain = 1;
    const OpenRef r = deep_open_ref(*g.self, *deep, x - ref, bc, mk.bpos);
    if (!(bc & 1)) copied += r.dref - total;
    extra = d - copied;
    st.hc = r.head;
  }
  if (!parse_extra(g, st, x, d, extra, pos)) return 0;
  return d;
}

// Temporal edge iterator of one vertex: successor ids in list order with their timestamps.
// The reference-chain state lives in a separate local object (see the file comment), so that the
// cursor's own fields stay in registers.
struct EdgeCursor {
  ListState top;
  DeepState* deep;
  SeqReader ts;
  int64_t prev;
  int remaining;
  int x;
  int chain;

  __device__ __forceinline__ explicit EdgeCursor(DeepState* d) : deep(d) {}

  // Returns the outdegree.  A sliced list starts from its first checkpoint (see deep_open).
  __device__ __forceinline__ int open(const GraphView& g, int v) {
    x = v;
    remaining = 0;
    chain = 0;
    if (v >= g.n) return 0;  // ids past the files' vertex count have empty lists
    if (const SliceState* cp = first_checkpoint(g, v)) {
      top = cp->top;
      chain = cp->chain;
      if (chain) *deep = g.slice_deep[cp->deep];
      ts.init(g.t, cp->tpos);
      prev = cp->prev;
      remaining = g.deg[v];
      return remaining;
    }
    remaining = top_open(g, top, deep, v, chain);
    if (remaining > 0) {
      ts.init(g.t, ef_get(g, g.tef, (uint64_t)v));
      prev = g.min_ts;
    }
    return remaining;
  }
  // Next (successor, timestamp); returns false when the list is exhausted.  kTimes = false skips
  // the timestamp stream (t is then 0 and the cursor's timestamp state is left behind): for
  // workloads whose result does not depend on time.
  template <bool kTimes = true>
  __device__ __forceinline__ bool next(const GraphView& g, int& y, int64_t& t) {
    if (remaining <= 0) return false;
    --remaining;
    y = top_next(g, top, deep);
    if (kTimes) {
      int len = 0;
      bool bad = false;
      const uint64_t z = win_zeta<2>(ts.window(), &len, &bad);
      if (bad) set_err(g, kErrCode);
      ts.skip(len);
      prev += d_nat2int(z);
      t = prev;
    } else {
      t = 0;
    }
    if (y == kInf || y < 0 || y >= g.n) {
      set_err(g, y == kInf ? kErrCount : kErrId);
      remaining = 0;
      return false;
    }
    return true;
  }
};

}  // namespace tga
