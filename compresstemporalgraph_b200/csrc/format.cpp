// Format writers; see format.hpp for the file layouts and the reference lines they follow.
#include "format.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <stdexcept>
#include <thread>

namespace tga {

bool write_file(const std::string& path, const void* data, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = n == 0 || std::fwrite(data, 1, n, f) == n;
  return std::fclose(f) == 0 && ok;
}

bool read_file(const std::string& path, std::vector<uint8_t>& out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) { std::fclose(f); return false; }
  out.resize((size_t)sz);
  const bool ok = sz == 0 || std::fread(out.data(), 1, (size_t)sz, f) == (size_t)sz;
  std::fclose(f);
  return ok;
}

// ---------------------------------------------------------------------------------------------
// Successor-list encoder

GraphEncoder::GraphEncoder(EncoderParams p) : params(p) {
  const int cyc = p.window_size + 1;
  list_.resize(cyc);
  list_len_.assign(cyc, 0);
  ref_count_.assign(cyc, 0);
}

// Splits a sorted list into runs of equal values (length >= 2 -> multiples) and
// singletons (BVMultiGraph.intervalizeMultiples, BVMultiGraph.java:1400-1433).
static int split_multiples(const int32_t* e, int n, std::vector<int32_t>& left, std::vector<int32_t>& len,
                           std::vector<int32_t>& singles) {
  left.clear(); len.clear(); singles.clear();
  if (n == 0) return 0;
  int run_start = 0;
  for (int i = 1; i <= n; ++i) {
    if (i < n && e[i] == e[i - 1]) continue;
    const int rl = i - run_start;
    if (rl > 1) { left.push_back(e[run_start]); len.push_back(rl); }
    else singles.push_back(e[run_start]);
    run_start = i;
  }
  return (int)left.size();
}

// Maximal runs of consecutive integers of length >= min_interval become intervals, the rest
// residuals (BVMultiGraph.intervalize, BVMultiGraph.java:1375-1398).
static int split_intervals(const std::vector<int32_t>& v, int min_interval, std::vector<int32_t>& left,
                           std::vector<int32_t>& len, std::vector<int32_t>& residuals) {
  left.clear(); len.clear(); residuals.clear();
  const int n = (int)v.size();
  int i = 0;
  while (i < n) {
    int j = i + 1;
    while (j < n && v[j] == v[j - 1] + 1) ++j;
    const int run = j - i;
    if (run >= min_interval) {
      left.push_back(v[i]);
      len.push_back(run);
    } else {
      for (int k = i; k < j; ++k) residuals.push_back(v[k]);
    }
    i = j;
  }
  return (int)left.size();
}

// One record's body (reference, copy blocks, multiples, intervals, residuals) relative to the list
// ref_list at distance ref, written to obs (a BitWriter, or a BitCounter to cost it).  st: the
// statistics to add to when the record is written for real, else nullptr.
template <class Out>
static void diff_comp(Out& obs, const EncoderParams& params, DiffScratch& sc, EncoderStats* st, int cur, int ref,
                      const int32_t* ref_list, int ref_len, const int32_t* cur_list, int cur_len) {
  const int mult_count = split_multiples(cur_list, cur_len, sc.mult_left, sc.mult_len, sc.singles);
  const int32_t* cl = sc.singles.data();
  const int cn = (int)sc.singles.size();
  if (ref == 0) ref_len = 0;
  sc.extras.clear();
  sc.blocks.clear();
  // Alternate copy/skip blocks over the reference list (BVMultiGraph.java:1668-1720).
  int j = 0, k = 0, blen = 0;
  bool copying = true;
  while (j < cn && k < ref_len) {
    if (copying) {
      if (cl[j] > ref_list[k]) { sc.blocks.push_back(blen); copying = false; blen = 0; }
      else if (cl[j] < ref_list[k]) sc.extras.push_back(cl[j++]);
      else { ++j; ++k; ++blen; if (st) ++st->copied_arcs; }
    } else {
      if (cl[j] < ref_list[k]) sc.extras.push_back(cl[j++]);
      else if (cl[j] > ref_list[k]) { ++k; ++blen; }
      else { sc.blocks.push_back(blen); copying = true; blen = 0; }
    }
  }
  if (copying && k < ref_len) sc.blocks.push_back(blen);
  while (j < cn) sc.extras.push_back(cl[j++]);

  int64_t t;
  if (params.window_size > 0) {
    t = obs.write_unary((uint64_t)ref);
    if (st) st->bits_references += t;
  }
  if (ref != 0) {
    const int bc = (int)sc.blocks.size();
    t = obs.write_gamma((uint64_t)bc);
    for (int i = 0; i < bc; ++i) t += obs.write_gamma((uint64_t)(i == 0 ? sc.blocks[0] : sc.blocks[i] - 1));
    if (st) st->bits_blocks += t;
  }
  if ((int)sc.extras.size() + mult_count > 0) {
    t = obs.write_gamma((uint64_t)mult_count);
    int64_t prev = 0;
    for (int i = 0; i < mult_count; ++i) {
      if (i == 0) t += obs.write_gamma(int2nat((int64_t)sc.mult_left[0] - cur));
      else t += obs.write_gamma((uint64_t)(sc.mult_left[i] - prev - 1));
      prev = sc.mult_left[i];
      t += obs.write_gamma((uint64_t)(sc.mult_len[i] - params.min_multiple));
      if (st) st->multiples_arcs += sc.mult_len[i];
    }
    if (st) st->bits_multiples += t;

    const int ic = split_intervals(sc.extras, params.min_interval, sc.left, sc.len, sc.residuals);
    t = obs.write_gamma((uint64_t)ic);
    for (int i = 0; i < ic; ++i) {
      if (i == 0) t += obs.write_gamma(int2nat((int64_t)sc.left[0] - cur));
      else t += obs.write_gamma((uint64_t)(sc.left[i] - prev - 1));
      prev = (int64_t)sc.left[i] + sc.len[i];
      t += obs.write_gamma((uint64_t)(sc.len[i] - params.min_interval));
      if (st) st->intervalised_arcs += sc.len[i];
    }
    if (st) st->bits_intervals += t;

    const int rc = (int)sc.residuals.size();
    if (rc) {
      t = obs.write_zeta(int2nat((int64_t)sc.residuals[0] - cur), params.zeta_k);
      prev = sc.residuals[0];
      for (int i = 1; i < rc; ++i) {
        if (sc.residuals[i] == prev) throw std::runtime_error("repeated residual successor");
        t += obs.write_zeta((uint64_t)(sc.residuals[i] - prev - 1), params.zeta_k);
        prev = sc.residuals[i];
      }
      if (st) { st->bits_residuals += t; st->residual_arcs += rc; }
    }
  }
}

void GraphEncoder::add_node(const int32_t* succ, int outd) {
  const int cyc = params.window_size + 1;
  const int cur = cur_node_++;
  const int ci = cur % cyc;
  // Offset delta of this record, then its outdegree (BVMultiGraph.java:1913-1922).
  offsets.write_gamma(graph.nbits - last_bit_);
  node_bit_offsets.push_back(graph.nbits);
  last_bit_ = graph.nbits;
  stats.bits_outdegrees += graph.write_gamma((uint64_t)outd);
  list_[ci].assign(succ, succ + outd);
  list_len_[ci] = outd;
  ++stats.nodes;
  if (outd > 0) {
    // Best reference over the window; ties keep the smallest distance (BVMultiGraph.java:1932-1949).
    int64_t best = INT32_MAX;
    int best_idx = -1;
    ref_count_[ci] = -1;
    for (int j = 0; j < cyc; ++j) {
      const int cand = (cur - j + cyc) % cyc;
      if (ref_count_[cand] < params.max_ref_count && list_len_[cand] != 0) {
        BitCounter bc;
        diff_comp(bc, params, scratch_, nullptr, cur, j, list_[cand].data(), list_len_[cand], list_[ci].data(), outd);
        if (params.no_empty_first_copy && j != 0 && !scratch_.blocks.empty() && scratch_.blocks[0] == 0) continue;
        if ((int64_t)bc.nbits < best) { best = (int64_t)bc.nbits; best_idx = cand; }
      }
    }
    ref_count_[ci] = ref_count_[best_idx] + 1;
    const int ref = (cur - best_idx + cyc) % cyc;
    diff_comp(graph, params, scratch_, &stats, cur, ref, list_[best_idx].data(), list_len_[best_idx], list_[ci].data(),
              outd);
    stats.arcs += outd;
    stats.tot_ref += ref_count_[ci];
    stats.tot_dist += ref;
    stats.max_chain = std::max<int64_t>(stats.max_chain, ref_count_[ci]);
  }
}

// Runs fn(t, lo, hi) for t < parts over [0, count) split into contiguous ranges.
template <class Fn>
static void parallel_ranges(int count, int parts, Fn fn) {
  parts = std::max(1, std::min(parts, count));
  std::vector<std::thread> pool;
  std::vector<std::exception_ptr> errs((size_t)parts);
  for (int t = 0; t < parts; ++t) {
    const int lo = (int)((int64_t)count * t / parts), hi = (int)((int64_t)count * (t + 1) / parts);
    auto run = [&, t, lo, hi] {
      try {
        fn(t, lo, hi);
      } catch (...) {
        errs[(size_t)t] = std::current_exception();
      }
    };
    if (t + 1 < parts) pool.emplace_back(run);
    else run();
  }
  for (auto& th : pool) th.join();
  for (auto& e : errs)
    if (e) std::rethrow_exception(e);
}

static void add_stats(EncoderStats& a, const EncoderStats& b) {
  a.copied_arcs += b.copied_arcs;
  a.intervalised_arcs += b.intervalised_arcs;
  a.residual_arcs += b.residual_arcs;
  a.multiples_arcs += b.multiples_arcs;
  a.bits_outdegrees += b.bits_outdegrees;
  a.bits_references += b.bits_references;
  a.bits_blocks += b.bits_blocks;
  a.bits_residuals += b.bits_residuals;
  a.bits_intervals += b.bits_intervals;
  a.bits_multiples += b.bits_multiples;
}

void GraphEncoder::add_block(const int32_t* const* succ, const int* outd, int count, int threads) {
  if (count <= 0) return;
  const int cyc = params.window_size + 1;
  const int64_t base = cur_node_;
  // List of node v (in this block, or one of the cyc - 1 before it, kept in the ring).
  auto list_of = [&](int64_t v, const int32_t** lp) -> int {
    if (v >= base) {
      *lp = succ[v - base];
      return outd[v - base];
    }
    const int slot = (int)(v % cyc);
    *lp = list_[(size_t)slot].data();
    return list_len_[(size_t)slot];
  };
  // 1. Cost of every candidate of every node (-1: not a candidate by content).
  std::vector<int64_t> cost((size_t)count * cyc, -1);
  parallel_ranges(count, threads, [&](int, int lo, int hi) {
    DiffScratch sc;
    for (int i = lo; i < hi; ++i) {
      if (outd[i] <= 0) continue;
      const int64_t v = base + i;
      for (int j = 0; j < cyc; ++j) {
        if (v - j < 0) continue;
        const int32_t* rl = nullptr;
        const int rlen = j == 0 ? outd[i] : list_of(v - j, &rl);
        if (rlen == 0) continue;
        BitCounter bc;
        diff_comp(bc, params, sc, nullptr, (int)v, j, rl, rlen, succ[i], outd[i]);
        if (params.no_empty_first_copy && j != 0 && !sc.blocks.empty() && sc.blocks[0] == 0) continue;
        cost[(size_t)i * cyc + j] = (int64_t)bc.nbits;
      }
    }
  });
  // 2. Choices in node order: the cheapest candidate whose chain is not full, ties to the nearest.
  std::vector<int> ref((size_t)count, 0), rc((size_t)count, 0);
  auto ref_count_of = [&](int64_t v) { return v >= base ? rc[(size_t)(v - base)] : ref_count_[(size_t)(v % cyc)]; };
  for (int i = 0; i < count; ++i) {
    ++stats.nodes;
    if (outd[i] <= 0) {
      rc[(size_t)i] = ref_count_[(size_t)((base + i) % cyc)];  // unchanged, as add_node leaves it
      continue;
    }
    const int64_t v = base + i;
    int64_t best = INT32_MAX;
    int bj = -1;
    for (int j = 0; j < cyc; ++j) {
      const int64_t c = cost[(size_t)i * cyc + j];
      if (c < 0) continue;
      const int r = j == 0 ? -1 : ref_count_of(v - j);
      if (r < params.max_ref_count && c < best) {
        best = c;
        bj = j;
      }
    }
    rc[(size_t)i] = (bj == 0 ? -1 : ref_count_of(v - bj)) + 1;
    ref[(size_t)i] = bj;
    stats.arcs += outd[i];
    stats.tot_ref += rc[(size_t)i];
    stats.tot_dist += bj;
    stats.max_chain = std::max<int64_t>(stats.max_chain, rc[(size_t)i]);
  }
  // 3. Records written in parallel, each range into its own stream.
  const int parts = std::max(1, std::min(threads, count));
  std::vector<WordWriter> outs((size_t)parts);
  std::vector<std::vector<uint64_t>> starts((size_t)parts);
  std::vector<EncoderStats> st((size_t)parts);
  parallel_ranges(count, parts, [&](int t, int lo, int hi) {
    DiffScratch sc;
    WordWriter& o = outs[(size_t)t];
    for (int i = lo; i < hi; ++i) {
      starts[(size_t)t].push_back(o.nbits);
      st[(size_t)t].bits_outdegrees += o.write_gamma((uint64_t)outd[i]);
      if (outd[i] > 0) {
        const int32_t* rl = nullptr;
        const int rlen = ref[(size_t)i] == 0 ? outd[i] : list_of(base + i - ref[(size_t)i], &rl);
        diff_comp(o, params, sc, &st[(size_t)t], (int)(base + i), ref[(size_t)i], rl, rlen, succ[i], outd[i]);
      }
    }
    o.finish();
  });
  // 4. Join in order; offsets of every record.
  for (int t = 0; t < parts; ++t) {
    const uint64_t at = graph.nbits;
    for (uint64_t s0 : starts[(size_t)t]) {
      offsets.write_gamma(at + s0 - last_bit_);
      node_bit_offsets.push_back(at + s0);
      last_bit_ = at + s0;
    }
    graph.append_words(outs[(size_t)t]);
    add_stats(stats, st[(size_t)t]);
  }
  // 5. The ring holds the last cyc nodes for the next block, as add_node leaves it.
  for (int i = std::max(0, count - cyc); i < count; ++i) {
    const size_t slot = (size_t)((base + i) % cyc);
    list_[slot].assign(succ[i], succ[i] + outd[i]);
    list_len_[slot] = outd[i];
    if (outd[i] > 0) ref_count_[slot] = rc[(size_t)i];
  }
  cur_node_ += count;
}

void GraphEncoder::finish() {
  offsets.write_gamma(graph.nbits - last_bit_);
  node_bit_offsets.push_back(graph.nbits);
}

// ---------------------------------------------------------------------------------------------
// Timestamps

TimestampEncoder::TimestampEncoder(int64_t mn, int k) : min_timestamp(mn), zeta_k(k) {
  out.write_long((uint64_t)mn, 64);
}

void TimestampEncoder::add_node(const int64_t* ts, int count) {
  node_bit_offsets.push_back(out.nbits);
  int64_t prev = min_timestamp;
  for (int i = 0; i < count; ++i) {
    out.write_zeta(int2nat(ts[i] - prev), zeta_k);
    prev = ts[i];
  }
}

void TimestampEncoder::add_block(const int64_t* const* ts, const int* count, int nodes, int threads) {
  if (nodes <= 0) return;
  const int parts = std::max(1, std::min(threads, nodes));
  std::vector<WordWriter> outs((size_t)parts);
  std::vector<std::vector<uint64_t>> starts((size_t)parts);
  parallel_ranges(nodes, parts, [&](int t, int lo, int hi) {
    WordWriter& o = outs[(size_t)t];
    for (int i = lo; i < hi; ++i) {
      starts[(size_t)t].push_back(o.nbits);
      int64_t prev = min_timestamp;
      for (int k = 0; k < count[i]; ++k) {
        o.write_zeta(int2nat(ts[i][k] - prev), zeta_k);
        prev = ts[i][k];
      }
    }
    o.finish();
  });
  for (int t = 0; t < parts; ++t) {
    const uint64_t at = out.nbits;
    for (uint64_t s0 : starts[(size_t)t]) node_bit_offsets.push_back(at + s0);
    out.append_words(outs[(size_t)t]);
  }
}

void TimestampEncoder::finish() { node_bit_offsets.push_back(out.nbits); }

// ---------------------------------------------------------------------------------------------
// Elias-Fano index

int ef_low_bits(uint64_t stream_bytes, int64_t max_label) {
  if (max_label <= 0) return 0;
  const uint64_t q = stream_bytes * 8 / (uint64_t)max_label;
  if (q == 0) return 0;  // the reference formula is undefined here (log2(0)); 0 keeps the index valid
  return (int)std::log2((double)q);
}

EFIndex ef_build(const std::vector<uint64_t>& v, int l) {
  EFIndex ef;
  ef.l = l;
  const uint64_t n = v.size();
  const uint64_t lower_bits = n * (uint64_t)l;
  ef.lower.assign(((lower_bits + 63) / 64) * 8, 0);
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t low = l ? (v[i] & ((l == 64) ? ~0ull : ((1ull << l) - 1))) : 0;
    for (int b = 0; b < l; ++b) {
      const uint64_t pos = i * (uint64_t)l + (uint64_t)b;
      if ((low >> (l - 1 - b)) & 1) ef.lower[pos >> 3] |= (uint8_t)(0x80 >> (pos & 7));
    }
  }
  const uint64_t top = n ? (v.back() >> l) + n : 0;
  ef.upper.assign(((top + 63) / 64 + 1) * 8, 0);
  for (uint64_t i = 0; i < n; ++i) {
    if (i && v[i] < v[i - 1]) throw std::runtime_error("EF values must be non-decreasing");
    const uint64_t pos = (v[i] >> l) + i;
    ef.upper[pos >> 3] |= (uint8_t)(1u << (pos & 7));
  }
  return ef;
}

void index_from_offsets(const std::vector<uint8_t>& graph, const std::vector<uint8_t>& offsets,
                        const std::vector<uint8_t>& timestamps, int64_t n, int ts_zeta_k, int64_t max_label,
                        EFIndex* graph_ef, EFIndex* ts_ef) {
  if (n <= 0) throw std::runtime_error("vertex count needed (the nodes property)");
  std::vector<uint64_t> goff((size_t)n + 1), toff((size_t)n + 1);
  FastBitReader ob(offsets);
  uint64_t at = 0;
  for (int64_t v = 0; v <= n; ++v) {
    at += ob.gamma();
    if (at > (uint64_t)graph.size() * 8) throw std::runtime_error("offsets point past the end of the graph stream");
    goff[(size_t)v] = at;
  }
  FastBitReader gb(graph), tb(timestamps, 64);
  for (int64_t v = 0; v < n; ++v) {
    gb.seek(goff[(size_t)v]);
    const uint64_t deg = goff[(size_t)v + 1] > goff[(size_t)v] ? gb.gamma() : 0;
    toff[(size_t)v] = tb.pos();
    for (uint64_t i = 0; i < deg; ++i) tb.zeta(ts_zeta_k);
  }
  toff[(size_t)n] = tb.pos();
  *graph_ef = ef_build(goff, ef_low_bits(graph.size(), max_label));
  *ts_ef = ef_build(toff, ef_low_bits(timestamps.size(), max_label));
}

std::vector<int32_t> reference_depths(const std::vector<uint8_t>& graph, const std::vector<uint8_t>& offsets,
                                      int64_t n, int window_size) {
  if (n <= 0) throw std::runtime_error("vertex count needed (the nodes property)");
  std::vector<int32_t> depth((size_t)n, 0);
  FastBitReader ob(offsets), gb(graph);
  uint64_t at = 0;
  for (int64_t v = 0; v < n; ++v) {
    at += ob.gamma();
    if (at >= (uint64_t)graph.size() * 8 + 1) throw std::runtime_error("offsets point past the end of the graph stream");
    gb.seek(at);
    const uint64_t deg = gb.gamma();
    if (deg == 0 || window_size <= 0) continue;
    const uint64_t ref = gb.unary();
    if (ref == 0) continue;
    if (ref > (uint64_t)v) throw std::runtime_error("reference before the first list at node " + std::to_string(v));
    depth[(size_t)v] = depth[(size_t)(v - (int64_t)ref)] + 1;
  }
  return depth;
}

uint64_t ef_get_host(const EFIndex& ef, uint64_t i) {
  uint64_t low = 0;
  for (int b = 0; b < ef.l; ++b) {
    const uint64_t pos = i * (uint64_t)ef.l + (uint64_t)b;
    low = (low << 1) | (uint64_t)((ef.lower[pos >> 3] >> (7 - (pos & 7))) & 1);
  }
  uint64_t seen = 0;
  for (uint64_t pos = 0; pos < ef.upper.size() * 8; ++pos) {
    if ((ef.upper[pos >> 3] >> (pos & 7)) & 1) {
      if (seen == i) return ((pos - i) << ef.l) | low;
      ++seen;
    }
  }
  throw std::runtime_error("EF index out of range");
}

// ---------------------------------------------------------------------------------------------
// Raw 4-column text

RawGraph parse_raw_text(const std::string& text) {
  RawGraph g;
  std::vector<int32_t> src;
  int64_t max_node = -1;
  const char* p = text.c_str();
  const char* end = p + text.size();
  long line = 0;
  int32_t last_src = -1;
  g.min_ts = INT64_MAX;
  while (p < end) {
    ++line;
    const char* eol = (const char*)std::memchr(p, '\n', (size_t)(end - p));
    if (!eol) eol = end;
    int64_t tok[4];
    int nt = 0;
    const char* q = p;
    while (q < eol && nt < 4) {
      while (q < eol && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
      if (q >= eol) break;
      char* e2;
      errno = 0;
      const long long v = std::strtoll(q, &e2, 10);
      if (e2 == q || errno) throw std::runtime_error("invalid number at line " + std::to_string(line));
      tok[nt++] = v;
      q = e2;
    }
    if (nt == 0) { p = eol + 1; continue; }
    if (nt < 4) throw std::runtime_error("expected at least four columns at input line " + std::to_string(line));
    for (int i = 0; i < 4; ++i)
      if (tok[i] < 0 || tok[i] > INT32_MAX) throw std::runtime_error("value out of range at line " + std::to_string(line));
    if (tok[0] < last_src) throw std::runtime_error("source nodes must be sorted at input line " + std::to_string(line));
    last_src = (int32_t)tok[0];
    src.push_back((int32_t)tok[0]);
    g.dst.push_back((int32_t)tok[1]);
    g.ts.push_back(tok[3]);
    g.min_ts = std::min(g.min_ts, tok[3]);
    max_node = std::max<int64_t>(max_node, std::max(tok[0], tok[1]));
    p = eol + 1;
  }
  if (src.empty()) throw std::runtime_error("the input graph contains no edges");
  g.n = max_node + 1;
  g.src_begin.assign((size_t)g.n + 1, 0);
  for (int32_t s : src) g.src_begin[(size_t)s + 1]++;
  for (int64_t i = 0; i < g.n; ++i) g.src_begin[(size_t)i + 1] += g.src_begin[(size_t)i];
  // Successor values are sorted per source, timestamps stay in line order.
  for (int64_t v = 0; v < g.n; ++v) std::sort(g.dst.begin() + g.src_begin[v], g.dst.begin() + g.src_begin[v + 1]);
  return g;
}

static std::string fmt_ratio(double x) {
  char b[64];
  std::snprintf(b, sizeof b, "%.3f", x);
  std::string s(b);
  while (!s.empty() && s.back() == '0') s.pop_back();
  if (!s.empty() && s.back() == '.') s.pop_back();
  return s;
}

static void ensure_dir(const std::string& dir) {
  std::string acc;
  for (size_t i = 0; i < dir.size(); ++i) {
    acc.push_back(dir[i]);
    if (dir[i] == '/' && acc.size() > 1) ::mkdir(acc.c_str(), 0755);
  }
  ::mkdir(dir.c_str(), 0755);
}

WrittenDataset write_dataset(const std::string& dir, const std::string& base, const GraphEncoder& ge,
                             const TimestampEncoder& te, int64_t n, int64_t max_label) {
  if (max_label < 0) max_label = n - 1;
  ensure_dir(dir);
  const std::string bp = dir + "/" + base;
  WrittenDataset w;
  w.n = n;
  w.m = ge.stats.arcs;
  w.stats = ge.stats;
  if (!write_file(bp + ".graph", ge.graph.bytes.data(), ge.graph.bytes.size()) ||
      !write_file(bp + ".offsets", ge.offsets.bytes.data(), ge.offsets.bytes.size()) ||
      !write_file(bp + ".timestamps", te.out.bytes.data(), te.out.bytes.size()))
    throw std::runtime_error("cannot write dataset files under " + dir);
  w.graph_bytes = ge.graph.bytes.size();
  w.ts_bytes = te.out.bytes.size();
  w.gl = ef_low_bits(w.graph_bytes, max_label);
  w.tl = ef_low_bits(w.ts_bytes, max_label);
  const EFIndex eg = ef_build(ge.node_bit_offsets, w.gl);
  const EFIndex et = ef_build(te.node_bit_offsets, w.tl);
  if (!write_file(dir + "/graph_lower_bits.bin", eg.lower.data(), eg.lower.size()) ||
      !write_file(dir + "/graph_upper_bits.bin", eg.upper.data(), eg.upper.size()) ||
      !write_file(dir + "/timestamp_lower_bits.bin", et.lower.data(), et.lower.size()) ||
      !write_file(dir + "/timestamp_upper_bits.bin", et.upper.data(), et.upper.size()))
    throw std::runtime_error("cannot write index files under " + dir);
  w.index_bytes = eg.lower.size() + eg.upper.size() + et.lower.size() + et.upper.size();

  const EncoderStats& s = ge.stats;
  const EncoderParams& p = ge.params;
  const double nn = (double)std::max<int64_t>(1, n);
  const double arcs = (double)std::max<int64_t>(1, s.arcs);
  std::string pr;
  pr += "#BVGraph properties\n";
  pr += "nodes=" + std::to_string(n) + "\n";
  pr += "arcs=" + std::to_string(s.arcs) + "\n";
  pr += "windowsize=" + std::to_string(p.window_size) + "\n";
  pr += "maxrefcount=" + std::to_string(p.max_ref_count) + "\n";
  pr += "minintervallength=" + std::to_string(p.min_interval) + "\n";
  pr += "zetak=" + std::to_string(p.zeta_k) + "\n";
  pr += "compressionflags=\n";
  pr += "avgref=" + fmt_ratio((double)s.tot_ref / nn) + "\n";
  pr += "avgdist=" + fmt_ratio((double)s.tot_dist / nn) + "\n";
  pr += "copiedarcs=" + std::to_string(s.copied_arcs) + "\n";
  pr += "intervalisedarcs=" + std::to_string(s.intervalised_arcs) + "\n";
  pr += "residualarcs=" + std::to_string(s.residual_arcs) + "\n";
  pr += "bitsperlink=" + fmt_ratio((double)ge.graph.nbits / arcs) + "\n";
  pr += "bitspernode=" + fmt_ratio((double)ge.graph.nbits / nn) + "\n";
  pr += "bitsforoutdegrees=" + std::to_string(s.bits_outdegrees) + "\n";
  pr += "bitsforreferences=" + std::to_string(s.bits_references) + "\n";
  pr += "bitsforblocks=" + std::to_string(s.bits_blocks) + "\n";
  pr += "bitsforresiduals=" + std::to_string(s.bits_residuals) + "\n";
  pr += "bitsforintervals=" + std::to_string(s.bits_intervals) + "\n";
  pr += "bitsformultiples=" + std::to_string(s.bits_multiples) + "\n";
  pr += "graphclass=gr.uoa.di.networkanalysis.BVMultiGraph\n";
  pr += "version=0\n";
  pr += "mintimestamp=" + std::to_string(te.min_timestamp) + "\n";
  write_file(bp + ".properties", pr.data(), pr.size());
  return w;
}

int encode_threads() {
  int threads = (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()));
  if (const char* e = std::getenv("TGA_ENCODE_THREADS")) threads = std::max(0, std::atoi(e));
  return threads;
}

WrittenDataset encode_and_write(const RawGraph& g, const std::string& dir, const std::string& base,
                                int64_t max_label, const EncoderParams& p) {
  GraphEncoder ge(p);
  TimestampEncoder te(g.min_ts, p.ts_zeta_k);
  const int threads = encode_threads();
  if (threads == 0) {
    for (int64_t v = 0; v < g.n; ++v) {
      const int64_t b = g.src_begin[v], e = g.src_begin[v + 1];
      ge.add_node(g.dst.data() + b, (int)(e - b));
      te.add_node(g.ts.data() + b, (int)(e - b));
    }
  } else {
    constexpr int64_t kBlockNodes = 1 << 16;
    std::vector<const int32_t*> sp;
    std::vector<const int64_t*> tp;
    std::vector<int> len;
    for (int64_t v0 = 0; v0 < g.n; v0 += kBlockNodes) {
      const int nb = (int)std::min<int64_t>(kBlockNodes, g.n - v0);
      sp.resize((size_t)nb);
      tp.resize((size_t)nb);
      len.resize((size_t)nb);
      for (int i = 0; i < nb; ++i) {
        const int64_t b = g.src_begin[v0 + i], e = g.src_begin[v0 + i + 1];
        sp[(size_t)i] = g.dst.data() + b;
        tp[(size_t)i] = g.ts.data() + b;
        len[(size_t)i] = (int)(e - b);
      }
      ge.add_block(sp.data(), len.data(), nb, threads);
      te.add_block(tp.data(), len.data(), nb, threads);
    }
  }
  ge.finish();
  te.finish();
  return write_dataset(dir, base, ge, te, g.n, max_label);
}

// key=value lines of a .properties file (missing file: empty map).
std::map<std::string, std::string> read_properties(const std::string& path) {
  std::map<std::string, std::string> m;
  std::vector<uint8_t> raw;
  if (!read_file(path, raw)) return m;
  std::string s(raw.begin(), raw.end());
  size_t p = 0;
  while (p < s.size()) {
    size_t e = s.find('\n', p);
    if (e == std::string::npos) e = s.size();
    std::string line = s.substr(p, e - p);
    p = e + 1;
    if (line.empty() || line[0] == '#') continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    m[line.substr(0, eq)] = line.substr(eq + 1);
  }
  return m;
}

}  // namespace tga
