// Seeded synthetic temporal multigraphs with the shapes of the benchmark configurations
// (the reference's real datasets are absent).  Edges are produced per source in id order and
// streamed straight into the encoders, so multi-hundred-million-edge graphs never exist as an
// edge list in memory.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <exception>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "format.hpp"
#include "gen.hpp"

namespace tga {

namespace {
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    for (auto& x : s) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t t = z;
      t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
      t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
      x = t ^ (t >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  int64_t range(int64_t lo, int64_t hi) { return lo + (int64_t)(next() % (uint64_t)(hi - lo + 1)); }  // inclusive
};
}  // namespace

GenSummary generate_dataset(const GenParams& p, const std::string& dir, const std::string& base, const std::string& raw_path) {
  if (p.n < 4 || p.m < 1) throw std::runtime_error("generator needs n >= 4 and m >= 1");
  const int64_t n = p.n;
  Rng rng(p.seed);
  // Out-degrees: Pareto weights with tail exponent (zipf-1), capped, scaled to exactly m; with hubs,
  // hub_count vertices spread over the id range take hub_degree edges each and the others share the
  // rest.
  std::vector<int64_t> deg((size_t)n, 0);
  const int64_t nhub = p.hub_degree > 0 ? std::max<int64_t>(0, std::min<int64_t>(p.hub_count, n - 2)) : 0;
  if (nhub * p.hub_degree >= p.m) throw std::runtime_error("hubs hold more edges than m");
  auto hub_vertex = [&](int64_t k) { return (int64_t)(((2 * k + 1) * (n - 1)) / (2 * nhub)); };
  const int64_t m_rest = p.m - nhub * p.hub_degree;
  {
    std::vector<double> w((size_t)n);
    const double a = std::max(0.05, p.deg_exponent - 1.0);
    const double cap = (double)std::max<int64_t>(1, p.max_degree);
    double tot = 0;
    for (int64_t v = 0; v < n; ++v) {
      double u = rng.uniform();
      if (u < 1e-300) u = 1e-300;
      w[(size_t)v] = std::min(cap, std::pow(u, -1.0 / a));
    }
    for (int64_t k = 0; k < nhub; ++k) w[(size_t)hub_vertex(k)] = 0.0;
    for (int64_t v = 0; v < n; ++v) tot += w[(size_t)v];
    long double cum = 0;
    int64_t prev = 0;
    for (int64_t v = 0; v < n; ++v) {
      cum += w[(size_t)v];
      const int64_t c = (int64_t)std::llround((long double)m_rest * cum / tot);
      deg[(size_t)v] = c - prev;
      prev = c;
    }
    // Make the largest id a source so that n = max id + 1 holds even with no in-edges to it (the
    // edge is taken from the largest list that is not a hub, so hubs keep exactly hub_degree).
    if (deg[(size_t)n - 1] == 0) {
      const auto it = std::max_element(deg.begin(), deg.end());
      --*it;
      deg[(size_t)n - 1] = 1;
    }
    for (int64_t k = 0; k < nhub; ++k) deg[(size_t)hub_vertex(k)] = p.hub_degree;
  }
  const int32_t lo_id = p.ref_safe ? 1 : 0;
  const int32_t hi_id = p.ref_safe ? (int32_t)(n - 2) : (int32_t)(n - 1);

  EncoderParams ep;
  // The reference-safe layout also keeps the reference GPU decoder away from copy masks that start
  // with an empty copy block.
  ep.no_empty_first_copy = p.ref_safe;
  GraphEncoder ge(ep);
  TimestampEncoder te(p.min_timestamp, ep.ts_zeta_k);
  FILE* raw = raw_path.empty() ? nullptr : std::fopen(raw_path.c_str(), "w");
  if (!raw_path.empty() && !raw) throw std::runtime_error("cannot write " + raw_path);

  const int threads = encode_threads();  // 0: node by node; the files are the same either way
  constexpr int64_t kBlockNodes = 1 << 16;
  struct Block {
    std::vector<int32_t> succ;    // the block's successor lists, back to back
    std::vector<int64_t> ts;      // and their timestamps
    std::vector<int64_t> off{0};  // list i of the block: [off[i], off[i+1])
    int nodes() const { return (int)off.size() - 1; }
  };
  // While one block is generated (one sequential random stream), the block before it is encoded
  // on its own thread (with the encoders' own worker threads).  Blocks reach the encoders one at a
  // time and in node order, so the files are the same as with no overlap.
  Block fill, busy;
  std::thread encoder;
  std::exception_ptr encoder_error;
  auto encode_block = [&](const Block& b) {
    const int nb = b.nodes();
    std::vector<const int32_t*> sp((size_t)nb);
    std::vector<const int64_t*> tp((size_t)nb);
    std::vector<int> len((size_t)nb);
    for (int i = 0; i < nb; ++i) {
      sp[(size_t)i] = b.succ.data() + b.off[(size_t)i];
      tp[(size_t)i] = b.ts.data() + b.off[(size_t)i];
      len[(size_t)i] = (int)(b.off[(size_t)i + 1] - b.off[(size_t)i]);
    }
    ge.add_block(sp.data(), len.data(), nb, threads);
    te.add_block(tp.data(), len.data(), nb, threads);
  };
  auto wait_encoder = [&]() {
    if (encoder.joinable()) encoder.join();
    if (encoder_error) std::rethrow_exception(std::exchange(encoder_error, nullptr));
  };
  auto flush = [&]() {
    if (fill.nodes() == 0) return;
    wait_encoder();
    std::swap(fill, busy);
    fill.succ.clear();
    fill.ts.clear();
    fill.off.assign(1, 0);
    encoder = std::thread([&] {
      try {
        encode_block(busy);
      } catch (...) {
        encoder_error = std::current_exception();
      }
    });
  };
  // Declared after everything the encoder thread uses, so an exception leaving this function
  // joins the thread before those are destroyed.
  struct Joiner {
    std::thread& t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } joiner{encoder};

  const int W = 7;
  std::vector<std::vector<int32_t>> ring(W + 1);  // distinct successors of the last vertices
  std::vector<std::pair<int32_t, int32_t>> pairs;  // (dst, multiplicity)
  std::vector<int32_t> succ;
  std::vector<int64_t> ts, tsbuf;
  bool forced_min = false;
  GenSummary sum;
  const double burst_lo = 0.5 * (double)p.ts_span, burst_w = 0.01 * (double)p.ts_span;

  auto draw_ts = [&]() -> int64_t {
    double x;
    if (p.ts_kind == 2 && rng.uniform() < 0.10) x = burst_lo + rng.uniform() * burst_w;
    else x = rng.uniform() * (double)p.ts_span;
    int64_t t = p.min_timestamp + (int64_t)x;
    if (t >= p.min_timestamp + p.ts_span) t = p.min_timestamp + p.ts_span - 1;
    return t;
  };
  auto draw_mult = [&]() -> int32_t { return rng.uniform() < p.repeat_frac ? (int32_t)rng.range(2, 5) : 1; };

  for (int64_t v = 0; v < n; ++v) {
    const int64_t D = deg[(size_t)v];
    pairs.clear();
    int64_t edges = 0;
    if (D > 0) {
      // Part of the list copied from a vertex inside the compression window.
      if (p.copy_frac > 0 && v > 0) {
        const int r = (int)rng.range(1, std::min<int64_t>(W, v));
        const auto& src = ring[(size_t)((v - r) % (W + 1))];
        const double want = p.copy_frac * (double)D;
        if (!src.empty() && want >= 1.0) {
          const double prob = std::min(1.0, want / (double)src.size());
          for (int32_t y : src) {
            if (edges >= D) break;
            if (rng.uniform() < prob) {
              const int32_t k = (int32_t)std::min<int64_t>(draw_mult(), D - edges);
              pairs.emplace_back(y, k);
              edges += k;
            }
          }
        }
      }
      int64_t prev_id = v;
      int guard = 0;
      while (edges < D) {
        int64_t y;
        if (rng.uniform() < p.local_frac) {
          y = prev_id + rng.range(-p.local_radius, p.local_radius);
        } else if (p.pref_frac > 0 && rng.uniform() < p.pref_frac) {
          // Preferential targets: a heavy-tailed rank mapped through a fixed multiplicative hash.
          const double u = std::max(1e-12, rng.uniform());
          const int64_t rank = std::min<int64_t>(n - 1, (int64_t)std::pow(u, -1.2) - 1);
          y = (int64_t)((uint64_t)(rank * 0x9E3779B1ull + 12345) % (uint64_t)n);
        } else {
          y = rng.range(0, n - 1);
        }
        if (y < lo_id) y = lo_id;
        if (y > hi_id) y = hi_id;
        prev_id = y;
        const int32_t k = (int32_t)std::min<int64_t>(draw_mult(), D - edges);
        pairs.emplace_back((int32_t)y, k);
        edges += k;
        if (++guard > 64 * D + 1024) break;
      }
      std::sort(pairs.begin(), pairs.end());
      // Merge repeated targets.
      size_t o = 0;
      for (size_t i = 0; i < pairs.size(); ++i) {
        if (o && pairs[o - 1].first == pairs[i].first) pairs[o - 1].second += pairs[i].second;
        else pairs[o++] = pairs[i];
      }
      pairs.resize(o);
    }
    succ.clear();
    ts.clear();
    auto& slot = ring[(size_t)(v % (W + 1))];
    slot.clear();
    for (const auto& pr : pairs) {
      slot.push_back(pr.first);
      tsbuf.clear();
      for (int32_t k = 0; k < pr.second; ++k) tsbuf.push_back(draw_ts());
      if (!forced_min) { tsbuf[0] = p.min_timestamp; forced_min = true; }
      std::sort(tsbuf.begin(), tsbuf.end());
      for (int64_t t : tsbuf) { succ.push_back(pr.first); ts.push_back(t); }
    }
    if (threads == 0) {
      ge.add_node(succ.data(), (int)succ.size());
      te.add_node(ts.data(), (int)ts.size());
    } else {
      fill.succ.insert(fill.succ.end(), succ.begin(), succ.end());
      fill.ts.insert(fill.ts.end(), ts.begin(), ts.end());
      fill.off.push_back((int64_t)fill.succ.size());
      if (fill.nodes() == kBlockNodes) flush();
    }
    if (raw)
      for (size_t i = 0; i < succ.size(); ++i) std::fprintf(raw, "%lld\t%d\t1\t%lld\n", (long long)v, succ[i], (long long)ts[i]);
    sum.m += (int64_t)succ.size();
    sum.max_degree = std::max<int64_t>(sum.max_degree, (int64_t)succ.size());
  }
  flush();
  wait_encoder();
  ge.finish();
  te.finish();
  if (raw) std::fclose(raw);
  if (!forced_min) throw std::runtime_error("generator produced no edges");

  const WrittenDataset w = write_dataset(dir, base, ge, te, n, n - 1);
  sum.n = n;
  sum.graph_bytes = w.graph_bytes;
  sum.ts_bytes = w.ts_bytes;
  sum.index_bytes = w.index_bytes;
  sum.stats = ge.stats;
  return sum;
}

}  // namespace tga
