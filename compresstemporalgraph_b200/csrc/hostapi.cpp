// Host-only C entry points of the format layer (no GPU needed).
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tga.h"
#include "format.hpp"
#include "gen.hpp"

#include <zlib.h>

namespace tga {
int fail(int code, const std::string& msg);
}

using namespace tga;

static void fill_summary(tga_gen_summary* out, int64_t n, int64_t m, int64_t maxdeg, uint64_t gb, uint64_t tb,
                         uint64_t ib, const EncoderStats& s) {
  if (!out) return;
  std::memset(out, 0, sizeof *out);
  out->n = n;
  out->m = m;
  out->max_degree = maxdeg;
  out->graph_bytes = gb;
  out->timestamp_bytes = tb;
  out->index_bytes = ib;
  out->copied_arcs = s.copied_arcs;
  out->intervalised_arcs = s.intervalised_arcs;
  out->residual_arcs = s.residual_arcs;
  out->multiples_arcs = s.multiples_arcs;
  out->max_chain = s.max_chain;
}

static int write_reversed_impl(const int64_t* offsets, const int32_t* dst, const int64_t* ts, int64_t n, int64_t pivot,
                               const char* dir, const char* base, tga_gen_summary* out) {
  if (!offsets || !dir || !base || n < 1 || n > INT32_MAX || pivot < 0) return fail(TGA_E_ARG, "bad argument");
  if (offsets[0] != 0) return fail(TGA_E_ARG, "offsets must start at 0");
  for (int64_t v = 0; v < n; ++v)
    if (offsets[v + 1] < offsets[v]) return fail(TGA_E_ARG, "offsets must not decrease");
  const int64_t m = offsets[n];
  if (m > 0 && (!dst || !ts)) return fail(TGA_E_ARG, "null edge arrays");
  // Counting sort by the new source (the old successor); old sources ascend, so every new list comes
  // out ordered by successor, and a stable sort by reversed time orders each run of repeats.
  RawGraph r;
  r.n = n;
  r.src_begin.assign((size_t)n + 1, 0);
  for (int64_t e = 0; e < m; ++e) {
    if (dst[e] < 0 || dst[e] >= n) return fail(TGA_E_ARG, "successor out of range");
    if (ts[e] < 0 || ts[e] > pivot) return fail(TGA_E_ARG, "timestamp outside [0, pivot]");
    ++r.src_begin[(size_t)dst[e] + 1];
  }
  for (int64_t v = 0; v < n; ++v) r.src_begin[(size_t)v + 1] += r.src_begin[(size_t)v];
  r.dst.resize((size_t)m);
  r.ts.resize((size_t)m);
  std::vector<int64_t> fill(r.src_begin.begin(), r.src_begin.end() - 1);
  r.min_ts = m ? INT64_MAX : 0;
  for (int64_t x = 0; x < n; ++x)
    for (int64_t e = offsets[x]; e < offsets[x + 1]; ++e) {
      const int64_t at = fill[(size_t)dst[e]]++;
      r.dst[(size_t)at] = (int32_t)x;
      r.ts[(size_t)at] = pivot - ts[e];
      r.min_ts = std::min(r.min_ts, pivot - ts[e]);
    }
  for (int64_t y = 0; y < n; ++y) {
    int64_t a = r.src_begin[(size_t)y];
    const int64_t end = r.src_begin[(size_t)y + 1];
    while (a < end) {
      int64_t b = a + 1;
      while (b < end && r.dst[(size_t)b] == r.dst[(size_t)a]) ++b;
      std::sort(r.ts.begin() + a, r.ts.begin() + b);
      a = b;
    }
  }
  try {
    const WrittenDataset w = encode_and_write(r, dir, base, n - 1, EncoderParams{});
    int64_t maxdeg = 0;
    for (int64_t v = 0; v < n; ++v) maxdeg = std::max<int64_t>(maxdeg, r.src_begin[(size_t)v + 1] - r.src_begin[(size_t)v]);
    fill_summary(out, w.n, w.m, maxdeg, w.graph_bytes, w.ts_bytes, w.index_bytes, w.stats);
  } catch (const std::exception& e) {
    return fail(TGA_E_FORMAT, e.what());
  }
  return TGA_OK;
}

static int reference_depths_impl(const char* dir, const char* base, tga_ref_depths* out, int32_t* depth_out) {
  if (!dir || !base || !out) return fail(TGA_E_ARG, "null argument");
  const std::string bp = std::string(dir) + "/" + base;
  std::vector<uint8_t> graph, offsets;
  if (!read_file(bp + ".graph", graph)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".graph");
  if (!read_file(bp + ".offsets", offsets)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".offsets");
  const auto pr = read_properties(bp + ".properties");
  auto prop = [&](const char* k, int64_t dflt) {
    const auto it = pr.find(k);
    return it == pr.end() ? dflt : (int64_t)std::atoll(it->second.c_str());
  };
  const int64_t n = prop("nodes", -1);
  if (n <= 0) return fail(TGA_E_FORMAT, "the nodes property of " + bp + ".properties is needed");
  std::memset(out, 0, sizeof *out);
  try {
    const std::vector<int32_t> depth = reference_depths(graph, offsets, n, (int)prop("windowsize", 7));
    out->nodes = n;
    out->configured_max_ref_count = (int32_t)prop("maxrefcount", 3);
    for (int64_t v = 0; v < n; ++v) {
      const int32_t d = depth[(size_t)v];
      out->referenced_nodes += d > 0;
      out->maximum_depth = std::max(out->maximum_depth, d);
      if (d < 16) ++out->depth_counts[d];
      else ++out->truncated_nodes;
    }
    if (depth_out) std::copy(depth.begin(), depth.end(), depth_out);
  } catch (const std::exception& e) {
    return fail(TGA_E_FORMAT, e.what());
  }
  return TGA_OK;
}

extern "C" {

int tga_generate(const tga_gen_params* p, const char* dir, const char* base, const char* raw_path, tga_gen_summary* out) {
  if (!p || !dir || !base) return fail(TGA_E_ARG, "null argument");
  GenParams g;
  g.n = p->n;
  g.m = p->m;
  g.deg_exponent = p->deg_exponent;
  g.max_degree = p->max_degree;
  g.repeat_frac = p->repeat_frac;
  g.local_frac = p->local_frac;
  g.local_radius = p->local_radius;
  g.pref_frac = p->pref_frac;
  g.copy_frac = p->copy_frac;
  g.ts_kind = p->ts_kind;
  g.ts_span = p->ts_span;
  g.min_timestamp = p->min_timestamp;
  g.seed = p->seed;
  g.ref_safe = p->ref_safe != 0;
  g.hub_count = p->hub_count;
  g.hub_degree = p->hub_degree;
  if (g.n > INT32_MAX || g.ts_span <= 0 || g.min_timestamp < 0 || g.ts_span > (INT64_C(1) << 62) ||
      g.min_timestamp > (INT64_C(1) << 62))
    return fail(TGA_E_ARG, "vertex ids must fit in [0, 2^31) and timestamps in [0, 2^63)");
  try {
    const GenSummary s = generate_dataset(g, dir, base, raw_path ? raw_path : "");
    fill_summary(out, s.n, s.m, s.max_degree, s.graph_bytes, s.ts_bytes, s.index_bytes, s.stats);
  } catch (const std::exception& e) {
    return fail(TGA_E_IO, e.what());
  }
  return TGA_OK;
}

// Whole file, gunzipped when its name ends in ".gz" (the reference keeps its raw inputs as
// data/raw/<DS>.raw.txt.gz).  False when it cannot be opened or is not valid gzip.
static bool read_raw_input(const std::string& path, std::vector<uint8_t>& out) {
  if (path.size() < 3 || path.compare(path.size() - 3, 3, ".gz") != 0) return read_file(path, out);
  gzFile f = gzopen(path.c_str(), "rb");
  if (!f) return false;
  out.clear();
  std::vector<uint8_t> buf(1 << 20);
  int got;
  while ((got = gzread(f, buf.data(), (unsigned)buf.size())) > 0) out.insert(out.end(), buf.begin(), buf.begin() + got);
  int err = Z_OK;
  gzerror(f, &err);
  gzclose(f);
  return got == 0 && (err == Z_OK || err == Z_STREAM_END);
}

int tga_encode_raw(const char* raw_path, const char* dir, const char* base, int64_t max_label, tga_gen_summary* out) {
  if (!raw_path || !dir || !base) return fail(TGA_E_ARG, "null argument");
  std::vector<uint8_t> raw;
  if (!read_raw_input(raw_path, raw)) return fail(TGA_E_IO, std::string("Cannot open required file: ") + raw_path);
  try {
    const RawGraph g = parse_raw_text(std::string(raw.begin(), raw.end()));
    const WrittenDataset w = encode_and_write(g, dir, base, max_label, EncoderParams{});
    int64_t maxdeg = 0;
    for (int64_t v = 0; v < g.n; ++v) maxdeg = std::max<int64_t>(maxdeg, g.src_begin[v + 1] - g.src_begin[v]);
    fill_summary(out, w.n, w.m, maxdeg, w.graph_bytes, w.ts_bytes, w.index_bytes, w.stats);
  } catch (const std::exception& e) {
    return fail(TGA_E_FORMAT, e.what());
  }
  return TGA_OK;
}

static int write_index(const std::string& d, const EFIndex& ge, const EFIndex& te) {
  if (!write_file(d + "/graph_lower_bits.bin", ge.lower.data(), ge.lower.size()) ||
      !write_file(d + "/graph_upper_bits.bin", ge.upper.data(), ge.upper.size()) ||
      !write_file(d + "/timestamp_lower_bits.bin", te.lower.data(), te.lower.size()) ||
      !write_file(d + "/timestamp_upper_bits.bin", te.upper.data(), te.upper.size()))
    return fail(TGA_E_IO, "cannot write the index files into " + d);
  return TGA_OK;
}

int tga_build_index_device(const char* dir, const char* base, int64_t max_label) {
  if (!dir || !base || max_label < 0) return fail(TGA_E_ARG, "bad argument");
  const std::string d(dir), bp = d + "/" + base;
  std::vector<uint8_t> graph, offsets, ts;
  if (!read_file(bp + ".graph", graph)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".graph");
  if (!read_file(bp + ".timestamps", ts)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".timestamps");
  if (!read_file(bp + ".offsets", offsets)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".offsets");
  const auto pr = read_properties(bp + ".properties");
  const auto it = pr.find("nodes");
  if (it == pr.end()) return fail(TGA_E_FORMAT, "the nodes property of " + bp + ".properties is needed");
  std::vector<uint64_t> goff, toff;
  if (int rc = offsets_on_device(graph, offsets, ts, std::atoll(it->second.c_str()), goff, toff)) return rc;
  try {
    return write_index(d, ef_build(goff, ef_low_bits(graph.size(), max_label)), ef_build(toff, ef_low_bits(ts.size(), max_label)));
  } catch (const std::exception& e) {
    return fail(TGA_E_FORMAT, std::string("packing the index: ") + e.what());
  }
}

int tga_build_index(const char* dir, const char* base, int64_t max_label) {
  if (!dir || !base || max_label < 0) return fail(TGA_E_ARG, "bad argument");
  const std::string d(dir), bp = d + "/" + base;
  std::vector<uint8_t> graph, offsets, ts;
  if (!read_file(bp + ".graph", graph)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".graph");
  if (!read_file(bp + ".timestamps", ts)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".timestamps");
  if (!read_file(bp + ".offsets", offsets)) return fail(TGA_E_IO, "Cannot open required file: " + bp + ".offsets");
  const auto pr = read_properties(bp + ".properties");
  const auto it = pr.find("nodes");
  if (it == pr.end()) return fail(TGA_E_FORMAT, "the nodes property of " + bp + ".properties is needed");
  try {
    EFIndex ge, te;
    index_from_offsets(graph, offsets, ts, std::atoll(it->second.c_str()), 2, max_label, &ge, &te);
    return write_index(d, ge, te);
  } catch (const std::exception& e) {
    return fail(TGA_E_FORMAT, std::string("rebuilding the index from .offsets: ") + e.what());
  }
  return TGA_OK;
}



int tga_decode_table(int32_t kind, int32_t* out) {
  if (!out || (kind != 0 && kind != 3)) return fail(TGA_E_ARG, "kind must be 0 (gamma) or 3 (zeta_3)");
  const std::vector<int32_t> t = table16(kind);
  std::memcpy(out, t.data(), t.size() * sizeof(int32_t));
  return TGA_OK;
}

int tga_encode_codes(int32_t kind, int32_t k, const uint64_t* values, int64_t n, uint8_t* out, int64_t cap,
                     int64_t* nbits) {
  if ((!values && n) || !nbits || n < 0) return fail(TGA_E_ARG, "null argument");
  if (kind == 1 && k < 1) return fail(TGA_E_ARG, "zeta needs k >= 1");
  BitWriter w;
  for (int64_t i = 0; i < n; ++i) {
    switch (kind) {
      case 0: w.write_gamma(values[i]); break;
      case 1: w.write_zeta(values[i], k); break;
      case 2: w.write_unary(values[i]); break;
      case 3: w.write_long(values[i], 64); break;
      default: return fail(TGA_E_ARG, "unknown code kind");
    }
  }
  *nbits = (int64_t)w.nbits;
  if (!out) return TGA_OK;
  if (cap < (int64_t)w.bytes.size()) return fail(TGA_E_ARG, "output buffer too small");
  std::memcpy(out, w.bytes.data(), w.bytes.size());
  return TGA_OK;
}

int tga_ef_encode(const uint64_t* values, int64_t n, int32_t l, uint8_t* lower, int64_t lower_cap, uint8_t* upper,
                  int64_t upper_cap, int64_t* lower_bytes, int64_t* upper_bytes) {
  if ((!values && n) || !lower_bytes || !upper_bytes || n < 0 || l < 0 || l > 62) return fail(TGA_E_ARG, "bad argument");
  EFIndex ef;
  try {
    ef = ef_build(std::vector<uint64_t>(values, values + n), l);
  } catch (const std::exception& e) {
    return fail(TGA_E_ARG, e.what());
  }
  *lower_bytes = (int64_t)ef.lower.size();
  *upper_bytes = (int64_t)ef.upper.size();
  if (!lower || !upper) return TGA_OK;
  if (lower_cap < *lower_bytes || upper_cap < *upper_bytes) return fail(TGA_E_ARG, "output buffer too small");
  std::memcpy(lower, ef.lower.data(), ef.lower.size());
  std::memcpy(upper, ef.upper.data(), ef.upper.size());
  return TGA_OK;
}

int tga_write_reversed(const int64_t* offsets, const int32_t* dst, const int64_t* ts, int64_t n, int64_t pivot,
                       const char* dir, const char* base, tga_gen_summary* out) {
  try {
    return write_reversed_impl(offsets, dst, ts, n, pivot, dir, base, out);
  } catch (const std::bad_alloc&) {
    return fail(TGA_E_OOM, "host allocation failed");
  }
}

int tga_reference_depths(const char* dir, const char* base, tga_ref_depths* out, int32_t* depth_out) {
  try {
    return reference_depths_impl(dir, base, out, depth_out);
  } catch (const std::bad_alloc&) {
    return fail(TGA_E_OOM, "host allocation failed");
  }
}

}  // extern "C"
