// Seeded synthetic temporal multigraph generator (see gen.cpp).
#pragma once
#include <cstdint>
#include <string>

#include "format.hpp"

namespace tga {

struct GenParams {
  int64_t n = 10000;            // vertices (ids 0..n-1; n-1 always has an out-edge)
  int64_t m = 200000;           // temporal edges, exact
  double deg_exponent = 2.1;    // Zipf exponent of the out-degree distribution
  int64_t max_degree = 1 << 20; // cap on the Pareto weight before scaling
  double repeat_frac = 0.30;    // fraction of (src,dst) pairs carrying 2-5 timestamps
  double local_frac = 0.60;     // successor within +-local_radius of the previous one
  int local_radius = 32;
  double pref_frac = 0.0;       // share of the non-local successors drawn preferentially
  double copy_frac = 0.0;       // share of each list copied from a vertex in the window of 7
  int ts_kind = 0;              // 0 uniform, 1 Poisson process (uniform given the count), 2 bursty
  int64_t ts_span = 1000000;
  int64_t min_timestamp = 0;    // forced to occur once
  uint64_t seed = 1;
  bool ref_safe = false;        // no in-edges to vertex 0 and to vertex n-1
  int32_t hub_count = 0;        // this many vertices, spread over the id range, get exactly
  int64_t hub_degree = 0;       // hub_degree out-edges each; the others share the remaining edges
};

struct GenSummary {
  int64_t n = 0, m = 0, max_degree = 0;
  uint64_t graph_bytes = 0, ts_bytes = 0, index_bytes = 0;
  EncoderStats stats;
};

// Generates, encodes and writes <dir>/<base>.{graph,offsets,properties,timestamps} plus the four
// GPU index files.  raw_path, when not empty, also receives the 4-column text edge list.
GenSummary generate_dataset(const GenParams& p, const std::string& dir, const std::string& base,
                            const std::string& raw_path);

}  // namespace tga
