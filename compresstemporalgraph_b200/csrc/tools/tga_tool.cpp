// Drop-in executables for the reference's seven per-dataset programs
// (gpu_cuda/<DS>/{bfs,connected_components,degree_centrality,graph_coloring,hits,neighbor_access,
// pagerank}.cu -> gpu_cuda/shared/<alg>.cu main()).  One binary picks its workload from the name
// it is run under (the build links the seven names to it) or from its first argument
// (`tga_tool bfs ...`).  It runs on the C ABI of libtga only.
//
// What stays the same as the reference:
//   - the files and paths: <root>/data/compressed/<STORAGE>/<STORAGE>.* with root from --root,
//     else $TGA_COMPRESS_ROOT, else ../.. (shared/path_config.cuh:10-24,
//     shared/dataset_config_base.cuh:39-67);
//   - the per-dataset settings (gpu_cuda/<DS>/dataset_config.cuh), here runtime options, with the
//     six shipped datasets as presets;
//   - what each program computes (full time window, the reference's CC early exits, cuRAND
//     colouring priorities, GPU-semantics HITS, TEMPORAL_ALPHA 0.1 and damping 0.85);
//   - the stdout lines ("Starting simple parallel bfs.", "BFS Elapsed time in milliseconds : %li ms.",
//     ..., shared/bfs.cu:1995,2041, connected_components.cu:2154, degree_centrality.cu:1948,1956,
//     graph_coloring.cu:2002,2010, hits.cu:2258,2352, neighbor_access.cu:1930,
//     pagerank.cu:1952,2010) and the optional PageRank summary line (pagerank.cu:2012-2042, enabled
//     there by compiling with TGA_DUMP_RANK_SUMMARY=1, here by --rank-summary or that variable
//     in the environment);
//   - a missing file prints "Cannot open required file: <path> (set TGA_COMPRESS_ROOT if needed)"
//     on stderr and exits with EXIT_FAILURE (path_config.cuh:26-36); a CUDA or decode error also
//     exits 1 (the reference's CHECK -> exit(1), bfs.cu:23-32).
// What is added: a time window, a BFS source, --json (one JSON result line), --out (raw result
// arrays), --repeat (several runs on one load) and --autotune.  Bad arguments exit 2.
//
// The elapsed lines report the device time of the call (CUDA events on the graph's stream,
// tga_get_timing); the reference times its host loop with steady_clock.  --json gives both.
#include <cerrno>
#include <chrono>
#include <cinttypes>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tga.h"

namespace {

enum class Alg { BFS, CC, DC, GC, HITS, NA, PR, NONE };

struct AlgName {
  const char* name;
  Alg alg;
};
constexpr AlgName kAlgs[] = {{"bfs", Alg::BFS},
                             {"connected_components", Alg::CC},
                             {"degree_centrality", Alg::DC},
                             {"graph_coloring", Alg::GC},
                             {"hits", Alg::HITS},
                             {"neighbor_access", Alg::NA},
                             {"pagerank", Alg::PR}};

Alg alg_of(const std::string& s) {
  for (const auto& a : kAlgs)
    if (s == a.name) return a.alg;
  return Alg::NONE;
}

const char* name_of(Alg a) {
  for (const auto& x : kAlgs)
    if (x.alg == a) return x.name;
  return "?";
}

// The per-dataset macros of the six datasets the reference ships (gpu_cuda/<DS>/dataset_config.cuh);
// every field not listed keeps the default of shared/dataset_config_base.cuh.
struct Preset {
  const char* name;
  const char* storage;
  int32_t max_label, max_vertex;
  int64_t min_timestamp;
  int32_t min_graph_vertex, multiple_initial_value, pr_iters, hits_iters;
  int32_t active_vertex_begin, bfs_start_vertex, cc_vertex_begin;
};
constexpr Preset kPresets[] = {
    {"Comm", nullptr, 9999, 10000, 0, 0, -1, 10, 10, 0, 1, 1},
    {"MyD", nullptr, 999967, 1000001, 0, 0, -1, 10, 10, 0, 1, 1},
    {"Flickr", nullptr, 2585568, 2585570, 0, 0, -1, 10, 10, 0, 1, 1},
    {"Wiki", nullptr, 42640545, 42640546, 979675713, 1, 0, 100, 100, 0, 1, 1},
    {"Yahoo", nullptr, 102867214, 102867263, 1206214540, 0, -1, 10, 10, 0, 1, 1},
    {"Yahoo-sub", "Yahoo", 102867214, 102867263, 1206214540, 0, -1, 10, 10, 2000, 2001, 2000},
};

struct Options {
  Alg alg = Alg::NONE;
  std::string prog;
  std::string dataset, storage, root, dir, base;
  bool have_max_label = false, have_max_vertex = false;
  tga_dataset_cfg cfg{};
  bool have_window = false;
  int64_t t_lo = TGA_T_MIN, t_hi = TGA_T_MAX;
  int32_t src = -1;
  bool early_exit = true;
  int32_t hits_mode = TGA_HITS_GPU;
  int32_t prio_mode = 0;
  bool java_isolated = false;
  bool json = false, rank_summary = false, autotune = false, show_config = false;
  std::string out;
  int repeat = 1;
};

void usage(FILE* f, const char* prog) {
  std::fprintf(f,
               "usage: %s [options]            (or: tga_tool <algorithm> [options])\n"
               "       tga_tool prepare <raw-input[.gz]> <output-basename> [max-label]\n"
               "       tga_tool reference_depths <graph-basename>   (ReferenceDepthScanner's report)\n"
               "algorithms: bfs connected_components degree_centrality graph_coloring hits\n"
               "            neighbor_access pagerank\n"
               "dataset (the reference's per-dataset macros; Comm, MyD, Flickr, Wiki, Yahoo and\n"
               "Yahoo-sub load their shipped settings, later options override them):\n"
               "  --dataset NAME        DATASET_NAME (required)\n"
               "  --storage NAME        DATASET_STORAGE_NAME (default: NAME)\n"
               "  --max-label N         MAX_LABEL (required for other names)\n"
               "  --max-vertex N        MAX_Vertex (default: MAX_LABEL + 1)\n"
               "  --min-timestamp T     minTimestamp (default: from the .timestamps header)\n"
               "  --min-graph-vertex N  MIN_GRAPH_VERTEX\n"
               "  --active-begin N      ACTIVE_VERTEX_BEGIN\n"
               "  --bfs-start N         BFS_START_VERTEX\n"
               "  --cc-begin N          CONNECTED_COMPONENTS_VERTEX_BEGIN\n"
               "  --multiple-initial N  MULTIPLE_INITIAL_VALUE\n"
               "  --pr-iters N          PAGERANK_ITERATIONS\n"
               "  --hits-iters N        HITS_ITERATIONS\n"
               "  --root DIR            repository root (default: $TGA_COMPRESS_ROOT, else ../..)\n"
               "  --dir DIR --base B    read DIR/B.* and DIR's index files instead\n"
               "query:\n"
               "  --window LO:HI        time window; [LO, HI) for bfs, connected_components, hits and\n"
               "                        pagerank, [LO, HI] for degree_centrality (default: all edges)\n"
               "  --src V               bfs source (default: BFS_START_VERTEX)\n"
               "  --no-early-exit       connected_components without the reference's early exits\n"
               "  --hits-java           hits with the Java reset-per-half-step semantics\n"
               "  --prio curand|java    graph_coloring priorities (default: curand, as the reference)\n"
               "  --java-isolated       graph_coloring colours vertices without out-edges in round 0\n"
               "output:\n"
               "  --json                one JSON result line after the reference's lines\n"
               "  --out FILE            raw little-endian result arrays of max_vertex entries each:\n"
               "                        bfs arrival i32, hops i32; connected_components label i32;\n"
               "                        degree_centrality degree i32, mean time i64; graph_coloring\n"
               "                        colour u32, priority u32; hits hub f32, authority f32;\n"
               "                        neighbor_access degree i32, checksum u64, small u8;\n"
               "                        pagerank rank f32\n"
               "  --rank-summary        pagerank: the reference's rank_sum / top10 line\n"
               "                        (also when TGA_DUMP_RANK_SUMMARY is set to a non-zero value)\n"
               "  --repeat N            run the workload N times on one load (one elapsed line each)\n"
               "  --autotune            time the work decompositions first and keep the fastest\n"
               "  --show-config         print the resolved dataset settings as JSON and exit\n"
               "exit status: 0 ok, 1 missing file / CUDA / decode / format error, 2 bad arguments\n",
               prog);
}

[[noreturn]] void bad_args(const Options& o, const std::string& msg) {
  std::fprintf(stderr, "%s: %s\n", o.prog.c_str(), msg.c_str());
  usage(stderr, o.prog.c_str());
  std::exit(2);
}

bool parse_i64(const char* s, int64_t* v) {
  if (!s || !*s) return false;
  errno = 0;
  char* end = nullptr;
  const long long x = std::strtoll(s, &end, 10);
  if (errno || *end) return false;
  *v = (int64_t)x;
  return true;
}

int64_t need_i64(const Options& o, const char* opt, const char* s, int64_t lo, int64_t hi) {
  int64_t v;
  if (!parse_i64(s, &v) || v < lo || v > hi) bad_args(o, std::string("bad value for ") + opt + ": " + (s ? s : "(missing)"));
  return v;
}

void apply_preset(Options& o, const Preset& p) {
  o.cfg.max_label = p.max_label;
  o.cfg.max_vertex = p.max_vertex;
  o.cfg.min_timestamp = p.min_timestamp;
  o.cfg.min_graph_vertex = p.min_graph_vertex;
  o.cfg.multiple_initial_value = p.multiple_initial_value;
  o.cfg.pr_iters = p.pr_iters;
  o.cfg.hits_iters = p.hits_iters;
  o.cfg.active_vertex_begin = p.active_vertex_begin;
  o.cfg.bfs_start_vertex = p.bfs_start_vertex;
  o.cfg.cc_vertex_begin = p.cc_vertex_begin;
  if (p.storage && o.storage.empty()) o.storage = p.storage;
  o.have_max_label = o.have_max_vertex = true;
}

Options parse(int argc, char** argv) {
  Options o;
  tga_cfg_default(&o.cfg);
  std::string self = argv[0];
  const size_t slash = self.find_last_of('/');
  if (slash != std::string::npos) self = self.substr(slash + 1);
  o.prog = self;
  int i = 1;
  o.alg = alg_of(self);
  if (o.alg == Alg::NONE) {
    if (argc > 1 && (!std::strcmp(argv[1], "--help") || !std::strcmp(argv[1], "-h"))) {
      usage(stdout, o.prog.c_str());
      std::exit(0);
    }
    if (argc < 2) bad_args(o, "no algorithm given");
    o.alg = alg_of(argv[1]);
    if (o.alg == Alg::NONE) bad_args(o, std::string("unknown algorithm: ") + argv[1]);
    o.prog = self + " " + argv[1];
    i = 2;
  }
  // Options that the preset must not override are collected first and applied after it.
  std::vector<std::pair<std::string, const char*>> later;
  for (; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&]() -> const char* {
      if (i + 1 >= argc) bad_args(o, "missing value for " + a);
      return argv[++i];
    };
    if (a == "--help" || a == "-h") {
      usage(stdout, o.prog.c_str());
      std::exit(0);
    } else if (a == "--dataset") o.dataset = val();
    else if (a == "--storage") o.storage = val();
    else if (a == "--root") o.root = val();
    else if (a == "--dir") o.dir = val();
    else if (a == "--base") o.base = val();
    else if (a == "--max-label" || a == "--max-vertex" || a == "--min-timestamp" || a == "--min-graph-vertex" ||
             a == "--active-begin" || a == "--bfs-start" || a == "--cc-begin" || a == "--multiple-initial" ||
             a == "--pr-iters" || a == "--hits-iters")
      later.emplace_back(a, val());
    else if (a == "--window") {
      const std::string w = val();
      const size_t c = w.find(':');
      if (c == std::string::npos || !parse_i64(w.substr(0, c).c_str(), &o.t_lo) ||
          !parse_i64(w.substr(c + 1).c_str(), &o.t_hi) || o.t_lo < 0 || o.t_hi < o.t_lo)
        bad_args(o, "bad --window (want LO:HI with 0 <= LO <= HI): " + w);
      o.have_window = true;
    } else if (a == "--src") o.src = (int32_t)need_i64(o, "--src", val(), 0, INT32_MAX);
    else if (a == "--no-early-exit") o.early_exit = false;
    else if (a == "--hits-java") o.hits_mode = TGA_HITS_JAVA;
    else if (a == "--prio") {
      const std::string p = val();
      if (p == "curand") o.prio_mode = 0;
      else if (p == "java") o.prio_mode = 1;
      else bad_args(o, "bad --prio (want curand or java): " + p);
    } else if (a == "--java-isolated") o.java_isolated = true;
    else if (a == "--json") o.json = true;
    else if (a == "--out") o.out = val();
    else if (a == "--rank-summary") o.rank_summary = true;
    else if (a == "--repeat") o.repeat = (int)need_i64(o, "--repeat", val(), 1, 1000000);
    else if (a == "--autotune") o.autotune = true;
    else if (a == "--show-config") o.show_config = true;
    else bad_args(o, "unknown option: " + a);
  }
  if (o.dir.empty() != o.base.empty()) bad_args(o, "--dir and --base go together");
  if (!o.dir.empty() && !o.root.empty()) bad_args(o, "--root and --dir exclude each other");
  if (o.dataset.empty() && o.base.empty()) bad_args(o, "--dataset (or --dir with --base) is required");
  if (o.dataset.empty()) o.dataset = o.base;
  for (const auto& p : kPresets)
    if (o.dataset == p.name) apply_preset(o, p);
  for (const auto& kv : later) {
    const std::string& k = kv.first;
    const char* v = kv.second;
    if (k == "--max-label") {
      o.cfg.max_label = (int32_t)need_i64(o, "--max-label", v, 0, INT32_MAX - 1);
      o.have_max_label = true;
    } else if (k == "--max-vertex") {
      o.cfg.max_vertex = (int32_t)need_i64(o, "--max-vertex", v, 1, INT32_MAX);
      o.have_max_vertex = true;
    } else if (k == "--min-timestamp") o.cfg.min_timestamp = need_i64(o, "--min-timestamp", v, 0, INT64_MAX);
    else if (k == "--min-graph-vertex") o.cfg.min_graph_vertex = (int32_t)need_i64(o, "--min-graph-vertex", v, 0, INT32_MAX);
    else if (k == "--active-begin") o.cfg.active_vertex_begin = (int32_t)need_i64(o, "--active-begin", v, 0, INT32_MAX);
    else if (k == "--bfs-start") o.cfg.bfs_start_vertex = (int32_t)need_i64(o, "--bfs-start", v, 0, INT32_MAX);
    else if (k == "--cc-begin") o.cfg.cc_vertex_begin = (int32_t)need_i64(o, "--cc-begin", v, 0, INT32_MAX);
    else if (k == "--multiple-initial") o.cfg.multiple_initial_value = (int32_t)need_i64(o, "--multiple-initial", v, INT32_MIN, INT32_MAX);
    else if (k == "--pr-iters") o.cfg.pr_iters = (int32_t)need_i64(o, "--pr-iters", v, 1, INT32_MAX);
    else if (k == "--hits-iters") o.cfg.hits_iters = (int32_t)need_i64(o, "--hits-iters", v, 1, INT32_MAX);
  }
  if (!o.have_max_label) bad_args(o, "--max-label is required for dataset " + o.dataset);
  if (!o.have_max_vertex) o.cfg.max_vertex = o.cfg.max_label + 1;
  if (o.cfg.max_vertex <= o.cfg.max_label) bad_args(o, "--max-vertex must exceed --max-label");
  if (o.have_window && (o.alg == Alg::GC || o.alg == Alg::NA))
    bad_args(o, std::string(name_of(o.alg)) + " takes no --window");
  if (o.alg == Alg::DC && !o.have_window) o.t_lo = o.t_hi = 0;  // (0,0): all edges
  if (const char* e = std::getenv("TGA_DUMP_RANK_SUMMARY"))
    if (*e && std::strcmp(e, "0") != 0) o.rank_summary = true;
  return o;
}

// Library failure: the message as the library wrote it (for a missing file, the reference's own
// line), exit status 1 as the reference's exit(EXIT_FAILURE) / CHECK -> exit(1).
[[noreturn]] void fail(const Options& o, int rc, const char* what) {
  if (rc == TGA_E_IO) std::fprintf(stderr, "%s\n", tga_last_error());
  else std::fprintf(stderr, "%s: %s failed (status %d): %s\n", o.prog.c_str(), what, rc, tga_last_error());
  std::exit(rc == TGA_E_ARG ? 2 : 1);
}

uint64_t fnv1a(const void* p, size_t n, uint64_t h = 0xcbf29ce484222325ull) {
  const auto* b = static_cast<const uint8_t*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

struct Outputs {
  std::vector<int32_t> i32a, i32b;
  std::vector<int64_t> i64;
  std::vector<uint32_t> u32a, u32b;
  std::vector<uint64_t> u64;
  std::vector<uint8_t> u8;
  std::vector<float> f32a, f32b;
  int32_t components = 0, rounds = 0;
};

// One run of the workload; the reference's "Starting ..." line comes first, as there.
void run_once(const Options& o, tga_graph* g, Outputs& r) {
  int rc = TGA_OK;
  switch (o.alg) {
    case Alg::BFS:
      std::printf("Starting simple parallel bfs.\n");
      std::fflush(stdout);
      rc = tga_bfs(g, o.src, o.t_lo, o.t_hi, r.i32a.data(), r.i32b.data());
      break;
    case Alg::CC:
      rc = tga_cc(g, o.t_lo, o.t_hi, o.early_exit ? TGA_CC_EARLY_EXIT : 0, r.i32a.data(), &r.components);
      break;
    case Alg::DC:
      std::printf("Starting simple parallel Degree Centre.\n");
      std::fflush(stdout);
      rc = tga_degree(g, o.t_lo, o.t_hi, r.i32a.data(), r.i64.data());
      break;
    case Alg::GC:
      std::printf("Starting simple parallel Graph Color.\n");
      std::fflush(stdout);
      rc = tga_color(g, o.prio_mode, nullptr, o.java_isolated ? TGA_GC_JAVA_ISOLATED : 0, r.u32a.data(), r.u32b.data(),
                     &r.rounds);
      break;
    case Alg::HITS:
      std::printf("Starting simple parallel HITS.\n");
      std::fflush(stdout);
      rc = tga_hits(g, 0, o.hits_mode, o.t_lo, o.t_hi, r.f32a.data(), r.f32b.data());
      break;
    case Alg::NA:
      rc = tga_neighbor_access(g, r.u8.data(), r.u64.data(), r.i32a.data());
      break;
    case Alg::PR:
      std::printf("Starting simple parallel PageRank.\n");
      std::fflush(stdout);
      rc = tga_pagerank(g, 0, 0.85f, 0.1f, o.t_lo, o.t_hi, r.f32a.data());
      break;
    case Alg::NONE:
      break;
  }
  if (rc) fail(o, rc, name_of(o.alg));
}

void print_elapsed(Alg a, double ms) {
  const long whole = (long)ms;
  switch (a) {
    case Alg::BFS: std::printf("BFS Elapsed time in milliseconds : %li ms.\n", whole); break;
    case Alg::PR: std::printf("PageRank Elapsed time in milliseconds : %li ms.\n", whole); break;
    case Alg::NA: std::printf("Time = %g ms.\n", ms); break;
    default: std::printf("Elapsed time in milliseconds : %li ms.\n", whole); break;
  }
}

// pagerank.cu:2012-2042: sum of all max_vertex ranks and the ten largest, ties to the lower id.
void print_rank_summary(const std::vector<float>& rank) {
  constexpr int K = 10;
  int idx[K];
  double val[K];
  for (int k = 0; k < K; ++k) {
    idx[k] = -1;
    val[k] = -1.0;
  }
  double sum = 0;
  for (size_t v = 0; v < rank.size(); ++v) {
    const double x = rank[v];
    sum += x;
    int k = 0;
    while (k < K && !(x > val[k])) ++k;
    if (k == K) continue;
    for (int j = K - 1; j > k; --j) {
      val[j] = val[j - 1];
      idx[j] = idx[j - 1];
    }
    val[k] = x;
    idx[k] = (int)v;
  }
  std::printf("PageRank alpha=%.12g rank_sum=%.12g top10=", 0.1, sum);
  for (int k = 0; k < K; ++k) std::printf("%s%d:%.12g", k ? "," : "", idx[k], val[k]);
  std::printf("\n");
}

template <class T>
bool write_raw(FILE* f, const std::vector<T>& v) {
  return v.empty() || std::fwrite(v.data(), sizeof(T), v.size(), f) == v.size();
}

std::string json_str(const std::string& s) {
  std::string r = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') r += '\\';
    if ((unsigned char)c < 0x20) {
      char b[8];
      std::snprintf(b, sizeof b, "\\u%04x", (unsigned)(unsigned char)c);
      r += b;
    } else {
      r += c;
    }
  }
  return r + "\"";
}

// A JSON number, or null when the value is not finite (JSON has no NaN or infinity).
std::string num(double x, const char* fmt = "%.9g") {
  if (!std::isfinite(x)) return "null";
  char b[64];
  std::snprintf(b, sizeof b, fmt, x);
  return b;
}

std::string hex64(uint64_t h) {
  char b[24];
  std::snprintf(b, sizeof b, "\"%016" PRIx64 "\"", h);
  return b;
}

// Result summary of the last run for the JSON line.
std::string summary(const Options& o, const Outputs& r) {
  char b[512];
  std::string s;
  switch (o.alg) {
    case Alg::BFS: {
      int64_t reached = 0;
      int32_t max_hops = 0;
      for (size_t v = 0; v < r.i32a.size(); ++v)
        if (r.i32a[v] != INT32_MAX) {
          ++reached;
          if (r.i32b[v] > max_hops) max_hops = r.i32b[v];
        }
      std::snprintf(b, sizeof b, "\"reached\": %" PRId64 ", \"max_hops\": %d, \"arrival_fnv1a\": ", reached, max_hops);
      s = b + hex64(fnv1a(r.i32a.data(), r.i32a.size() * 4)) + ", \"hops_fnv1a\": " + hex64(fnv1a(r.i32b.data(), r.i32b.size() * 4));
      break;
    }
    case Alg::CC: {
      int64_t labelled = 0;
      for (int32_t l : r.i32a) labelled += l != -1;
      std::snprintf(b, sizeof b, "\"components\": %d, \"labelled\": %" PRId64 ", \"label_fnv1a\": ", r.components, labelled);
      s = b + hex64(fnv1a(r.i32a.data(), r.i32a.size() * 4));
      break;
    }
    case Alg::DC: {
      int64_t sum = 0;
      for (int32_t d : r.i32a) sum += d;
      std::snprintf(b, sizeof b, "\"degree_sum\": %" PRId64 ", \"degree_fnv1a\": ", sum);
      s = b + hex64(fnv1a(r.i32a.data(), r.i32a.size() * 4)) + ", \"mean_fnv1a\": " + hex64(fnv1a(r.i64.data(), r.i64.size() * 8));
      break;
    }
    case Alg::GC: {
      int64_t coloured = 0;
      for (uint32_t c : r.u32a) coloured += c != UINT32_MAX;
      std::snprintf(b, sizeof b, "\"rounds\": %d, \"coloured\": %" PRId64 ", \"color_fnv1a\": ", r.rounds, coloured);
      s = b + hex64(fnv1a(r.u32a.data(), r.u32a.size() * 4));
      break;
    }
    case Alg::HITS: {
      double hs = 0, as = 0;
      for (float x : r.f32a) hs += (double)x * x;
      for (float x : r.f32b) as += (double)x * x;
      s = "\"hub_l2sq\": " + num(hs) + ", \"auth_l2sq\": " + num(as);
      break;
    }
    case Alg::NA: {
      int64_t edges = 0, small = 0;
      uint64_t csum = 0;
      for (int32_t d : r.i32a) edges += d;
      for (uint8_t x : r.u8) small += x;
      for (uint64_t c : r.u64) csum += c;
      std::snprintf(b, sizeof b, "\"edges\": %" PRId64 ", \"small\": %" PRId64 ", \"checksum_sum\": ", edges, small);
      s = b + hex64(csum);
      break;
    }
    case Alg::PR: {
      double sum = 0;
      size_t top = 0;
      for (size_t v = 0; v < r.f32a.size(); ++v) {
        sum += r.f32a[v];
        if (r.f32a[v] > r.f32a[top]) top = v;
      }
      std::snprintf(b, sizeof b, ", \"top_vertex\": %zu", top);
      s = "\"rank_sum\": " + num(sum) + b;
      break;
    }
    case Alg::NONE:
      break;
  }
  return s;
}

}  // namespace

// `tga_tool reference_depths <graph-basename>`: cpu_java ReferenceDepthScanner.java:89-110, same
// argument and RESULT line (host only, no GPU).
int reference_depths_main(int argc, char** argv) {
  if (argc != 3 || argv[2][0] == '-') {
    std::fprintf(stderr, "Usage: tga_tool reference_depths <graph-basename>\n");
    return 2;
  }
  const std::string bn = argv[2];
  const size_t slash = bn.find_last_of('/');
  const std::string dir = slash == std::string::npos ? "." : bn.substr(0, slash);
  const std::string base = slash == std::string::npos ? bn : bn.substr(slash + 1);
  tga_ref_depths r{};
  const int rc = tga_reference_depths(dir.c_str(), base.c_str(), &r, nullptr);
  if (rc) {
    std::fprintf(stderr, "%s\n", tga_last_error());
    return rc == TGA_E_ARG ? 2 : 1;
  }
  std::printf("RESULT basename=%s maximum_depth=%d configured_max_ref_count=%d referenced_nodes=%" PRId64
              " truncated_nodes=%" PRId64 " depth_counts=0:%" PRId64 ",1:%" PRId64 ",2:%" PRId64 ",3:%" PRId64 "\n",
              bn.c_str(), r.maximum_depth, r.configured_max_ref_count, r.referenced_nodes, r.truncated_nodes,
              r.depth_counts[0], r.depth_counts[1], r.depth_counts[2], r.depth_counts[3]);
  return 0;
}

// `tga_tool prepare <raw-input> <output-basename> [max-label]`: the dataset preparation of the
// reference (BaselineRunner.java:243-259 and its --prepare-only line, 657-666: a raw edge list,
// gzipped or not, through EvolvingMultiGraph.store), plus the four GPU index files (host only).
int prepare_main(int argc, char** argv) {
  if (argc < 4 || argc > 5 || argv[2][0] == '-') {
    std::fprintf(stderr, "Usage: tga_tool prepare <raw-input> <output-basename> [max-label]\n");
    return 2;
  }
  int64_t max_label = -1;
  if (argc == 5 && (!parse_i64(argv[4], &max_label) || max_label < 0)) {
    std::fprintf(stderr, "tga_tool prepare: bad max-label: %s\n", argv[4]);
    return 2;
  }
  const std::string bn = argv[3];
  const size_t slash = bn.find_last_of('/');
  const std::string dir = slash == std::string::npos ? "." : bn.substr(0, slash);
  const std::string base = slash == std::string::npos ? bn : bn.substr(slash + 1);
  tga_gen_summary s{};
  const int rc = tga_encode_raw(argv[2], dir.c_str(), base.c_str(), max_label, &s);
  if (rc) {
    std::fprintf(stderr, "%s\n", tga_last_error());
    return rc == TGA_E_ARG ? 2 : 1;
  }
  std::printf("PREPARED basename=%s nodes=%" PRId64 " arcs=%" PRId64 " graph_bytes=%" PRIu64 " timestamp_bytes=%" PRIu64
              " index_bytes=%" PRIu64 "\n",
              bn.c_str(), s.n, s.m, s.graph_bytes, s.timestamp_bytes, s.index_bytes);
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 2 && !std::strcmp(argv[1], "reference_depths")) return reference_depths_main(argc, argv);
  if (argc >= 2 && !std::strcmp(argv[1], "prepare")) return prepare_main(argc, argv);
  const Options o = parse(argc, argv);
  tga_dataset_cfg cfg = o.cfg;
  const std::string storage = o.storage.empty() ? o.dataset : o.storage;
  cfg.name = o.dataset.c_str();
  cfg.storage_name = storage.c_str();
  if (o.show_config) {
    const std::string mts = cfg.min_timestamp == TGA_UNSET_TS ? "null" : std::to_string(cfg.min_timestamp);
    std::printf("{\"DATASET_NAME\": %s, \"DATASET_STORAGE_NAME\": %s, \"MAX_LABEL\": %d, \"MAX_Vertex\": %d, "
                "\"minTimestamp\": %s, \"MIN_GRAPH_VERTEX\": %d, \"ACTIVE_VERTEX_BEGIN\": %d, \"BFS_START_VERTEX\": %d, "
                "\"CONNECTED_COMPONENTS_VERTEX_BEGIN\": %d, \"MULTIPLE_INITIAL_VALUE\": %d, \"PAGERANK_ITERATIONS\": %d, "
                "\"HITS_ITERATIONS\": %d}\n",
                json_str(o.dataset).c_str(), json_str(storage).c_str(), cfg.max_label, cfg.max_vertex, mts.c_str(),
                cfg.min_graph_vertex, cfg.active_vertex_begin, cfg.bfs_start_vertex, cfg.cc_vertex_begin,
                cfg.multiple_initial_value, cfg.pr_iters, cfg.hits_iters);
    return 0;
  }

  tga_graph* g = nullptr;
  const int orc = o.dir.empty() ? tga_open(o.root.empty() ? nullptr : o.root.c_str(), &cfg, &g)
                                : tga_open_dir(o.dir.c_str(), o.base.c_str(), &cfg, &g);
  if (orc) fail(o, orc, "opening the dataset");

  tga_tune_result tune{};
  if (o.autotune) {
    const int rc = tga_autotune(g, &tune);
    if (rc) fail(o, rc, "autotune");
  }

  const size_t nv = (size_t)o.cfg.max_vertex;
  Outputs r;
  switch (o.alg) {
    case Alg::BFS: r.i32a.resize(nv); r.i32b.resize(nv); break;
    case Alg::CC: r.i32a.resize(nv); break;
    case Alg::DC: r.i32a.resize(nv); r.i64.resize(nv); break;
    case Alg::GC: r.u32a.resize(nv); r.u32b.resize(nv); break;
    case Alg::HITS: r.f32a.resize(nv); r.f32b.resize(nv); break;
    case Alg::NA: r.u8.resize(nv); r.u64.resize(nv); r.i32a.resize(nv); break;
    case Alg::PR: r.f32a.resize(nv); break;
    case Alg::NONE: break;
  }

  tga_timing t{};
  double wall_ms = 0;
  for (int k = 0; k < o.repeat; ++k) {
    const auto t0 = std::chrono::steady_clock::now();
    run_once(o, g, r);
    wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const int rc = tga_get_timing(g, &t);
    if (rc) fail(o, rc, "reading the timing");
    print_elapsed(o.alg, t.total_ms);
    std::fflush(stdout);
  }
  if (o.alg == Alg::PR && o.rank_summary) print_rank_summary(r.f32a);

  if (!o.out.empty()) {
    FILE* f = std::fopen(o.out.c_str(), "wb");
    bool ok = f != nullptr;
    if (ok) {
      switch (o.alg) {
        case Alg::BFS: ok = write_raw(f, r.i32a) && write_raw(f, r.i32b); break;
        case Alg::CC: ok = write_raw(f, r.i32a); break;
        case Alg::DC: ok = write_raw(f, r.i32a) && write_raw(f, r.i64); break;
        case Alg::GC: ok = write_raw(f, r.u32a) && write_raw(f, r.u32b); break;
        case Alg::HITS: ok = write_raw(f, r.f32a) && write_raw(f, r.f32b); break;
        case Alg::NA: ok = write_raw(f, r.i32a) && write_raw(f, r.u64) && write_raw(f, r.u8); break;
        case Alg::PR: ok = write_raw(f, r.f32a); break;
        case Alg::NONE: break;
      }
      ok = (std::fclose(f) == 0) && ok;
    }
    if (!ok) {
      std::fprintf(stderr, "%s: cannot write %s\n", o.prog.c_str(), o.out.c_str());
      tga_close(g);
      return 1;
    }
  }

  if (o.json) {
    tga_info info{};
    int rc = tga_get_info(g, &info);
    if (rc) fail(o, rc, "reading the graph info");
    const double gteps = t.total_ms > 0 ? (double)t.edges_decoded / (t.total_ms * 1e6) : 0.0;
    std::string line = "{\"tool\": " + json_str(name_of(o.alg)) + ", \"dataset\": " + json_str(o.dataset) +
                       ", \"storage\": " + json_str(storage);
    char b[768];
    std::snprintf(b, sizeof b,
                  ", \"n\": %d, \"max_label\": %d, \"max_vertex\": %d, \"window\": [%" PRId64 ", %" PRId64
                  "], \"repeat\": %d, \"edges_decoded\": %" PRId64 ", \"iterations\": %d, \"launches\": %" PRId64
                  ", \"compressed_bytes\": %" PRIu64 ", \"device_bytes\": %" PRIu64,
                  info.n, info.max_label, info.max_vertex, o.t_lo, o.t_hi, o.repeat, t.edges_decoded, t.iterations,
                  t.launches, t.compressed_bytes, info.device_bytes);
    line += b;
    line += ", \"device_ms\": " + num(t.total_ms, "%.6f") + ", \"decode_ms\": " + num(t.decode_ms, "%.6f") +
            ", \"wall_ms\": " + num(wall_ms, "%.6f") + ", \"gteps\": " + num(gteps, "%.6f");
    if (o.autotune) {
      std::snprintf(b, sizeof b, ", \"tuned\": {\"slice_edges\": %d, \"item_edges\": %d, \"dense_div\": %d}",
                    tune.slice_edges, tune.item_edges, tune.dense_div);
      line += b;
    }
    const std::string s = summary(o, r);
    if (!s.empty()) line += ", " + s;
    line += "}";
    std::printf("%s\n", line.c_str());
  }
  tga_close(g);
  return 0;
}
