// Format layer: writers for the compressed temporal multigraph and its GPU index.
//
// Files produced for a dataset stored under <dir>/<base>:
//   <base>.graph       successor lists, BVMultiGraph layout (BVMultiGraph.java:1640-1852)
//   <base>.offsets     gamma-coded bit deltas between consecutive records, n+1 codes
//                      (BVMultiGraph.java:1911-1915,1982)
//   <base>.properties  java.util.Properties-style summary (BVMultiGraph.java:2101-2200)
//   <base>.timestamps  64-bit minimum timestamp, then per edge zeta_2(int2nat(t_i - t_{i-1})),
//                      t_{-1} = minimum, restarted for every source (EvolvingMultiGraph.java:131-144,
//                      202-267)
//   graph_lower_bits.bin / graph_upper_bits.bin,
//   timestamp_lower_bits.bin / timestamp_upper_bits.bin
//                      Elias-Fano index of the per-vertex bit offsets of the two streams, in the
//                      layout read by gpu_cuda/shared/bfs.cu:543-565 (value = ((select1(upper,i)-i)
//                      << l) | low_i, low bits l wide and MSB-first, upper bits LSB-first in
//                      little-endian 64-bit words, l = (int)log2(fileBytes*8 / MAX_LABEL) from
//                      bfs.cu:1785-1786).  The reference ships no producer for these files.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "bitio.hpp"

namespace tga {

struct EncoderParams {
  int window_size = 7;       // BVMultiGraph.DEFAULT_WINDOW_SIZE
  int max_ref_count = 3;     // BVMultiGraph.DEFAULT_MAX_REF_COUNT
  int min_interval = 4;      // BVMultiGraph.DEFAULT_MIN_INTERVAL_LENGTH
  int min_multiple = 2;      // BVMultiGraph.DEFAULT_MIN_MULTIPLE_LENGTH
  int zeta_k = 3;            // BVMultiGraph.DEFAULT_ZETA_K (residuals)
  int ts_zeta_k = 2;         // BaselineRunner.ZETA_K (timestamps)
  // Never reference a list when the copy mask would start with an empty copy block (a valid
  // record, but one that the reference's GPU decoder reads differently): for datasets that its
  // GPU programs must decode as the format defines.
  bool no_empty_first_copy = false;
};

struct EncoderStats {
  int64_t nodes = 0, arcs = 0, tot_ref = 0, tot_dist = 0;
  int64_t copied_arcs = 0, intervalised_arcs = 0, residual_arcs = 0, multiples_arcs = 0;
  int64_t bits_outdegrees = 0, bits_references = 0, bits_blocks = 0, bits_residuals = 0;
  int64_t bits_intervals = 0, bits_multiples = 0;
  int64_t max_chain = 0;
};

// Scratch of one diff_comp evaluation (one per thread of the block encoder).
struct DiffScratch {
  std::vector<int32_t> mult_left, mult_len, singles, extras, blocks, left, len, residuals;
};

// Streaming successor-list encoder.  Nodes must be added in id order 0..n-1, each with
// its successor list sorted by value (duplicates = parallel temporal edges).
class GraphEncoder {
 public:
  explicit GraphEncoder(EncoderParams p = {});
  void add_node(const int32_t* succ, int outd);
  // The next `count` nodes at once, on `threads` threads, with the same bytes, offsets and
  // statistics as `count` calls of add_node.  A node's reference choice depends on earlier choices
  // (the chain-depth limit), but the costs it compares do not: the costs of every candidate of
  // every node are computed in parallel, the choices are made in node order, and the records are
  // written in parallel into separate streams that are then joined bit by bit.
  void add_block(const int32_t* const* succ, const int* outd, int count, int threads);
  void finish();  // writes the last offset delta
  BitWriter graph, offsets;
  std::vector<uint64_t> node_bit_offsets;  // n+1 entries
  EncoderStats stats;
  EncoderParams params;

 private:
  int cur_node_ = 0;
  uint64_t last_bit_ = 0;
  std::vector<std::vector<int32_t>> list_;
  std::vector<int> list_len_, ref_count_;
  DiffScratch scratch_;
};

// Threads of the block encoders: $TGA_ENCODE_THREADS, else the hardware's (at most 32); 0 means
// node by node (add_node).  The encoded files are the same for every value.
int encode_threads();

// Streaming timestamp writer (one call per node, in node order).
class TimestampEncoder {
 public:
  TimestampEncoder(int64_t min_timestamp, int zeta_k = 2);
  void add_node(const int64_t* ts, int count);
  // The next `nodes` nodes at once on `threads` threads (same bytes and offsets as add_node).
  void add_block(const int64_t* const* ts, const int* count, int nodes, int threads);
  void finish();
  BitWriter out;
  std::vector<uint64_t> node_bit_offsets;  // n+1 entries (first = 64)
  int64_t min_timestamp;
  int zeta_k;
};

// Elias-Fano index in the reference GPU layout.
struct EFIndex {
  int l = 0;
  std::vector<uint8_t> lower, upper;
};
int ef_low_bits(uint64_t stream_bytes, int64_t max_label);
EFIndex ef_build(const std::vector<uint64_t>& values, int l);
uint64_t ef_get_host(const EFIndex& ef, uint64_t i);

// Java-semantics parse of 4-column raw lines "src dst w ts" (ArcListASCIIEvolvingGraph.java:
// 150-228, EvolvingMultiGraph.java:202-267): sources must be non-decreasing, successors are
// sorted by value per source while timestamps keep line order.
struct RawGraph {
  int64_t n = 0;
  std::vector<int64_t> src_begin;  // per node index into dst/ts (n+1)
  std::vector<int32_t> dst;
  std::vector<int64_t> ts;
  int64_t min_ts = 0;
};
RawGraph parse_raw_text(const std::string& text);

struct WrittenDataset {
  uint64_t graph_bytes = 0, ts_bytes = 0, index_bytes = 0;
  int64_t n = 0, m = 0;
  int gl = 0, tl = 0;
  EncoderStats stats;
};

// Writes every file of a dataset from finished encoders (max_label < 0 means n - 1).
WrittenDataset write_dataset(const std::string& dir, const std::string& base, const GraphEncoder& ge,
                             const TimestampEncoder& te, int64_t n, int64_t max_label);

// Encodes a whole in-memory temporal graph and writes every file of the dataset.
// max_label < 0 means n - 1.
WrittenDataset encode_and_write(const RawGraph& g, const std::string& dir, const std::string& base,
                                int64_t max_label, const EncoderParams& p = {});

// The four GPU index files' content for a directory that holds the webgraph offsets the Java
// encoder writes instead of them: graph record offsets from <base>.offsets (n+1 gamma-coded deltas,
// BVMultiGraph.java:1913-1922), each record's outdegree from the gamma at its start, and the
// timestamp offsets by walking the timestamp stream (after its 64-bit header, outdegree(v) zeta_k
// codes per vertex, EvolvingMultiGraph.java:131-275).  EF widths as the reference reader expects
// (ef_low_bits of each stream).  Throws std::runtime_error on malformed input.
void index_from_offsets(const std::vector<uint8_t>& graph, const std::vector<uint8_t>& offsets,
                        const std::vector<uint8_t>& timestamps, int64_t n, int ts_zeta_k, int64_t max_label,
                        EFIndex* graph_ef, EFIndex* ts_ef);

// The same offsets walked on the GPU (indexbuild.cu: speculative chunked decoding of the offsets
// and timestamp streams): graph record offsets goff[0..n] and timestamp offsets toff[0..n], which
// ef_build packs as index_from_offsets does.  Returns a TGA_E_* code (TGA_E_TIMEOUT when the
// speculative chunks did not fall into step, for which the host walk is the answer).
int offsets_on_device(const std::vector<uint8_t>& graph, const std::vector<uint8_t>& offsets,
                      const std::vector<uint8_t>& timestamps, int64_t n, std::vector<uint64_t>& goff,
                      std::vector<uint64_t>& toff);

std::map<std::string, std::string> read_properties(const std::string& path);

// Realised reference-chain depth of every list (ReferenceDepthScanner.java:24-87): a list that
// copies from the list `ref` positions back has depth one more than that list, others depth 0.
// Reads each record's outdegree and reference only, entering it at its offset from <base>.offsets
// (gamma-coded bit-position deltas, n+1 of them).  window_size 0 means records carry no
// reference.  Throws std::runtime_error on malformed input.
std::vector<int32_t> reference_depths(const std::vector<uint8_t>& graph, const std::vector<uint8_t>& offsets,
                                      int64_t n, int window_size);
bool write_file(const std::string& path, const void* data, size_t n);
bool read_file(const std::string& path, std::vector<uint8_t>& out);

}  // namespace tga
