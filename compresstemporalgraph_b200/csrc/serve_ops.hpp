// Delivery entry points of the served form (server.cpp): batched BFS and PageRank that copy each
// query's row from the device batch straight into its own destination (no contiguous host
// staging).  Internal to the library (C++ linkage, implemented in batch.cu); same semantics as
// tga_bfs_batch and tga_pagerank_batch_iters.
#pragma once
#include <cstdint>

#include "../../include/tga.h"

namespace tga {
int bfs_batch_rows(tga_graph* g, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                   int32_t* const* rows);
int pagerank_batch_rows(tga_graph* g, int32_t nq, const int32_t* iters, float damping, float alpha,
                        const int64_t* t_lo, const int64_t* t_hi, float* const* rows);
}  // namespace tga
