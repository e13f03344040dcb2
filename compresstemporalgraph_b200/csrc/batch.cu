// Batched query entry points.  This first version answers the queries one after another with the
// single-query kernels; the bitmask multi-source traversal replaces it.
#include <cstring>
#include <vector>

#include "engine.hpp"

using namespace tga;

extern "C" {

int tga_bfs(tga_graph*, int32_t, int64_t, int64_t, int32_t*, int32_t*);
int tga_pagerank(tga_graph*, int32_t, float, float, int64_t, int64_t, float*);

int tga_bfs_batch(tga_graph* g, int32_t nsrc, const int32_t* src, const int64_t* t_lo, const int64_t* t_hi,
                  int32_t* arrival_out) {
  if (!g || nsrc < 0 || (nsrc && (!src || !t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  const size_t nv = (size_t)g->view.max_vertex;
  for (int32_t i = 0; i < nsrc; ++i) {
    const int rc = tga_bfs(g, src[i], t_lo[i], t_hi[i], arrival_out ? arrival_out + i * nv : nullptr, nullptr);
    if (rc) return rc;
  }
  return TGA_OK;
}

int tga_pagerank_batch(tga_graph* g, int32_t nq, int32_t iters, float damping, float alpha, const int64_t* t_lo,
                       const int64_t* t_hi, float* rank_out) {
  if (!g || nq < 0 || (nq && (!t_lo || !t_hi))) return fail(TGA_E_ARG, "bad argument");
  const size_t nv = (size_t)g->view.max_vertex;
  for (int32_t i = 0; i < nq; ++i) {
    const int rc = tga_pagerank(g, iters, damping, alpha, t_lo[i], t_hi[i], rank_out ? rank_out + i * nv : nullptr);
    if (rc) return rc;
  }
  return TGA_OK;
}

}  // extern "C"
