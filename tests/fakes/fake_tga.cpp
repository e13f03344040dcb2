// A fake of the tga C ABI for testing the drop-in executables' host logic on a machine without a
// GPU: every call the tool makes returns fixed, easily predicted arrays.  $FAKE_TGA_FAIL=<status>
// makes the algorithm calls fail with that status and the message "fake failure".
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "tga.h"

struct tga_graph {
  tga_dataset_cfg cfg;
};

namespace {
int32_t g_nv = 0;
const char* g_err = "";

int status() {
  const char* e = std::getenv("FAKE_TGA_FAIL");
  if (e && *e) {
    g_err = "fake failure";
    return std::atoi(e);
  }
  return TGA_OK;
}
}  // namespace

extern "C" {
void tga_cfg_default(tga_dataset_cfg* c) {
  std::memset(c, 0, sizeof *c);
  c->min_timestamp = TGA_UNSET_TS;
  c->bfs_start_vertex = 1;
  c->cc_vertex_begin = 1;
  c->multiple_initial_value = -1;
  c->pr_iters = 10;
  c->hits_iters = 10;
}
const char* tga_last_error(void) { return g_err; }
static int open_fake(const tga_dataset_cfg* c, tga_graph** o) {
  *o = new tga_graph{*c};
  g_nv = c->max_vertex;
  return TGA_OK;
}
int tga_open(const char*, const tga_dataset_cfg* c, tga_graph** o) { return open_fake(c, o); }
int tga_open_dir(const char*, const char*, const tga_dataset_cfg* c, tga_graph** o) { return open_fake(c, o); }
int tga_close(tga_graph* g) {
  delete g;
  return TGA_OK;
}
int tga_get_info(tga_graph* g, tga_info* i) {
  std::memset(i, 0, sizeof *i);
  i->n = g_nv;
  i->max_label = g->cfg.max_label;
  i->max_vertex = g_nv;
  return TGA_OK;
}
int tga_get_timing(tga_graph*, tga_timing* t) {
  std::memset(t, 0, sizeof *t);
  t->total_ms = 12.75;
  t->edges_decoded = 1000;
  t->iterations = 3;
  return TGA_OK;
}
int tga_autotune(tga_graph*, tga_tune_result* r) {
  std::memset(r, 0, sizeof *r);
  r->slice_edges = 16;
  r->item_edges = 128;
  r->dense_div = 8;
  return TGA_OK;
}
int tga_bfs(tga_graph*, int32_t, int64_t, int64_t, int32_t* a, int32_t* h) {
  for (int32_t i = 0; i < g_nv; ++i) {
    a[i] = i % 3 ? i : INT32_MAX;
    h[i] = i % 7;
  }
  return status();
}
int tga_cc(tga_graph*, int64_t, int64_t, int32_t, int32_t* l, int32_t* c) {
  for (int32_t i = 0; i < g_nv; ++i) l[i] = i % 4 - 1;
  *c = 3;
  return status();
}
int tga_degree(tga_graph*, int64_t, int64_t, int32_t* d, int64_t* a) {
  for (int32_t i = 0; i < g_nv; ++i) {
    d[i] = i;
    a[i] = -i;
  }
  return status();
}
int tga_color(tga_graph*, int32_t, const uint32_t*, int32_t, uint32_t* c, uint32_t* p, int32_t* r) {
  for (int32_t i = 0; i < g_nv; ++i) {
    c[i] = i % 5 ? (uint32_t)(i % 5) : UINT32_MAX;
    p[i] = (uint32_t)(i * 7 % 256);
  }
  *r = 5;
  return status();
}
int tga_hits(tga_graph*, int32_t, int32_t, int64_t, int64_t, float* h, float* a) {
  for (int32_t i = 0; i < g_nv; ++i) {
    h[i] = i == 0 ? NAN : 0.5f;
    a[i] = 0.25f;
  }
  return status();
}
int tga_neighbor_access(tga_graph*, uint8_t* s, uint64_t* c, int32_t* d) {
  for (int32_t i = 0; i < g_nv; ++i) {
    s[i] = (uint8_t)(i & 1);
    c[i] = 0xFFFFFFFFFFFFFFFFull - (uint64_t)i;
    d[i] = 2 * i;
  }
  return status();
}
int tga_pagerank(tga_graph*, int32_t, float, float, int64_t, int64_t, float* r) {
  for (int32_t i = 0; i < g_nv; ++i) r[i] = (float)((i * 37) % 11) / 100.0f;
  return status();
}
int tga_reference_depths(const char*, const char*, tga_ref_depths*, int32_t*) { return TGA_E_ARG; }
int tga_encode_raw(const char*, const char*, const char*, int64_t, tga_gen_summary*) { return TGA_E_ARG; }
}
