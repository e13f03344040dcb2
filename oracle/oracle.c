/*
 * oracle.c - CPU oracle for the compressed temporal-graph engine.  TEST INFRASTRUCTURE ONLY:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library,
 * and only as the checker / the timed CPU port.  Nothing in the product links it.
 *
 * It restates, with its own code and data structures, the reference's definitions:
 *   - instantaneous codes of dsiutils' InputBitStream as used by the reference
 *     (readGamma/readZeta/readUnary/readLongZeta at BVMultiGraph.java:485-563,
 *     EvolvingMultiGraph.java:374,379,434), read bit by bit from their definitions;
 *   - BVMultiGraph.successors (BVMultiGraph.java:738-886) with materialised lists:
 *     copy blocks masked over the fully decoded referenced list (MaskedIntIterator),
 *     multiples (IntMultiplesSequenceIterator.java:106-126), intervals, residuals
 *     (ResidualIntIterator, BVMultiGraph.java:655-707), merged pairwise with the
 *     equal-heads-once rule of MergedIntIterator in the same nesting as BVMultiGraph.java:853-878;
 *   - per-vertex graph offsets from the .offsets gamma deltas (BVMultiGraph.java:590-617),
 *     NOT from the GPU Elias-Fano files, and timestamp offsets by walking the .timestamps
 *     stream in vertex order (EvolvingMultiGraph.java:202-267), so the engine's index is
 *     checked independently;
 *   - timestamps t_i = t_{i-1} + nat2int(zeta_2), t_{-1} = 64-bit header
 *     (EvolvingMultiGraph.java:396-443);
 *   - the workloads with the result contracts of the engine (reference GPU kernels
 *     gpu_cuda/shared/{bfs,connected_components,pagerank,hits,degree_centrality,graph_coloring,
 *     neighbor_access}.cu and BaselineRunner.java:273-614), in FP64.
 * Parity against the Java encoder's bytes is unpinned (no JDK and no webgraph jars exist here);
 * the decode tables gpu_cuda/decode_tables/{gammaInA,zetaInA}.txt and the reference's known-answer
 * tests pin the codes.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INF32 0x7fffffff

typedef struct {
  const uint8_t* d;
  uint64_t nbits;
  int bad;
} obits;

static int ob_bit(obits* b, uint64_t* p) {
  if (*p >= b->nbits) { b->bad = 1; ++*p; return 1; }
  const int v = (b->d[*p >> 3] >> (7 - (*p & 7))) & 1;
  ++*p;
  return v;
}
static uint64_t ob_bits(obits* b, uint64_t* p, int n) {
  uint64_t v = 0;
  for (int i = 0; i < n; ++i) v = (v << 1) | (uint64_t)ob_bit(b, p);
  return v;
}
static uint64_t ob_unary(obits* b, uint64_t* p) {
  uint64_t z = 0;
  while (!ob_bit(b, p)) { if (++z > 200) { b->bad = 1; return 0; } }
  return z;
}
/* gamma: unary(m) then the m low bits of x+1 */
static uint64_t ob_gamma(obits* b, uint64_t* p) {
  const uint64_t m = ob_unary(b, p);
  if (m > 63) { b->bad = 1; return 0; }
  return ((1ull << m) | ob_bits(b, p, (int)m)) - 1;
}
/* zeta_k: unary(h), then minimal binary of x+1-2^(hk) over [0, 2^(hk)(2^k-1)) */
static uint64_t ob_zeta(obits* b, uint64_t* p, int k) {
  const uint64_t h = ob_unary(b, p);
  if (h * (uint64_t)k + (uint64_t)k > 63) { b->bad = 1; return 0; }
  const uint64_t left = 1ull << (h * k);
  const uint64_t v = ob_bits(b, p, (int)(h * k + k - 1));
  if (v < left) return v + left - 1;
  return ((v << 1) | (uint64_t)ob_bit(b, p)) - 1;
}
static int64_t orc_nat2int(uint64_t x) { return (x & 1) ? -(int64_t)(x >> 1) - 1 : (int64_t)(x >> 1); }

static int read_all(const char* path, uint8_t** out, uint64_t* n) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  *out = (uint8_t*)malloc((size_t)sz + 16);
  if (!*out) { fclose(f); return -1; }
  memset(*out + sz, 0, 16);
  if (sz && fread(*out, 1, (size_t)sz, f) != (size_t)sz) { fclose(f); free(*out); return -1; }
  fclose(f);
  *n = (uint64_t)sz;
  return 0;
}

typedef struct {
  uint8_t *g, *t, *o;
  uint64_t gn, tn, on;
  int64_t n;             /* vertices */
  uint64_t* goff;        /* n+1 */
  uint64_t* toff;        /* n+1 */
  int32_t* deg;          /* n */
  int64_t min_ts;
  int min_interval;
  /* materialised CSR (filled by orc_materialize) */
  int64_t* off;
  int32_t* dst;
  int64_t* ts;
  int64_t m;
  int err;
} orc;

typedef struct {
  int32_t* v;
  int64_t n, cap;
} ivec;
static void iv_push(ivec* a, int32_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 16;
    a->v = (int32_t*)realloc(a->v, (size_t)a->cap * sizeof(int32_t));
  }
  a->v[a->n++] = x;
}

/* MergedIntIterator: sorted union, one output per pair of equal heads. */
static void merge_once(const ivec* a, const ivec* b, ivec* out) {
  int64_t i = 0, j = 0;
  out->n = 0;
  while (i < a->n || j < b->n) {
    if (i == a->n) iv_push(out, b->v[j++]);
    else if (j == b->n) iv_push(out, a->v[i++]);
    else if (a->v[i] < b->v[j]) iv_push(out, a->v[i++]);
    else if (a->v[i] > b->v[j]) iv_push(out, b->v[j++]);
    else { iv_push(out, a->v[i]); ++i; ++j; }
  }
}

static int64_t outdeg_at(orc* o, int64_t x) {
  obits b = {o->g, o->gn * 8, 0};
  uint64_t p = o->goff[x];
  const int64_t d = (int64_t)ob_gamma(&b, &p);
  if (b.bad) o->err = 1;
  return d;
}

/* Successor list of x in Java order (with duplicates). */
static void decode_list(orc* o, int64_t x, ivec* out, int depth) {
  out->n = 0;
  if (x < 0 || x >= o->n || depth > 16) { o->err = 1; return; }
  obits b = {o->g, o->gn * 8, 0};
  uint64_t p = o->goff[x];
  const int64_t d = (int64_t)ob_gamma(&b, &p);
  if (d == 0) return;
  const int64_t ref = (int64_t)ob_unary(&b, &p);
  int64_t extra = d, bc = 0;
  int64_t* blocks = NULL;
  if (ref > 0) {
    bc = (int64_t)ob_gamma(&b, &p);
    blocks = (int64_t*)malloc((size_t)(bc + 1) * sizeof(int64_t));
    int64_t copied = 0, total = 0;
    for (int64_t i = 0; i < bc; ++i) {
      blocks[i] = (int64_t)ob_gamma(&b, &p) + (i == 0 ? 0 : 1);
      total += blocks[i];
      if (i % 2 == 0) copied += blocks[i];
    }
    if (bc % 2 == 0) copied += outdeg_at(o, x - ref) - total;
    extra = d - copied;
  }
  ivec M = {0}, I = {0}, R = {0}, IM = {0}, E = {0}, C = {0}, RL = {0};
  int64_t mc = 0, ic = 0;
  if (extra > 0) {
    mc = (int64_t)ob_gamma(&b, &p);
    int64_t prev = 0;
    for (int64_t i = 0; i < mc; ++i) {
      const int64_t left = i == 0 ? x + orc_nat2int(ob_gamma(&b, &p)) : (int64_t)ob_gamma(&b, &p) + prev + 1;
      const int64_t len = (int64_t)ob_gamma(&b, &p) + 2;
      prev = left;
      for (int64_t k = 0; k < len; ++k) iv_push(&M, (int32_t)left);
      extra -= len;
    }
  }
  if (extra > 0) {
    ic = (int64_t)ob_gamma(&b, &p);
    int64_t prev = 0;
    for (int64_t i = 0; i < ic; ++i) {
      const int64_t left = i == 0 ? x + orc_nat2int(ob_gamma(&b, &p)) : (int64_t)ob_gamma(&b, &p) + prev + 1;
      const int64_t len = (int64_t)ob_gamma(&b, &p) + o->min_interval;
      for (int64_t k = 0; k < len; ++k) iv_push(&I, (int32_t)(left + k));
      prev = left + len;
      extra -= len;
    }
  }
  if (extra > 0) {
    int64_t cur = x + orc_nat2int(ob_zeta(&b, &p, 3));
    iv_push(&R, (int32_t)cur);
    for (int64_t i = 1; i < extra; ++i) {
      cur += (int64_t)ob_zeta(&b, &p, 3) + 1;
      iv_push(&R, (int32_t)cur);
    }
  }
  if (b.bad) o->err = 1;
  /* extra part: Merged(Merged(intervals, multiples), residuals) when each is present */
  const ivec* im;
  if (mc + ic == 0) im = NULL;
  else if (mc <= 0) im = &I;
  else if (ic <= 0) im = &M;
  else { merge_once(&I, &M, &IM); im = &IM; }
  const ivec* ex;
  if (!im) ex = R.n ? &R : NULL;
  else if (R.n == 0) ex = im;
  else { merge_once(im, &R, &E); ex = &E; }
  if (ref > 0) {
    decode_list(o, x - ref, &RL, depth + 1);
    /* MaskedIntIterator over the referenced list */
    int64_t mi = 0, left, pos = 0;
    if (bc) { left = blocks[mi++]; } else left = -1;
    for (;;) {
      if (left == 0) {
        if (mi < bc) {
          pos += blocks[mi++];
          left = mi < bc ? blocks[mi++] : -1;
          continue;
        }
        break;
      }
      if (pos >= RL.n) break;
      iv_push(&C, RL.v[pos++]);
      if (left > 0) --left;
    }
    if (ex) merge_once(&C, ex, out);
    else { out->n = 0; for (int64_t i = 0; i < C.n; ++i) iv_push(out, C.v[i]); }
  } else if (ex) {
    out->n = 0;
    for (int64_t i = 0; i < ex->n; ++i) iv_push(out, ex->v[i]);
  }
  free(blocks);
  free(M.v); free(I.v); free(R.v); free(IM.v); free(E.v); free(C.v); free(RL.v);
}

/* ---- public API ------------------------------------------------------------------------- */

void orc_close(orc* o) {
  if (!o) return;
  free(o->g); free(o->t); free(o->o); free(o->goff); free(o->toff); free(o->deg);
  free(o->off); free(o->dst); free(o->ts);
  free(o);
}

/* Opens <dir>/<base>.{graph,offsets,timestamps}; n = vertices (nodes of the properties). */
orc* orc_open(const char* dir, const char* base, int64_t n, int min_interval) {
  char path[4096];
  orc* o = (orc*)calloc(1, sizeof(orc));
  o->n = n;
  o->min_interval = min_interval;
  snprintf(path, sizeof path, "%s/%s.graph", dir, base);
  if (read_all(path, &o->g, &o->gn)) { orc_close(o); return NULL; }
  snprintf(path, sizeof path, "%s/%s.timestamps", dir, base);
  if (read_all(path, &o->t, &o->tn)) { orc_close(o); return NULL; }
  snprintf(path, sizeof path, "%s/%s.offsets", dir, base);
  if (read_all(path, &o->o, &o->on)) { orc_close(o); return NULL; }
  o->goff = (uint64_t*)malloc((size_t)(n + 1) * 8);
  o->toff = (uint64_t*)malloc((size_t)(n + 1) * 8);
  o->deg = (int32_t*)malloc((size_t)(n + 1) * 4);
  obits ob = {o->o, o->on * 8, 0};
  uint64_t p = 0, acc = 0;
  for (int64_t i = 0; i <= n; ++i) {
    acc += ob_gamma(&ob, &p);
    o->goff[i] = acc;
  }
  obits tb = {o->t, o->tn * 8, 0};
  uint64_t tp = 0;
  o->min_ts = (int64_t)ob_bits(&tb, &tp, 64);
  for (int64_t v = 0; v < n; ++v) {
    o->toff[v] = tp;
    o->deg[v] = (int32_t)outdeg_at(o, v);
    for (int32_t i = 0; i < o->deg[v]; ++i) ob_zeta(&tb, &tp, 2);
  }
  o->toff[n] = tp;
  if (ob.bad || tb.bad) o->err = 1;
  return o;
}

int orc_error(orc* o) { return o->err; }
int64_t orc_min_ts(orc* o) { return o->min_ts; }
int64_t orc_graph_offset(orc* o, int64_t v) { return (int64_t)o->goff[v]; }
int64_t orc_ts_offset(orc* o, int64_t v) { return (int64_t)o->toff[v]; }
int32_t orc_outdegree(orc* o, int64_t v) { return o->deg[v]; }
void orc_outdegrees(orc* o, int32_t* out) { memcpy(out, o->deg, (size_t)o->n * 4); }

/* Decodes v's list and timestamps into dst/ts (capacity cap); returns the outdegree. */
int64_t orc_neighbors(orc* o, int64_t v, int32_t* dst, int64_t* ts, int64_t cap) {
  ivec L = {0};
  decode_list(o, v, &L, 0);
  obits tb = {o->t, o->tn * 8, 0};
  uint64_t tp = o->toff[v];
  int64_t prev = o->min_ts;
  for (int64_t i = 0; i < L.n; ++i) {
    prev += orc_nat2int(ob_zeta(&tb, &tp, 2));
    if (i < cap) { dst[i] = L.v[i]; ts[i] = prev; }
  }
  if (tb.bad) o->err = 1;
  const int64_t k = L.n;
  free(L.v);
  return k;
}

/* Decodes every list into the oracle's CSR; returns m. */
int64_t orc_materialize(orc* o) {
  free(o->off); free(o->dst); free(o->ts);
  o->off = (int64_t*)malloc((size_t)(o->n + 1) * 8);
  o->off[0] = 0;
  for (int64_t v = 0; v < o->n; ++v) o->off[v + 1] = o->off[v] + o->deg[v];
  o->m = o->off[o->n];
  o->dst = (int32_t*)malloc((size_t)(o->m + 1) * 4);
  o->ts = (int64_t*)malloc((size_t)(o->m + 1) * 8);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : bad)
  for (int64_t v = 0; v < o->n; ++v) {
    const int64_t k = orc_neighbors(o, v, o->dst + o->off[v], o->ts + o->off[v], o->deg[v]);
    if (k != o->deg[v]) bad = 1;
  }
  if (bad) o->err = 1;
  return o->m;
}

void orc_csr(orc* o, int64_t* off, int32_t* dst, int64_t* ts) {
  memcpy(off, o->off, (size_t)(o->n + 1) * 8);
  memcpy(dst, o->dst, (size_t)o->m * 4);
  memcpy(ts, o->ts, (size_t)o->m * 8);
}

/* Neighbour-access checksum of a list: sum mod 2^64 over its edges of a mix of (vertex, edge
 * index, successor, timestamp) -- the engine's definition, additive so that it can be split. */
static uint64_t orc_edge_hash(uint32_t v, uint32_t i, int32_t y, int64_t t) {
  uint64_t z = (((uint64_t)v << 32) | i) * 0x9E3779B97F4A7C15ull;
  z ^= (uint64_t)(uint32_t)y * 0xC2B2AE3D27D4EB4Full;
  z ^= (uint64_t)t * 0x165667B19E3779F9ull;
  z ^= z >> 31;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 29;
  z *= 0x94D049BB133111EBull;
  return z ^ (z >> 32);
}

void orc_checksums(orc* o, int64_t begin, int64_t end, uint64_t* csum, uint8_t* small) {
  for (int64_t x = begin; x < end; ++x) {
    uint64_t h = 0;
    for (int64_t e = o->off[x]; e < o->off[x + 1]; ++e)
      h += orc_edge_hash((uint32_t)x, (uint32_t)(e - o->off[x]), o->dst[e], o->ts[e]);
    csum[x] = h;
    small[x] = o->deg[x] < 4;
  }
}

/* ---- workloads (engine result contracts, FP64) -------------------------------------------- */

static void atomic_add_f64(double* p, double v) {
#pragma omp atomic
  *p += v;
}

typedef struct {
  int32_t max_label, max_vertex, active;
} orc_cfg;

/* Edge filter shared by BFS/CC/PR/HITS/GC: first in-window occurrence of equal consecutive ids. */
#define FOR_DEDUP_EDGES(o, x, lo, hi, Y, T, BODY)                          \
  do {                                                                     \
    int32_t prev_y_ = -1;                                                  \
    for (int64_t e_ = (o)->off[x]; e_ < (o)->off[(x) + 1]; ++e_) {        \
      const int64_t T = (o)->ts[e_];                                       \
      if (T < (lo) || T >= (hi)) continue;                                 \
      const int32_t Y = (o)->dst[e_];                                      \
      if (Y == prev_y_) continue;                                          \
      prev_y_ = Y;                                                         \
      BODY                                                                 \
    }                                                                      \
  } while (0)

/* Binary heap of (key, vertex) for the lexicographic (arrival, hops) fixpoint. */
typedef struct { uint64_t key; int32_t v; } hent;
typedef struct { hent* a; int64_t n, cap; } heap;
static void hpush(heap* h, uint64_t key, int32_t v) {
  if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->a = (hent*)realloc(h->a, (size_t)h->cap * sizeof(hent)); }
  int64_t i = h->n++;
  while (i > 0) {
    const int64_t p = (i - 1) / 2;
    if (h->a[p].key <= key) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i].key = key; h->a[i].v = v;
}
static hent hpop(heap* h) {
  hent top = h->a[0], last = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t c = 2 * i + 1;
    if (c >= h->n) break;
    if (c + 1 < h->n && h->a[c + 1].key < h->a[c].key) ++c;
    if (last.key <= h->a[c].key) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n) h->a[i] = last;
  return top;
}

/* Source of a vertex's list for the workloads below: the materialised CSR (s == NULL), or the
 * compressed streams decoded at each visit (streaming mode, used by the timed CPU baseline; s
 * counts the edges decoded).  succ_only: timestamps are not decoded (left at 0). */
typedef struct {
  ivec L;
  int64_t* ts;
  int64_t cap;
  int64_t edges;
  int succ_only;
} sctx;

static int64_t stream_list(orc* o, int64_t x, ivec* L, int64_t** tsbuf, int64_t* tscap);

static int64_t view_list(orc* o, int64_t x, sctx* s, const int32_t** dst, const int64_t** ts) {
  if (!s) {
    *dst = o->dst + o->off[x];
    *ts = o->ts + o->off[x];
    return o->off[x + 1] - o->off[x];
  }
  int64_t k;
  if (s->succ_only) {
    decode_list(o, x, &s->L, 0);
    k = s->L.n;
    if (k > s->cap) { s->cap = 2 * k; s->ts = (int64_t*)realloc(s->ts, (size_t)s->cap * 8); }
    if (k) memset(s->ts, 0, (size_t)k * 8);
  } else {
    k = stream_list(o, x, &s->L, &s->ts, &s->cap);
  }
  s->edges += k;
  *dst = s->L.v;
  *ts = s->ts;
  return k;
}

static void sctx_free(sctx* s) { free(s->L.v); free(s->ts); }

/* FOR_DEDUP_EDGES over a list source. */
#define FOR_DEDUP_VIEW(o, s, x, lo, hi, Y, T, BODY)                        \
  do {                                                                     \
    const int32_t* vd_;                                                    \
    const int64_t* vt_;                                                    \
    const int64_t vk_ = view_list((o), (x), (s), &vd_, &vt_);              \
    int32_t prev_y_ = -1;                                                  \
    for (int64_t e_ = 0; e_ < vk_; ++e_) {                                 \
      const int64_t T = vt_[e_];                                           \
      if (T < (lo) || T >= (hi)) continue;                                 \
      const int32_t Y = vd_[e_];                                           \
      if (Y == prev_y_) continue;                                          \
      prev_y_ = Y;                                                         \
      BODY                                                                 \
    }                                                                      \
  } while (0)

/* Earliest arrival by Dijkstra on arrival times (the relaxation fixpoint is unique); returns the
 * number of vertices other than src that were reached.  key[] holds arrival << 32. */
static int64_t bfs_core(orc* o, const orc_cfg* c, int32_t src, int64_t lo, int64_t hi, uint64_t* key, sctx* sc) {
  heap h = {0};
  const uint64_t start = (uint64_t)(lo > 0 ? lo : 0) << 32;
  key[src] = start;
  hpush(&h, start, src);
  int64_t touched = 0;
  while (h.n) {
    const hent top = hpop(&h);
    const int32_t x = top.v;
    if (top.key != key[x]) continue;
    if (x < c->active || x > c->max_label || x >= o->n) continue;
    const uint64_t ax = top.key >> 32;
    FOR_DEDUP_VIEW(o, sc, x, lo, hi, y, t, {
      if (y < c->active || y >= c->max_vertex) continue;
      if ((int64_t)ax > t || t >= 0xFFFFFFFFll) continue;
      const uint64_t nv = (uint64_t)t << 32;
      if (nv < key[y]) {
        if (key[y] == ~0ull) ++touched;
        key[y] = nv;
        hpush(&h, nv, y);
      }
    });
  }
  free(h.a);
  return touched;
}

/* Hop counts: breadth-first over tight edges (arrival(x) <= t == arrival(y)) from src. */
static void bfs_hops(orc* o, const orc_cfg* c, int32_t src, int64_t lo, int64_t hi, const uint64_t* key,
                     int32_t* hops, sctx* sc) {
  int32_t* q = (int32_t*)malloc((size_t)c->max_vertex * 4 + 4);
  int64_t qh = 0, qt = 0;
  hops[src] = 0;
  q[qt++] = src;
  while (qh < qt) {
    const int32_t x = q[qh++];
    if (x < c->active || x > c->max_label || x >= o->n) continue;
    const int64_t ax = (int64_t)(key[x] >> 32);
    FOR_DEDUP_VIEW(o, sc, x, lo, hi, y, t, {
      if (y < c->active || y >= c->max_vertex) continue;
      if (ax > t || t >= 0xFFFFFFFFll) continue;
      if ((int64_t)(key[y] >> 32) != t || hops[y] != ORC_INF32) continue;
      hops[y] = hops[x] + 1;
      q[qt++] = y;
    });
  }
  free(q);
}

void orc_bfs(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t src, int64_t lo, int64_t hi,
             int32_t* arr, int32_t* hops) {
  orc_cfg c = {max_label, max_vertex, active};
  uint64_t* key = (uint64_t*)malloc((size_t)max_vertex * 8);
  for (int32_t i = 0; i < max_vertex; ++i) { key[i] = ~0ull; hops[i] = ORC_INF32; }
  bfs_core(o, &c, src, lo, hi, key, NULL);
  bfs_hops(o, &c, src, lo, hi, key, hops, NULL);
  for (int32_t i = 0; i < max_vertex; ++i) {
    const int inf = (key[i] >> 32) == 0xFFFFFFFFull;
    arr[i] = inf ? ORC_INF32 : (int32_t)(key[i] >> 32);
    if (inf) hops[i] = ORC_INF32;
  }
  free(key);
}

static int32_t cc_core(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t begin, int64_t lo,
                       int64_t hi, int32_t early_exit, int32_t* label, sctx* sc) {
  orc_cfg c = {max_label, max_vertex, active};
  uint64_t* key = (uint64_t*)malloc((size_t)max_vertex * 8);
  uint8_t* reached = (uint8_t*)calloc((size_t)max_vertex, 1);
  for (int32_t i = 0; i < max_vertex; ++i) { key[i] = ~0ull; label[i] = -1; }
  const int32_t limit = (int32_t)(0.8 * max_label);
  const int32_t end = max_label < max_vertex ? max_label : max_vertex;
  int64_t total = 0;
  int small = 0;
  int32_t comp = 0;
  for (int32_t v = begin < 0 ? 0 : begin; v < end; ++v) {
    if (early_exit && total > limit) break;
    if (reached[v] || v >= o->n || o->deg[v] <= 9) continue;
    const int64_t t = bfs_core(o, &c, v, lo, hi, key, sc);
    for (int32_t y = 0; y < max_vertex; ++y)
      if (key[y] != ~0ull) { label[y] = comp; reached[y] = 1; key[y] = ~0ull; }
    ++comp;
    total += t + 1;
    if (t + 1 < 5) ++small; else small = 0;
    if (early_exit && small > 50) break;
  }
  free(key);
  free(reached);
  return comp;
}

int32_t orc_cc(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t begin, int64_t lo, int64_t hi,
               int32_t early_exit, int32_t* label) {
  return cc_core(o, max_label, max_vertex, active, begin, lo, hi, early_exit, label, NULL);
}

/* PageRank with the engine's contract (reference pagerank.cu semantics, reset before scatter). */
void orc_pagerank(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t iters, double d,
                  double alpha, int64_t lo, int64_t hi, double* rank) {
  double* nw = (double*)malloc((size_t)max_vertex * 8);
  double* invdeg = (double*)malloc((size_t)max_vertex * 8);
  const int windowed = !(lo <= 0 && hi == INT64_MAX);
  for (int32_t x = 0; x < max_vertex; ++x) {
    rank[x] = 1.0 / max_vertex;
    int64_t cnt = 0;
    if (x < o->n) {
      if (windowed) { for (int64_t e = o->off[x]; e < o->off[x + 1]; ++e) cnt += o->ts[e] >= lo && o->ts[e] < hi; }
      else cnt = o->deg[x];
    }
    invdeg[x] = cnt ? 1.0 / (double)cnt : 0.0;
  }
  const double base = (1.0 - d) / max_label;
  for (int it = 0; it < iters; ++it) {
    for (int32_t u = 0; u < max_vertex; ++u) nw[u] = base;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t x = active; x < max_label; ++x) {
      if (x >= o->n || invdeg[x] == 0.0) continue;
      const double c0 = d * rank[x] * invdeg[x];
      FOR_DEDUP_EDGES(o, x, lo, hi, y, t, {
        if (y < active || y >= max_vertex) continue;
        const double contrib = c0 * (1.0 - exp(-alpha * (double)t));
        atomic_add_f64(&nw[y], contrib);
      });
    }
    double s = 0;
    for (int32_t u = 0; u < max_vertex; ++u) s += nw[u];
    for (int32_t u = 0; u < max_vertex; ++u) rank[u] = nw[u] / s;
  }
  free(nw);
  free(invdeg);
}

/* HITS; java=0 reference GPU semantics (no reset), java=1 BaselineRunner semantics.  stream:
 * lists decoded at each visit (successors only when the window holds every timestamp, as the
 * engine does); returns the edges decoded in streaming mode. */
static int64_t hits_core(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t iters, int32_t java,
                         int64_t lo, int64_t hi, double* hub, double* auth, int stream) {
  const int succ_only = lo <= o->min_ts && hi == INT64_MAX;  /* every timestamp is >= the header */
  int64_t edges = 0;
  for (int32_t u = 0; u < max_vertex; ++u) hub[u] = auth[u] = 1.0;
  for (int it = 0; it < iters; ++it) {
    if (java) for (int32_t u = 0; u < max_vertex; ++u) hub[u] = 0.0;
#pragma omp parallel reduction(+ : edges)
    {
      sctx tsc = {0};
      tsc.succ_only = succ_only;
      sctx* sc = stream ? &tsc : NULL;
#pragma omp for schedule(dynamic, 1024)
      for (int32_t x = active; x < max_label; ++x) {
        if (x >= o->n) continue;
        double acc = 0;
        FOR_DEDUP_VIEW(o, sc, x, lo, hi, y, t, {
          (void)t;
          if (y < active || y >= max_vertex) continue;
          acc += auth[y];
        });
        hub[x] += acc;
      }
      edges += tsc.edges;
      sctx_free(&tsc);
    }
    double s = 0;
    for (int32_t u = 0; u < max_vertex; ++u) s += hub[u] * hub[u];
    s = sqrt(s);
    if (s > 0) for (int32_t u = 0; u < max_vertex; ++u) hub[u] /= s;
    if (java) for (int32_t u = 0; u < max_vertex; ++u) auth[u] = 0.0;
#pragma omp parallel reduction(+ : edges)
    {
      sctx tsc = {0};
      tsc.succ_only = succ_only;
      sctx* sc = stream ? &tsc : NULL;
#pragma omp for schedule(dynamic, 1024)
      for (int32_t x = active; x < max_label; ++x) {
        if (x >= o->n) continue;
        const double hx = hub[x];
        FOR_DEDUP_VIEW(o, sc, x, lo, hi, y, t, {
          (void)t;
          if (y < active || y >= max_vertex) continue;
          atomic_add_f64(&auth[y], hx);
        });
      }
      edges += tsc.edges;
      sctx_free(&tsc);
    }
    s = 0;
    for (int32_t u = 0; u < max_vertex; ++u) s += auth[u] * auth[u];
    s = sqrt(s);
    if (s > 0) for (int32_t u = 0; u < max_vertex; ++u) auth[u] /= s;
  }
  return edges;
}

void orc_hits(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t iters, int32_t java, int64_t lo,
              int64_t hi, double* hub, double* auth) {
  hits_core(o, max_label, max_vertex, active, iters, java, lo, hi, hub, auth, 0);
}

/* Degree centrality, Java semantics (BaselineRunner.java:316-346). */
static int64_t degree_core(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int64_t s, int64_t e,
                           int32_t* deg, int64_t* avg, int stream) {
  const int32_t lim = max_label + 1 < max_vertex ? max_label + 1 : max_vertex;
  int64_t edges = 0;
#pragma omp parallel reduction(+ : edges)
  {
    sctx tsc = {0};
    sctx* sc = stream ? &tsc : NULL;
#pragma omp for schedule(dynamic, 1024)
    for (int32_t x = 0; x < max_vertex; ++x) {
      int32_t d = 0;
      int64_t mean = 0;
      if (x >= active && x <= max_label && x < o->n) {
        const int32_t* vd;
        const int64_t* vt;
        const int64_t k = view_list(o, x, sc, &vd, &vt);
        for (int64_t i = 0; i < k; ++i) {
          const int32_t y = vd[i];
          const int64_t t = vt[i];
          if (y < active || y >= lim) continue;
          if ((s == 0 && e == 0) || (s <= t && e >= t)) {
            ++d;
            mean += (t - mean) / d;
          }
        }
        if (s != e) d = (int32_t)(0.85 * d + 0.15 * d * (double)(mean - s) / (double)(e - s) + 1);
      }
      deg[x] = d;
      avg[x] = mean;
    }
    edges += tsc.edges;
    sctx_free(&tsc);
  }
  return edges;
}

void orc_degree(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int64_t s, int64_t e, int32_t* deg,
                int64_t* avg) {
  degree_core(o, max_label, max_vertex, active, s, e, deg, avg, 0);
}

/* Jones-Plassmann rounds with given priorities; returns rounds executed.  A round decides every
 * vertex of the worklist from the colours at its start (snap), so the vertices of a round are
 * independent and run in parallel; the worklist keeps its order. */
static int32_t color_core(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, const uint32_t* prio,
                          int32_t java_isolated, uint32_t* color, int stream, int64_t* edges_out) {
  int32_t* wl = (int32_t*)malloc((size_t)max_vertex * 4);
  int32_t* nwl = (int32_t*)malloc((size_t)max_vertex * 4);
  uint8_t* keep = (uint8_t*)malloc((size_t)max_vertex + 1);
  uint32_t* snap = (uint32_t*)malloc((size_t)max_vertex * 4);
  int64_t wn = max_vertex, edges = 0;
  for (int32_t i = 0; i < max_vertex; ++i) { wl[i] = i; color[i] = 0xFFFFFFFFu; }
  int32_t round = 0;
  while (wn && round < 512) {
    memcpy(snap, color, (size_t)max_vertex * 4);
#pragma omp parallel reduction(+ : edges)
    {
      sctx tsc = {0};
      tsc.succ_only = 1;
      sctx* sc = stream ? &tsc : NULL;
#pragma omp for schedule(dynamic, 256)
      for (int64_t i = 0; i < wn; ++i) {
        const int32_t x = wl[i];
        keep[i] = 0;
        if (x < active || snap[x] != 0xFFFFFFFFu || x > max_label) continue;
        if (x >= o->n || o->deg[x] == 0) {
          if (java_isolated) color[x] = (uint32_t)round;
          continue;
        }
        int larger = 0;
        FOR_DEDUP_VIEW(o, sc, x, INT64_MIN, INT64_MAX, y, t, {
          (void)t;
          if (larger) break;
          if (y < active || y >= max_vertex) continue;
          if ((prio[y] > prio[x] || (prio[y] == prio[x] && y < x)) && snap[y] >= (uint32_t)round) larger = 1;
        });
        if (larger) keep[i] = 1;
        else color[x] = (uint32_t)round;
      }
      edges += tsc.edges;
      sctx_free(&tsc);
    }
    int64_t nn = 0;
    for (int64_t i = 0; i < wn; ++i)
      if (keep[i]) nwl[nn++] = wl[i];
    int32_t* tmp = wl; wl = nwl; nwl = tmp;
    wn = nn;
    ++round;
  }
  free(wl); free(nwl); free(keep); free(snap);
  if (edges_out) *edges_out = edges;
  return round;
}

int32_t orc_color(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, const uint32_t* prio,
                  int32_t java_isolated, uint32_t* color) {
  return color_core(o, max_label, max_vertex, active, prio, java_isolated, color, 0, NULL);
}

/* Fewest-hop temporal paths: hops[v] = the fewest edges on a time-respecting path from src to v
 * within [lo, hi) (edge (x->y, t) usable when arr(x) <= t, BFS's edge rule), arr[v] = the earliest
 * arrival.  Level-synchronous relaxation: A_k[v] = min(A_{k-1}[v], min over usable edges (x->v, t)
 * with A_{k-1}[x] <= t of t), expanding only the vertices whose A dropped at level k-1; hops[v] is the
 * first k with A_k[v] finite. */
void orc_shortest(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t src, int64_t lo, int64_t hi,
                  int32_t* arr, int32_t* hops) {
  orc_cfg c = {max_label, max_vertex, active};
  (void)c;
  int64_t* prev = (int64_t*)malloc((size_t)max_vertex * 8);
  int64_t* next = (int64_t*)malloc((size_t)max_vertex * 8);
  int32_t* fr = (int32_t*)malloc((size_t)max_vertex * 4);
  int32_t* nf = (int32_t*)malloc((size_t)max_vertex * 4);
  uint8_t* mark = (uint8_t*)calloc((size_t)max_vertex, 1);
  const int64_t INF = INT64_MAX;
  for (int32_t i = 0; i < max_vertex; ++i) { prev[i] = next[i] = INF; hops[i] = ORC_INF32; }
  prev[src] = next[src] = lo > 0 ? lo : 0;
  hops[src] = 0;
  int64_t fn = 0;
  fr[fn++] = src;
  for (int32_t level = 1; fn > 0 && level <= max_vertex; ++level) {
    int64_t nn = 0;
    for (int64_t i = 0; i < fn; ++i) {
      const int32_t x = fr[i];
      if (x < active || x > max_label || x >= o->n) continue;
      const int64_t ax = prev[x];
      FOR_DEDUP_EDGES(o, x, lo, hi, y, t, {
        if (y < active || y >= max_vertex) continue;
        if (ax > t || t >= 0xFFFFFFFFll) continue;
        if (t < next[y]) {
          next[y] = t;
          if (!mark[y]) { mark[y] = 1; nf[nn++] = y; }
        }
      });
    }
    for (int64_t i = 0; i < nn; ++i) {
      const int32_t y = nf[i];
      mark[y] = 0;
      if (prev[y] == INF) hops[y] = level;
      prev[y] = next[y];
    }
    int32_t* tmp = fr; fr = nf; nf = tmp;
    fn = nn;
  }
  for (int32_t i = 0; i < max_vertex; ++i) arr[i] = prev[i] == INF ? ORC_INF32 : (int32_t)prev[i];
  free(prev); free(next); free(fr); free(nf); free(mark);
}

/* java.util.Random(seed).nextInt(256) sequence (documented JDK LCG). */
void orc_java_random256(int64_t seed, int32_t n, uint32_t* out) {
  uint64_t s = ((uint64_t)seed ^ 0x5DEECE66Dull) & ((1ull << 48) - 1);
  for (int32_t i = 0; i < n; ++i) {
    s = (s * 0x5DEECE66Dull + 0xBull) & ((1ull << 48) - 1);
    const int32_t bits = (int32_t)(s >> 17);
    out[i] = (uint32_t)(((int64_t)256 * bits) >> 31);
  }
}

/* ---- streaming workloads for the timed CPU baseline ---------------------------------------
 * These decode every visited list from the compressed streams at each visit, like the Java
 * runner's SuccessorIterator, instead of reading the materialised CSR. */

static int64_t stream_list(orc* o, int64_t x, ivec* L, int64_t** tsbuf, int64_t* tscap) {
  decode_list(o, x, L, 0);
  if (L->n > *tscap) { *tscap = L->n * 2; *tsbuf = (int64_t*)realloc(*tsbuf, (size_t)*tscap * 8); }
  obits tb = {o->t, o->tn * 8, 0};
  uint64_t tp = o->toff[x];
  int64_t prev = o->min_ts;
  for (int64_t i = 0; i < L->n; ++i) {
    prev += orc_nat2int(ob_zeta(&tb, &tp, 2));
    (*tsbuf)[i] = prev;
  }
  return L->n;
}

/* One temporal PageRank iteration sweep decoded on the fly; returns edges decoded. */
int64_t orc_stream_pagerank(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t iters, double d,
                            double alpha, double* rank, int32_t threads) {
  double* nw = (double*)malloc((size_t)max_vertex * 8);
  for (int32_t x = 0; x < max_vertex; ++x) rank[x] = 1.0 / max_vertex;
  const double base = (1.0 - d) / max_label;
  int64_t edges = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  for (int it = 0; it < iters; ++it) {
    for (int32_t u = 0; u < max_vertex; ++u) nw[u] = base;
#pragma omp parallel reduction(+ : edges)
    {
      ivec L = {0};
      int64_t* tsb = NULL;
      int64_t cap = 0;
#pragma omp for schedule(dynamic, 256)
      for (int32_t x = active; x < max_label; ++x) {
        if (x >= o->n || o->deg[x] == 0) continue;
        const int64_t k = stream_list(o, x, &L, &tsb, &cap);
        edges += k;
        const double c0 = d * rank[x] / (double)o->deg[x];
        int32_t prev_y = -1;
        for (int64_t i = 0; i < k; ++i) {
          const int32_t y = L.v[i];
          if (y == prev_y) continue;
          prev_y = y;
          if (y < active || y >= max_vertex) continue;
          const double contrib = c0 * (1.0 - exp(-alpha * (double)tsb[i]));
#pragma omp atomic
          nw[y] += contrib;
        }
      }
      free(L.v);
      free(tsb);
    }
    double s = 0;
    for (int32_t u = 0; u < max_vertex; ++u) s += nw[u];
    for (int32_t u = 0; u < max_vertex; ++u) rank[u] = nw[u] / s;
  }
  free(nw);
  return edges;
}

/* Full decode sweep of [begin, end) decoded on the fly (neighbour access); returns edges. */
int64_t orc_stream_decode(orc* o, int64_t begin, int64_t end, uint64_t* csum, int32_t threads) {
  int64_t edges = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel reduction(+ : edges)
  {
    ivec L = {0};
    int64_t* tsb = NULL;
    int64_t cap = 0;
#pragma omp for schedule(dynamic, 256)
    for (int64_t x = begin; x < end; ++x) {
      const int64_t k = stream_list(o, x, &L, &tsb, &cap);
      uint64_t h = 0;
      for (int64_t i = 0; i < k; ++i) h += orc_edge_hash((uint32_t)x, (uint32_t)i, L.v[i], tsb[i]);
      if (csum) csum[x] = h;
      edges += k;
    }
    free(L.v);
    free(tsb);
  }
  return edges;
}

/* The remaining workloads of the benchmark step, decoded on the fly (streaming mode of the
 * functions above); each returns the edges it decoded.  threads > 0 sets the OpenMP thread count
 * (BFS and CC are sequential searches and use one thread). */
static void set_threads(int32_t threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
}

int64_t orc_stream_bfs(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t src, int64_t lo,
                       int64_t hi, int32_t* arr, int32_t* hops) {
  orc_cfg c = {max_label, max_vertex, active};
  sctx sc = {0};
  uint64_t* key = (uint64_t*)malloc((size_t)max_vertex * 8);
  for (int32_t i = 0; i < max_vertex; ++i) { key[i] = ~0ull; hops[i] = ORC_INF32; }
  bfs_core(o, &c, src, lo, hi, key, &sc);
  bfs_hops(o, &c, src, lo, hi, key, hops, &sc);
  for (int32_t i = 0; i < max_vertex; ++i) {
    const int inf = (key[i] >> 32) == 0xFFFFFFFFull;
    arr[i] = inf ? ORC_INF32 : (int32_t)(key[i] >> 32);
    if (inf) hops[i] = ORC_INF32;
  }
  free(key);
  sctx_free(&sc);
  return sc.edges;
}

int64_t orc_stream_cc(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t begin, int64_t lo,
                      int64_t hi, int32_t early_exit, int32_t* label, int32_t* comps) {
  sctx sc = {0};
  *comps = cc_core(o, max_label, max_vertex, active, begin, lo, hi, early_exit, label, &sc);
  sctx_free(&sc);
  return sc.edges;
}

int64_t orc_stream_hits(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int32_t iters, int32_t java,
                        double* hub, double* auth, int32_t threads) {
  set_threads(threads);
  return hits_core(o, max_label, max_vertex, active, iters, java, 0, INT64_MAX, hub, auth, 1);
}

int64_t orc_stream_degree(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, int64_t s, int64_t e,
                          int32_t* deg, int64_t* avg, int32_t threads) {
  set_threads(threads);
  return degree_core(o, max_label, max_vertex, active, s, e, deg, avg, 1);
}

int64_t orc_stream_color(orc* o, int32_t max_label, int32_t max_vertex, int32_t active, const uint32_t* prio,
                         int32_t java_isolated, uint32_t* color, int32_t* rounds, int32_t threads) {
  set_threads(threads);
  int64_t edges = 0;
  *rounds = color_core(o, max_label, max_vertex, active, prio, java_isolated, color, 1, &edges);
  return edges;
}

/* Reads n codes of one kind from a byte buffer: 0 gamma, 1 zeta_k, 2 unary, 3 64-bit fixed. */
int64_t orc_read_codes(const uint8_t* bytes, int64_t nbytes, int32_t kind, int32_t k, uint64_t* out, int64_t n) {
  obits b = {bytes, (uint64_t)nbytes * 8, 0};
  uint64_t p = 0;
  for (int64_t i = 0; i < n; ++i) {
    switch (kind) {
      case 0: out[i] = ob_gamma(&b, &p); break;
      case 1: out[i] = ob_zeta(&b, &p, k); break;
      case 2: out[i] = ob_unary(&b, &p); break;
      default: out[i] = ob_bits(&b, &p, 64); break;
    }
  }
  return b.bad ? -1 : (int64_t)p;
}

/* Value i of an Elias-Fano index in the GPU layout, following the reference reader
 * (gpu_cuda/shared/bfs.cu:543-565): l low bits MSB-first at bit i*l, high part = position of
 * the i-th one of the LSB-first upper bits minus i.  Independent of the engine's select samples. */
uint64_t orc_ef_get(const uint8_t* lower, const uint8_t* upper, int64_t upper_bytes, int32_t l, int64_t i) {
  uint64_t low = 0;
  for (int32_t j = 0; j < l; ++j) {
    const uint64_t pos = (uint64_t)i * (uint64_t)l + (uint64_t)j;
    low = (low << 1) | (uint64_t)((lower[pos >> 3] >> (7 - (pos & 7))) & 1);
  }
  int64_t seen = 0;
  for (int64_t pos = 0; pos < upper_bytes * 8; ++pos) {
    if ((upper[pos >> 3] >> (pos & 7)) & 1) {
      if (seen == i) return ((uint64_t)(pos - i) << l) | low;
      ++seen;
    }
  }
  return ~0ull;
}

int32_t orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
