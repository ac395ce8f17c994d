/*
 * bvh_oracle.c -- CPU restatement of the reference shared-bvh path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: tests, the smoke check and bench.py's cpu_baseline leg may call it,
 * the product library never does.
 *
 * It restates, in plain C with IEEE double arithmetic (the JS "number" the
 * reference computes in) and no FMA contraction (-ffp-contract=off):
 *
 *   orc_build_array_bvh    packages/shared-bvh/src/buildArrayBvh.ts:342-780
 *                          (binned SAH, recursive `build` :511-706,
 *                          `surfaceArea` :223-231, defaults :72-77,
 *                          node store :751-765)
 *   orc_collapse_wide      packages/shared-bvh/src/compressedWideBvh.ts:248-418
 *                          (`collectWideChildren` :215-242, `quantizeBound`
 *                          :197-204, stack proof :60-92)
 *   orc_first_hit          packages/shared-bvh/src/compressedWideBvh.ts:754-860
 *                          (`intersectTriangle` :551-614, `intersectAabb`
 *                          :616-645, `dequantizeBound` :206-213)
 *   orc_watertight_f32     packages/shared-bvh/src/opticalWatertightTriangle.ts:98-220
 *                          (every operation rounded to binary32, the
 *                          Math.fround mirror)
 *
 * plus a near-first traversal of the same wide tree that only counts node
 * visits and triangle tests (the algorithmic-bytes model of the bench).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>
#include <unistd.h>

#define ORC_LEAF_FLAG 0xFFFF0000u
#define ORC_WIDE 8
#define ORC_STACK_CAPACITY 64 /* CWBVH_TRAVERSAL_STACK_DEPTH, strides.ts:111 */

/* ------------------------------------------------------------------ */
/* error reporting                                                     */
/* ------------------------------------------------------------------ */
static char g_err[512];
const char* orc_last_error(void) { return g_err; }
static int fail(const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return -1;
}

/* ------------------------------------------------------------------ */
/* tiny pthread parallel-for over [0, n) in chunks                     */
/* ------------------------------------------------------------------ */
typedef void (*orc_range_fn)(void* ctx, long begin, long end, int worker);
typedef struct {
  orc_range_fn fn;
  void* ctx;
  long n, chunk;
  long next;
  pthread_mutex_t mu;
  int worker;
} pfor_t;
typedef struct { pfor_t* p; int id; } pfor_arg_t;

static void* pfor_worker(void* a) {
  pfor_arg_t* arg = (pfor_arg_t*)a;
  pfor_t* p = arg->p;
  for (;;) {
    pthread_mutex_lock(&p->mu);
    long b = p->next;
    p->next += p->chunk;
    pthread_mutex_unlock(&p->mu);
    if (b >= p->n) break;
    long e = b + p->chunk < p->n ? b + p->chunk : p->n;
    p->fn(p->ctx, b, e, arg->id);
  }
  return NULL;
}

int orc_hw_threads(void) {
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

static void parallel_for(long n, long chunk, int nthreads, orc_range_fn fn, void* ctx) {
  if (nthreads <= 0) nthreads = orc_hw_threads();
  if (nthreads > 256) nthreads = 256;
  pfor_t p;
  p.fn = fn; p.ctx = ctx; p.n = n; p.chunk = chunk; p.next = 0;
  pthread_mutex_init(&p.mu, NULL);
  if (nthreads == 1) {
    pfor_arg_t a = {&p, 0};
    pfor_worker(&a);
  } else {
    pthread_t th[256];
    pfor_arg_t args[256];
    for (int i = 0; i < nthreads; ++i) {
      args[i].p = &p; args[i].id = i;
      pthread_create(&th[i], NULL, pfor_worker, &args[i]);
    }
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
  }
  pthread_mutex_destroy(&p.mu);
}

/* ------------------------------------------------------------------ */
/* binary SAH build (buildArrayBvh.ts)                                 */
/* ------------------------------------------------------------------ */
typedef struct {
  uint32_t tri;
  double cen[3], mn[3], mx[3];
} rec_t;

typedef struct {
  double mn[3], mx[3];
  uint32_t w6, w7;
} bnode_t;

typedef struct {
  const rec_t* recs;
  bnode_t* nodes;
  size_t n_nodes, cap_nodes;
  uint32_t* ordered;
  size_t n_ordered;
  int max_leaf, nbins, max_depth;
  int err;
  /* per-axis bins and sweeps (Float32Array / Int32Array in the reference) */
  double bmn[256][3], bmx[256][3];
  int bcnt[256];
  float pmn[3][256], pmx[3][256], smn[3][256], smx[3][256];
  int pc[256], sc[256];
} bstate_t;

/* surfaceArea, buildArrayBvh.ts:223-231 (half area, extents clamped at 0). */
static double sa_half(double mnx, double mny, double mnz, double mxx, double mxy, double mxz) {
  double dx = mxx - mnx, dy = mxy - mny, dz = mxz - mnz;
  if (!(dx > 0)) dx = 0; /* Math.max(0, x) */
  if (!(dy > 0)) dy = 0;
  if (!(dz > 0)) dz = 0;
  return dx * dy + dy * dz + dz * dx;
}

/* Math.min / Math.max of two numbers: NaN propagates and -0 < +0. */
static double jsmin(double a, double b) {
  if (isnan(a) || isnan(b)) return NAN;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
static double jsmax(double a, double b) {
  if (isnan(a) || isnan(b)) return NAN;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

static size_t push_node(bstate_t* s) {
  if (s->n_nodes == s->cap_nodes) {
    s->cap_nodes = s->cap_nodes ? s->cap_nodes * 2 : 1024;
    s->nodes = (bnode_t*)realloc(s->nodes, s->cap_nodes * sizeof(bnode_t));
  }
  return s->n_nodes++;
}

static const rec_t* g_sort_recs;
static int g_sort_axis;
static int cmp_fallback(const void* pa, const void* pb) {
  const rec_t* a = &g_sort_recs[*(const uint32_t*)pa];
  const rec_t* b = &g_sort_recs[*(const uint32_t*)pb];
  double d = a->cen[g_sort_axis] - b->cen[g_sort_axis];
  if (d != 0) return d < 0 ? -1 : 1;
  return a->tri < b->tri ? -1 : (a->tri > b->tri ? 1 : 0);
}

/* `build`, buildArrayBvh.ts:511-706.  `subset` holds record indices. */
static size_t build_rec(bstate_t* s, uint32_t* subset, size_t count, int depth) {
  size_t ni = push_node(s);
  bnode_t nd;
  for (int k = 0; k < 3; ++k) { nd.mn[k] = INFINITY; nd.mx[k] = -INFINITY; }
  for (size_t i = 0; i < count; ++i) {
    const rec_t* r = &s->recs[subset[i]];
    for (int k = 0; k < 3; ++k) {
      nd.mn[k] = jsmin(nd.mn[k], r->mn[k]);
      nd.mx[k] = jsmax(nd.mx[k], r->mx[k]);
    }
  }
  nd.w6 = 0; nd.w7 = 0;
  s->nodes[ni] = nd;

  if ((int)count <= s->max_leaf) { /* makeLeaf :463-480 */
    s->nodes[ni].w6 = (uint32_t)s->n_ordered;
    s->nodes[ni].w7 = ORC_LEAF_FLAG | (uint32_t)count;
    for (size_t i = 0; i < count; ++i) s->ordered[s->n_ordered++] = s->recs[subset[i]].tri;
    return ni;
  }
  if (depth >= s->max_depth) { s->err = 1; fail("maxDepth prevents enforcing maxLeafTriangles"); return ni; }

  double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = 0; i < count; ++i) {
    const rec_t* r = &s->recs[subset[i]];
    for (int k = 0; k < 3; ++k) { cmn[k] = jsmin(cmn[k], r->cen[k]); cmx[k] = jsmax(cmx[k], r->cen[k]); }
  }
  double parent_sa = sa_half(nd.mn[0], nd.mn[1], nd.mn[2], nd.mx[0], nd.mx[1], nd.mx[2]);
  double leaf_cost = (double)count;
  double best_cost = INFINITY;
  int best_axis = 0, best_split = 0;
  const int K = s->nbins;

  for (int axis = 0; axis < 3; ++axis) {
    double span = cmx[axis] - cmn[axis];
    if (span <= 1e-9) continue;
    for (int b = 0; b < K; ++b) {
      for (int k = 0; k < 3; ++k) { s->bmn[b][k] = INFINITY; s->bmx[b][k] = -INFINITY; }
      s->bcnt[b] = 0;
    }
    for (size_t i = 0; i < count; ++i) {
      const rec_t* r = &s->recs[subset[i]];
      double t = (r->cen[axis] - cmn[axis]) / span;
      double fb = floor(t * K);
      int b = fb < (double)(K - 1) ? (int)fb : K - 1;
      for (int k = 0; k < 3; ++k) {
        s->bmn[b][k] = jsmin(s->bmn[b][k], r->mn[k]);
        s->bmx[b][k] = jsmax(s->bmx[b][k], r->mx[k]);
      }
      s->bcnt[b] += 1;
    }
    { /* prefix sweep :588-605 */
      double a0 = INFINITY, a1 = INFINITY, a2 = INFINITY, b0 = -INFINITY, b1 = -INFINITY, b2 = -INFINITY;
      int c = 0;
      for (int i = 0; i < K; ++i) {
        a0 = jsmin(a0, s->bmn[i][0]); a1 = jsmin(a1, s->bmn[i][1]); a2 = jsmin(a2, s->bmn[i][2]);
        b0 = jsmax(b0, s->bmx[i][0]); b1 = jsmax(b1, s->bmx[i][1]); b2 = jsmax(b2, s->bmx[i][2]);
        c += s->bcnt[i];
        s->pmn[0][i] = (float)a0; s->pmn[1][i] = (float)a1; s->pmn[2][i] = (float)a2;
        s->pmx[0][i] = (float)b0; s->pmx[1][i] = (float)b1; s->pmx[2][i] = (float)b2;
        s->pc[i] = c;
      }
    }
    { /* suffix sweep :608-625 */
      double a0 = INFINITY, a1 = INFINITY, a2 = INFINITY, b0 = -INFINITY, b1 = -INFINITY, b2 = -INFINITY;
      int c = 0;
      for (int i = K - 1; i >= 0; --i) {
        a0 = jsmin(a0, s->bmn[i][0]); a1 = jsmin(a1, s->bmn[i][1]); a2 = jsmin(a2, s->bmn[i][2]);
        b0 = jsmax(b0, s->bmx[i][0]); b1 = jsmax(b1, s->bmx[i][1]); b2 = jsmax(b2, s->bmx[i][2]);
        c += s->bcnt[i];
        s->smn[0][i] = (float)a0; s->smn[1][i] = (float)a1; s->smn[2][i] = (float)a2;
        s->smx[0][i] = (float)b0; s->smx[1][i] = (float)b1; s->smx[2][i] = (float)b2;
        s->sc[i] = c;
      }
    }
    for (int sp = 0; sp < K - 1; ++sp) { /* :628-653 */
      int lc = s->pc[sp], rc = s->sc[sp + 1];
      if (lc == 0 || rc == 0) continue;
      double lsa = sa_half(s->pmn[0][sp], s->pmn[1][sp], s->pmn[2][sp], s->pmx[0][sp], s->pmx[1][sp], s->pmx[2][sp]);
      double rsa = sa_half(s->smn[0][sp + 1], s->smn[1][sp + 1], s->smn[2][sp + 1], s->smx[0][sp + 1],
                           s->smx[1][sp + 1], s->smx[2][sp + 1]);
      double num = lsa * (double)lc + rsa * (double)rc;
      double cost = parent_sa > 0 ? num / parent_sa : num;
      if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = sp; }
    }
  }

  int split_axis = best_axis;
  uint32_t* left = (uint32_t*)malloc(count * sizeof(uint32_t));
  uint32_t* right = (uint32_t*)malloc(count * sizeof(uint32_t));
  size_t nl = 0, nr = 0;
  if (best_cost < leaf_cost && best_cost != INFINITY) { /* :659-671 */
    double span = cmx[best_axis] - cmn[best_axis];
    for (size_t i = 0; i < count; ++i) {
      const rec_t* r = &s->recs[subset[i]];
      double t = (r->cen[best_axis] - cmn[best_axis]) / span;
      double fb = floor(t * K);
      int b = fb < (double)(K - 1) ? (int)fb : K - 1;
      if (b <= best_split) left[nl++] = subset[i]; else right[nr++] = subset[i];
    }
  }
  if (nl == 0 || nr == 0) { /* balanced fallback :677-694 */
    split_axis = 0;
    double widest = cmx[0] - cmn[0];
    for (int axis = 1; axis < 3; ++axis) {
      double sp = cmx[axis] - cmn[axis];
      if (sp > widest) { split_axis = axis; widest = sp; }
    }
    uint32_t* ord = (uint32_t*)malloc(count * sizeof(uint32_t));
    memcpy(ord, subset, count * sizeof(uint32_t));
    g_sort_recs = s->recs;
    g_sort_axis = split_axis;
    qsort(ord, count, sizeof(uint32_t), cmp_fallback);
    size_t mid = count / 2;
    nl = mid; nr = count - mid;
    memcpy(left, ord, nl * sizeof(uint32_t));
    memcpy(right, ord + mid, nr * sizeof(uint32_t));
    free(ord);
  }
  build_rec(s, left, nl, depth + 1);
  free(left);
  size_t rc = s->err ? ni : build_rec(s, right, nr, depth + 1);
  free(right);
  s->nodes[ni].w6 = (uint32_t)(rc - ni);
  s->nodes[ni].w7 = (uint32_t)split_axis;
  return ni;
}

/*
 * Build the binary BVH.  Output: nodes (8 u32 words per node, the 32-byte
 * layout of buildArrayBvh.ts:13-27) and reordered-to-source triangle ids.
 * `out_nodes` must hold 2*ntri (at least 1) nodes.  Returns node count or -1.
 */
long orc_build_array_bvh(const float* positions, long n_pos_words, int pos_stride, const uint32_t* indices,
                         long ntri, int idx_stride, int max_leaf, int nbins, int max_depth, uint32_t* out_nodes,
                         uint32_t* out_reordered_to_source) {
  if (pos_stride != 3 && pos_stride != 4) return fail("positionStride must be 3 or 4");
  if (idx_stride != 3 && idx_stride != 4) return fail("indexStride must be 3 or 4");
  if (max_leaf < 1 || max_leaf > 0xFFFF) return fail("maxLeafTriangles out of range");
  if (nbins < 2 || nbins > 256) return fail("binCount out of range");
  if (max_depth < 0 || max_depth > 58) return fail("maxDepth out of range");
  if (n_pos_words % pos_stride) return fail("positions length not divisible by stride");
  for (long i = 0; i < n_pos_words; ++i)
    if (!isfinite(positions[i])) return fail("positions must be finite");
  if (ntri == 0) {
    memset(out_nodes, 0, 32);
    out_nodes[7] = ORC_LEAF_FLAG;
    return 1;
  }
  long nvert = n_pos_words / pos_stride;
  rec_t* recs = (rec_t*)malloc((size_t)ntri * sizeof(rec_t));
  for (long t = 0; t < ntri; ++t) {
    uint32_t iv[3] = {indices[t * idx_stride], indices[t * idx_stride + 1], indices[t * idx_stride + 2]};
    if (iv[0] >= (uint32_t)nvert || iv[1] >= (uint32_t)nvert || iv[2] >= (uint32_t)nvert) {
      free(recs);
      return fail("triangle references an out-of-range vertex");
    }
    rec_t r;
    r.tri = (uint32_t)t;
    for (int k = 0; k < 3; ++k) {
      double a = positions[(size_t)iv[0] * pos_stride + k], b = positions[(size_t)iv[1] * pos_stride + k],
             c = positions[(size_t)iv[2] * pos_stride + k];
      r.mn[k] = jsmin(jsmin(a, b), c); /* min3, buildArrayBvh.ts:165-175 */
      r.mx[k] = jsmax(jsmax(a, b), c);
      r.cen[k] = 0.5 * (r.mn[k] + r.mx[k]);
    }
    recs[t] = r;
  }
  bstate_t* s = (bstate_t*)calloc(1, sizeof(bstate_t));
  s->recs = recs;
  s->max_leaf = max_leaf;
  s->nbins = nbins;
  s->max_depth = max_depth;
  s->ordered = (uint32_t*)malloc((size_t)ntri * sizeof(uint32_t));
  uint32_t* all = (uint32_t*)malloc((size_t)ntri * sizeof(uint32_t));
  for (long t = 0; t < ntri; ++t) all[t] = (uint32_t)t;
  build_rec(s, all, (size_t)ntri, 0);
  free(all);
  long result = -1;
  if (!s->err) {
    for (size_t i = 0; i < s->n_nodes; ++i) {
      float f[6];
      for (int k = 0; k < 3; ++k) { f[k] = (float)s->nodes[i].mn[k]; f[3 + k] = (float)s->nodes[i].mx[k]; }
      memcpy(out_nodes + i * 8, f, 24);
      out_nodes[i * 8 + 6] = s->nodes[i].w6;
      out_nodes[i * 8 + 7] = s->nodes[i].w7;
    }
    memcpy(out_reordered_to_source, s->ordered, (size_t)ntri * sizeof(uint32_t));
    result = (long)s->n_nodes;
  }
  free(s->nodes);
  free(s->ordered);
  free(s);
  free(recs);
  return result;
}

/* ------------------------------------------------------------------ */
/* 8-wide collapse (compressedWideBvh.ts:180-418)                      */
/* ------------------------------------------------------------------ */
typedef struct {
  float mn[3], mx[3];
  uint32_t w6, w7;
} rnode_t; /* binary node as read back from the packed buffer */

static rnode_t read_bnode(const uint32_t* nodes, uint32_t i) {
  rnode_t r;
  memcpy(r.mn, nodes + (size_t)i * 8, 12);
  memcpy(r.mx, nodes + (size_t)i * 8 + 3, 12);
  r.w6 = nodes[(size_t)i * 8 + 6];
  r.w7 = nodes[(size_t)i * 8 + 7];
  return r;
}
static int is_leaf_word(uint32_t w) { return (w >> 16) == 0xFFFFu; }

static double sa_node(const rnode_t* n) {
  return sa_half(n->mn[0], n->mn[1], n->mn[2], n->mx[0], n->mx[1], n->mx[2]);
}

/* stableUnitOffset :185-195; returns 0 and sets *ok=0 for the null case. */
static double stable_unit_offset(double v, double mn, double mx, int* ok) {
  *ok = 1;
  if (!isfinite(v) || !isfinite(mn) || !isfinite(mx) || mn > mx) { *ok = 0; return 0; }
  if (mx == mn) return 0;
  double ext = mx - mn;
  if (isfinite(ext)) return (v - mn) / ext;
  double half = mx * 0.5 - mn * 0.5;
  if (!(half > 0) || !isfinite(half)) { *ok = 0; return 0; }
  return (v * 0.5 - mn * 0.5) / half;
}

static uint16_t clamp_u16(double v) {
  if (!isfinite(v)) return 0;
  double r = floor(v + 0.5); /* Math.round (integers here) */
  if (r < 0) r = 0;
  if (r > 65535) r = 65535;
  return (uint16_t)r;
}

/* quantizeBound :197-204 */
static uint16_t quantize_bound(double v, double mn, double mx, int ceil_mode) {
  int ok;
  double nrm = stable_unit_offset(v, mn, mx, &ok);
  if (!ok) return 0;
  if (mx == mn) return ceil_mode ? 65535 : 0;
  double q = nrm * 65535;
  double rounded = ceil_mode ? ceil(q) : floor(q);
  return clamp_u16(ceil_mode ? rounded + 1 : rounded - 1);
}

/* dequantizeBound :206-213 */
static double dequantize_bound(double q, double mn, double mx) {
  if (!isfinite(mn) || !isfinite(mx) || mn > mx) return NAN;
  if (mx == mn) return mn;
  if (q <= 0) return mn;
  if (q >= 65535) return mx;
  double t = q / 65535;
  return mn * (1 - t) + mx * t;
}

typedef struct {
  const uint32_t* bnodes;
  float* node_bounds;     /* 6 per wide node */
  uint16_t* child_bounds; /* 48 per wide node */
  uint32_t* child_meta;   /* 24 per wide node */
  uint32_t* child_count;  /* 1 per wide node */
  uint32_t* wide_to_binary; /* binary node index each wide node came from */
  long n, cap;
  int valid;
} wstate_t;

/* collectWideChildren :215-242 */
static int collect_children(const uint32_t* bn, uint32_t root, uint32_t* ch) {
  rnode_t r = read_bnode(bn, root);
  if (is_leaf_word(r.w7)) { ch[0] = root; return 1; }
  int n = 2;
  ch[0] = root + 1;
  ch[1] = root + r.w6;
  while (n < ORC_WIDE) {
    int at = -1;
    double best = -1;
    for (int i = 0; i < n; ++i) {
      rnode_t c = read_bnode(bn, ch[i]);
      if (is_leaf_word(c.w7)) continue;
      double a = sa_node(&c);
      if (a > best) { best = a; at = i; }
    }
    if (at < 0) break;
    uint32_t x = ch[at];
    rnode_t xn = read_bnode(bn, x);
    memmove(ch + at + 2, ch + at + 1, (size_t)(n - at - 1) * sizeof(uint32_t));
    ch[at] = x + 1;
    ch[at + 1] = x + xn.w6;
    ++n;
  }
  return n;
}

static long build_wide(wstate_t* w, uint32_t bi) {
  rnode_t parent = read_bnode(w->bnodes, bi);
  long wi = w->n++;
  if (wi >= w->cap) { w->valid = 0; return wi; }
  for (int k = 0; k < 3; ++k) { w->node_bounds[wi * 6 + k] = parent.mn[k]; w->node_bounds[wi * 6 + 3 + k] = parent.mx[k]; }
  memset(w->child_bounds + wi * 48, 0, 48 * sizeof(uint16_t));
  memset(w->child_meta + wi * 24, 0, 24 * sizeof(uint32_t));
  w->wide_to_binary[wi] = bi;
  uint32_t ch[ORC_WIDE];
  int nc = collect_children(w->bnodes, bi, ch);
  w->child_count[wi] = (uint32_t)nc;
  for (int slot = 0; slot < nc; ++slot) {
    rnode_t c = read_bnode(w->bnodes, ch[slot]);
    for (int k = 0; k < 3; ++k) { /* fillChildBounds validity :323-335 */
      int ok1, ok2;
      stable_unit_offset(c.mn[k], parent.mn[k], parent.mx[k], &ok1);
      stable_unit_offset(c.mx[k], parent.mn[k], parent.mx[k], &ok2);
      if (c.mn[k] < parent.mn[k] || c.mx[k] > parent.mx[k] || c.mn[k] > c.mx[k] || !ok1 || !ok2) w->valid = 0;
    }
    uint16_t* cb = w->child_bounds + wi * 48 + slot * 6;
    for (int k = 0; k < 3; ++k) {
      cb[k] = quantize_bound(c.mn[k], parent.mn[k], parent.mx[k], 0);
      cb[3 + k] = quantize_bound(c.mx[k], parent.mn[k], parent.mx[k], 1);
    }
    uint32_t* m = w->child_meta + wi * 24 + slot * 3;
    if (is_leaf_word(c.w7)) {
      m[0] = 2; m[1] = c.w6; m[2] = c.w7 & 0xFFFFu;
    } else {
      long cw = build_wide(w, ch[slot]);
      m = w->child_meta + wi * 24 + slot * 3;
      m[0] = 1; m[1] = (uint32_t)cw; m[2] = 0;
    }
  }
  return wi;
}

/* requiredCwbvhTraversalStackEntries :60-92 */
long orc_wide_stack_entries(const uint32_t* meta, const uint32_t* count, long n) {
  if (n == 0) return 0;
  uint32_t* stack = (uint32_t*)malloc((size_t)n * 8 * sizeof(uint32_t) + 64);
  uint8_t* seen = (uint8_t*)calloc((size_t)n, 1);
  long sp = 0, maximum = 1;
  stack[sp++] = 0;
  while (sp > 0) {
    uint32_t node = stack[--sp];
    if (seen[node]) { maximum = -1; break; }
    seen[node] = 1;
    uint32_t c = count[node];
    if (c > 8) { maximum = -1; break; }
    for (uint32_t s = 0; s < c; ++s) {
      const uint32_t* m = meta + (size_t)node * 24 + s * 3;
      if (m[0] != 1) continue;
      if (m[1] >= (uint32_t)n) { maximum = -1; break; }
      stack[sp++] = m[1];
    }
    if (maximum < 0) break;
    if (sp > maximum) maximum = sp;
  }
  free(stack);
  free(seen);
  return maximum;
}

/*
 * Collapse a binary BVH to the 8-wide quantised form.  Buffers must hold
 * `cap` wide nodes (a binary tree with B nodes gives at most B wide nodes).
 * Returns wide node count; *status: 0 wide, 1 empty, 2 binary-fallback.
 */
long orc_collapse_wide(const uint32_t* bnodes, long n_bnodes, long ntri, long cap, float* node_bounds,
                       uint16_t* child_bounds, uint32_t* child_meta, uint32_t* child_count,
                       uint32_t* wide_to_binary, int* status) {
  *status = 1;
  if (n_bnodes == 0) return 0;
  if (ntri == 0 || (n_bnodes == 1 && is_leaf_word(bnodes[7]) && (bnodes[7] & 0xFFFFu) == 0)) {
    memset(node_bounds, 0, 6 * sizeof(float));
    memset(child_bounds, 0, 48 * sizeof(uint16_t));
    memset(child_meta, 0, 24 * sizeof(uint32_t));
    child_count[0] = 0;
    return 1;
  }
  for (long i = 0; i < n_bnodes; ++i) {
    rnode_t r = read_bnode(bnodes, (uint32_t)i);
    for (int k = 0; k < 3; ++k) {
      int ok;
      stable_unit_offset(r.mn[k], r.mn[k], r.mx[k], &ok);
      if (!ok) {
        child_count[0] = 0xFFFFFFFFu;
        *status = 2;
        return 1;
      }
    }
  }
  wstate_t w = {bnodes, node_bounds, child_bounds, child_meta, child_count, wide_to_binary, 0, cap, 1};
  build_wide(&w, 0);
  if (w.n > cap) return fail("wide node capacity exceeded");
  long need = w.valid ? orc_wide_stack_entries(child_meta, child_count, w.n) : -1;
  if (!w.valid || need < 0 || need > ORC_STACK_CAPACITY) {
    for (long i = 0; i < w.n; ++i) child_count[i] = 0xFFFFFFFFu;
    *status = 2;
  } else {
    *status = 0;
  }
  return w.n;
}

/* ------------------------------------------------------------------ */
/* FP64 first-hit query (compressedWideBvh.ts:551-860)                 */
/* ------------------------------------------------------------------ */
typedef struct {
  const float* node_bounds;
  const uint16_t* child_bounds;
  const uint32_t* child_meta;
  const uint32_t* child_count;
  long n_wide;
  const float* positions;
  int pos_stride;
  const uint32_t* reordered_indices; /* source indices in BVH order, idx_stride words each */
  int idx_stride;
  const uint32_t* reordered_to_source;
  long ntri;
} orc_wide_t;

/* intersectTriangle :551-614.  Returns 1 on hit, writes t and bary (w,u,v). */
static int tri_fp64(const double o[3], const double d[3], const double a[3], const double b[3], const double c[3],
                    double tmin, double* t_out, double bary[3]) {
  double e1r[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double e2r[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double es = 0, ds = 0;
  for (int k = 0; k < 3; ++k) { es = jsmax(es, fabs(e1r[k])); }
  for (int k = 0; k < 3; ++k) { es = jsmax(es, fabs(e2r[k])); }
  for (int k = 0; k < 3; ++k) { ds = jsmax(ds, fabs(d[k])); }
  if (!(es > 0) || !isfinite(es) || !(ds > 0) || !isfinite(ds)) return 0;
  double ies = 1 / es, ids = 1 / ds;
  double e1[3] = {e1r[0] * ies, e1r[1] * ies, e1r[2] * ies};
  double e2[3] = {e2r[0] * ies, e2r[1] * ies, e2r[2] * ies};
  double dir[3] = {d[0] * ids, d[1] * ids, d[2] * ids};
  double ao[3] = {(o[0] - a[0]) * ies, (o[1] - a[1]) * ies, (o[2] - a[2]) * ies};
  double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  double det = -(dir[0] * n[0] + dir[1] * n[1] + dir[2] * n[2]);
  double nl = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  double dl = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  if (!(nl > 0) || !isfinite(nl) || !(dl > 0) || !isfinite(dl) || fabs(det) / (nl * dl) <= 1e-7) return 0;
  double inv = 1 / det;
  double dao[3] = {ao[1] * dir[2] - ao[2] * dir[1], ao[2] * dir[0] - ao[0] * dir[2], ao[0] * dir[1] - ao[1] * dir[0]};
  double u = (e2[0] * dao[0] + e2[1] * dao[1] + e2[2] * dao[2]) * inv;
  double v = -(e1[0] * dao[0] + e1[1] * dao[1] + e1[2] * dao[2]) * inv;
  double t = ((ao[0] * n[0] + ao[1] * n[1] + ao[2] * n[2]) * inv * es) / ds;
  double w = 1 - u - v;
  const double eps = 1e-6;
  if (!isfinite(u) || !isfinite(v) || !isfinite(w) || !isfinite(t) || u < -eps || v < -eps || w < -eps ||
      t < jsmax(tmin, 0))
    return 0;
  *t_out = t;
  bary[0] = w; bary[1] = u; bary[2] = v;
  return 1;
}

/* intersectAabb :616-645; returns 1 when the slab interval is non-empty. */
static int aabb_fp64(const double o[3], const double d[3], const double mn[3], const double mx[3], double tmin,
                     double tmax, double* tnear) {
  for (int k = 0; k < 3; ++k) {
    if (d[k] == 0) {
      if (o[k] < mn[k] || o[k] > mx[k]) return 0;
      continue;
    }
    double inv = 1 / d[k];
    double t0 = (mn[k] - o[k]) * inv, t1 = (mx[k] - o[k]) * inv;
    if (t0 > t1) { double x = t0; t0 = t1; t1 = x; }
    tmin = jsmax(tmin, t0);
    tmax = jsmin(tmax, t1);
    if (tmax < tmin) return 0;
  }
  if (tnear) *tnear = tmin;
  return 1;
}

static void child_box(const orc_wide_t* W, long node, int slot, double mn[3], double mx[3]) {
  const float* nb = W->node_bounds + node * 6;
  const uint16_t* cb = W->child_bounds + node * 48 + slot * 6;
  for (int k = 0; k < 3; ++k) {
    mn[k] = dequantize_bound(cb[k], nb[k], nb[3 + k]);
    mx[k] = dequantize_bound(cb[3 + k], nb[k], nb[3 + k]);
  }
}

static void vtx(const orc_wide_t* W, uint32_t i, double p[3]) {
  const float* q = W->positions + (size_t)i * W->pos_stride;
  p[0] = q[0]; p[1] = q[1]; p[2] = q[2];
}

typedef struct {
  int32_t prim;      /* source triangle index, -1 on miss */
  int32_t bvh_tri;   /* triangle index in BVH order */
  double t;
  double bary[3];    /* (w, u, v) */
} orc_hit_t;

/* intersectCompressedWideBvhFirstHit :754-860 (LIFO over slots, first-found wins on ties). */
static void first_hit_one(const orc_wide_t* W, const double o[3], const double d[3], double tmin, double tmax,
                          int any_hit, orc_hit_t* h) {
  double closest = tmax;
  h->prim = -1; h->bvh_tri = -1; h->t = tmax; h->bary[0] = h->bary[1] = h->bary[2] = 0;
  if (W->n_wide == 0) return;
  const float* rb = W->node_bounds;
  double rmn[3] = {rb[0], rb[1], rb[2]}, rmx[3] = {rb[3], rb[4], rb[5]};
  if (!aabb_fp64(o, d, rmn, rmx, tmin, closest, NULL)) return;
  uint32_t stack[4096];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    uint32_t node = stack[--sp];
    uint32_t cnt = W->child_count[node];
    if (cnt > 8) return;
    for (uint32_t slot = 0; slot < cnt; ++slot) {
      const uint32_t* m = W->child_meta + (size_t)node * 24 + slot * 3;
      double mn[3], mx[3];
      child_box(W, node, (int)slot, mn, mx);
      if (!aabb_fp64(o, d, mn, mx, tmin, closest, NULL)) continue;
      if (m[0] == 1) { if (sp < 4096) stack[sp++] = m[1]; continue; }
      for (uint32_t i = 0; i < m[2]; ++i) {
        uint32_t tri = m[1] + i;
        const uint32_t* ib = W->reordered_indices + (size_t)tri * W->idx_stride;
        double a[3], b[3], c[3], t, bary[3];
        vtx(W, ib[0], a); vtx(W, ib[1], b); vtx(W, ib[2], c);
        if (tri_fp64(o, d, a, b, c, tmin, &t, bary) && t > tmin && t < closest) {
          closest = t;
          h->prim = (int32_t)W->reordered_to_source[tri];
          h->bvh_tri = (int32_t)tri;
          h->t = t;
          h->bary[0] = bary[0]; h->bary[1] = bary[1]; h->bary[2] = bary[2];
          (void)any_hit;
        }
      }
    }
  }
}

/*
 * Near-first traversal of the same wide tree that counts wide-node visits
 * and triangle tests: children sorted by slab entry distance, internal
 * children pushed far-to-near with their entry distance, popped entries
 * culled once they lie beyond the current closest hit.  Hits are identical
 * to first_hit_one up to exact t ties.
 */
static void count_one(const orc_wide_t* W, const double o[3], const double d[3], double tmin, double tmax,
                      long* n_nodes, long* n_tris, int any) {
  double closest = tmax;
  if (W->n_wide == 0) return;
  const float* rb = W->node_bounds;
  double rmn[3] = {rb[0], rb[1], rb[2]}, rmx[3] = {rb[3], rb[4], rb[5]};
  double t0;
  if (!aabb_fp64(o, d, rmn, rmx, tmin, closest, &t0)) return;
  uint32_t st_node[4096];
  double st_t[4096];
  int sp = 0;
  st_node[sp] = 0; st_t[sp] = t0; ++sp;
  while (sp > 0) {
    --sp;
    uint32_t node = st_node[sp];
    if (st_t[sp] > closest) continue;
    *n_nodes += 1;
    uint32_t cnt = W->child_count[node];
    if (cnt > 8) return;
    int order[8];
    double tn[8];
    int nh = 0;
    for (uint32_t slot = 0; slot < cnt; ++slot) {
      double mn[3], mx[3], te;
      child_box(W, node, (int)slot, mn, mx);
      if (!aabb_fp64(o, d, mn, mx, tmin, closest, &te)) continue;
      int j = nh++;
      while (j > 0 && tn[j - 1] > te) { tn[j] = tn[j - 1]; order[j] = order[j - 1]; --j; }
      tn[j] = te; order[j] = (int)slot;
    }
    /* leaves in near-to-far order */
    for (int k = 0; k < nh; ++k) {
      const uint32_t* m = W->child_meta + (size_t)node * 24 + order[k] * 3;
      if (m[0] != 2 || tn[k] > closest) continue;
      for (uint32_t i = 0; i < m[2]; ++i) {
        uint32_t tri = m[1] + i;
        const uint32_t* ib = W->reordered_indices + (size_t)tri * W->idx_stride;
        double a[3], b[3], c[3], t, bary[3];
        vtx(W, ib[0], a); vtx(W, ib[1], b); vtx(W, ib[2], c);
        *n_tris += 1;
        if (tri_fp64(o, d, a, b, c, tmin, &t, bary) && t > tmin && t < closest) {
          closest = t;
          if (any) return;
        }
      }
    }
    /* internal children far-to-near so the nearest pops first */
    for (int k = nh - 1; k >= 0; --k) {
      const uint32_t* m = W->child_meta + (size_t)node * 24 + order[k] * 3;
      if (m[0] != 1 || sp >= 4096) continue;
      st_node[sp] = m[1]; st_t[sp] = tn[k]; ++sp;
    }
  }
}

typedef struct {
  orc_wide_t W;
  const float* rays;
  int32_t* prim;
  double* t;
  double* bary_uv;
  int32_t* bvh_tri;
  int any;
  long nodes[256], tris[256];
} batch_ctx_t;

static void first_hit_range(void* c, long b, long e, int worker) {
  batch_ctx_t* x = (batch_ctx_t*)c;
  (void)worker;
  for (long r = b; r < e; ++r) {
    const float* ry = x->rays + r * 8;
    double o[3] = {ry[0], ry[1], ry[2]}, d[3] = {ry[4], ry[5], ry[6]};
    orc_hit_t h;
    first_hit_one(&x->W, o, d, ry[3], ry[7], 0, &h);
    if (x->prim) x->prim[r] = h.prim;
    if (x->t) x->t[r] = h.prim >= 0 ? h.t : INFINITY;
    if (x->bary_uv) { x->bary_uv[2 * r] = h.bary[1]; x->bary_uv[2 * r + 1] = h.bary[2]; }
    if (x->bvh_tri) x->bvh_tri[r] = h.bvh_tri;
  }
}

static void count_range(void* c, long b, long e, int worker) {
  batch_ctx_t* x = (batch_ctx_t*)c;
  for (long r = b; r < e; ++r) {
    const float* ry = x->rays + r * 8;
    double o[3] = {ry[0], ry[1], ry[2]}, d[3] = {ry[4], ry[5], ry[6]};
    long a = 0, q = 0;
    count_one(&x->W, o, d, ry[3], ry[7], &a, &q, x->any);
    x->nodes[worker] += a;
    x->tris[worker] += q;
  }
}

/*
 * Batch first-hit.  rays: 8 floats per ray (ox oy oz tmin dx dy dz tmax).
 * Outputs (each optional): prim (source id or -1), t (f64), bary (u,v f64
 * pairs), bvh_tri.  nthreads <= 0 uses every online core.
 */
int orc_first_hit_batch(const float* node_bounds, const uint16_t* child_bounds, const uint32_t* child_meta,
                        const uint32_t* child_count, long n_wide, const float* positions, int pos_stride,
                        const uint32_t* reordered_indices, int idx_stride, const uint32_t* reordered_to_source,
                        long ntri, const float* rays, long nrays, int32_t* prim, double* t, double* bary_uv,
                        int32_t* bvh_tri, int nthreads) {
  batch_ctx_t* x = (batch_ctx_t*)calloc(1, sizeof(batch_ctx_t));
  orc_wide_t W = {node_bounds, child_bounds, child_meta, child_count, n_wide, positions,
                  pos_stride, reordered_indices, idx_stride, reordered_to_source, ntri};
  x->W = W; x->rays = rays; x->prim = prim; x->t = t; x->bary_uv = bary_uv; x->bvh_tri = bvh_tri;
  parallel_for(nrays, 512, nthreads, first_hit_range, x);
  free(x);
  return 0;
}

/* Near-first node-visit / triangle-test counts summed over a ray batch. */
int orc_count_visits(const float* node_bounds, const uint16_t* child_bounds, const uint32_t* child_meta,
                     const uint32_t* child_count, long n_wide, const float* positions, int pos_stride,
                     const uint32_t* reordered_indices, int idx_stride, const float* rays, long nrays,
                     long* out_nodes, long* out_tris, int nthreads, int any) {
  batch_ctx_t* x = (batch_ctx_t*)calloc(1, sizeof(batch_ctx_t));
  orc_wide_t W = {node_bounds, child_bounds, child_meta, child_count, n_wide, positions,
                  pos_stride, reordered_indices, idx_stride, NULL, 0};
  x->W = W; x->rays = rays; x->any = any;
  parallel_for(nrays, 512, nthreads, count_range, x);
  long sn = 0, st = 0;
  for (int i = 0; i < 256; ++i) { sn += x->nodes[i]; st += x->tris[i]; }
  *out_nodes = sn;
  *out_tris = st;
  free(x);
  return 0;
}

/* Brute force over all triangles with the same FP64 test (small cases). */
int orc_brute_first_hit(const float* positions, int pos_stride, const uint32_t* indices, int idx_stride, long ntri,
                        const float* rays, long nrays, int32_t* prim, double* t, double* bary_uv,
                        double* second_t) {
  for (long r = 0; r < nrays; ++r) {
    const float* ry = rays + r * 8;
    double o[3] = {ry[0], ry[1], ry[2]}, d[3] = {ry[4], ry[5], ry[6]};
    double tmin = ry[3], closest = ry[7], second = INFINITY;
    int32_t best = -1;
    double bb[3] = {0, 0, 0};
    for (long k = 0; k < ntri; ++k) {
      double a[3], b[3], c[3], tt, bary[3];
      const uint32_t* ib = indices + (size_t)k * idx_stride;
      for (int j = 0; j < 3; ++j) {
        a[j] = positions[(size_t)ib[0] * pos_stride + j];
        b[j] = positions[(size_t)ib[1] * pos_stride + j];
        c[j] = positions[(size_t)ib[2] * pos_stride + j];
      }
      if (!tri_fp64(o, d, a, b, c, tmin, &tt, bary) || !(tt > tmin)) continue;
      if (tt < closest) {
        if (best >= 0 && closest < second) second = closest;
        closest = tt; best = (int32_t)k; bb[0] = bary[0]; bb[1] = bary[1]; bb[2] = bary[2];
      } else if (tt < second) {
        second = tt;
      }
    }
    prim[r] = best;
    if (t) t[r] = best >= 0 ? closest : INFINITY;
    if (bary_uv) { bary_uv[2 * r] = bb[1]; bary_uv[2 * r + 1] = bb[2]; }
    if (second_t) second_t[r] = second;
  }
  return 0;
}

/* FP64 triangle test on double inputs (the path-tracer oracle uses it). */
int orc_tri_hit_d(const double o[3], const double d[3], const double a[3], const double b[3], const double c[3],
                  double tmin, double* t) {
  double bary[3];
  return tri_fp64(o, d, a, b, c, tmin, t, bary);
}

/* FP64 single triangle test exposed for unit tests. */
int orc_triangle_fp64(const float* o, const float* d, const float* a, const float* b, const float* c, double tmin,
                      double* t, double* bary) {
  double O[3] = {o[0], o[1], o[2]}, D[3] = {d[0], d[1], d[2]};
  double A[3] = {a[0], a[1], a[2]}, B[3] = {b[0], b[1], b[2]}, C[3] = {c[0], c[1], c[2]};
  return tri_fp64(O, D, A, B, C, tmin, t, bary);
}

/* ------------------------------------------------------------------ */
/* f32 watertight triangle (opticalWatertightTriangle.ts:98-220)        */
/* ------------------------------------------------------------------ */
static float edge_fn(const float a[2], const float b[2]) {
  if (a[0] == b[0] && a[1] == b[1]) return 0.0f;
  int ordered = a[0] < b[0] || (a[0] == b[0] && a[1] < b[1]);
  const float* f = ordered ? a : b;
  const float* s = ordered ? b : a;
  float p = f[0] * s[1];
  float q = f[1] * s[0];
  float canon = p - q;
  return ordered ? canon : -canon;
}

/* Math.max over f32 values: NaN propagates. */
static float fmax3n(float a, float b, float c) {
  if (isnan(a) || isnan(b) || isnan(c)) return NAN;
  return fmaxf(fmaxf(a, b), c);
}

static float ray_param(const float o[3], const float d[3], const float p[3]) {
  float del[3] = {p[0] - o[0], p[1] - o[1], p[2] - o[2]};
  float dls = fmax3n(fabsf(del[0]), fabsf(del[1]), fabsf(del[2]));
  float drs = fmax3n(fabsf(d[0]), fabsf(d[1]), fabsf(d[2]));
  if (!(drs > 0) || !isfinite(drs) || !isfinite(dls)) return -1.0f;
  if (!(dls > 0)) return 0.0f;
  float dd[3] = {d[0] / drs, d[1] / drs, d[2] / drs};
  float q[3] = {del[0] / dls, del[1] / dls, del[2] / dls};
  float m0 = q[0] * dd[0], m1 = q[1] * dd[1], m2 = q[2] * dd[2];
  float num = (m0 + m1) + m2;
  float n0 = dd[0] * dd[0], n1 = dd[1] * dd[1], n2 = dd[2] * dd[2];
  float den = (n0 + n1) + n2;
  float r1 = num / den, r2 = dls / drs;
  return r1 * r2;
}

static int lex_before(const float a[3], const float b[3]) {
  return a[0] < b[0] || (a[0] == b[0] && (a[1] < b[1] || (a[1] == b[1] && a[2] < b[2])));
}

static float edge_ray_param(const float o[3], const float d[3], const float fi[3], const float si[3],
                            const float fpi[2], const float spi[2], float pt[3]) {
  int ordered = lex_before(fi, si);
  const float* f = ordered ? fi : si;
  const float* s = ordered ? si : fi;
  const float* fp = ordered ? fpi : spi;
  const float* sp = ordered ? spi : fpi;
  float del[2] = {sp[0] - fp[0], sp[1] - fp[1]};
  float ip;
  if (fabsf(del[0]) >= fabsf(del[1])) {
    if (del[0] == 0) { pt[0] = pt[1] = pt[2] = 0; return -1.0f; }
    ip = -fp[0] / del[0];
  } else {
    if (del[1] == 0) { pt[0] = pt[1] = pt[2] = 0; return -1.0f; }
    ip = -fp[1] / del[1];
  }
  for (int k = 0; k < 3; ++k) {
    float e = s[k] - f[k];
    float m = ip * e;
    pt[k] = f[k] + m;
  }
  return ray_param(o, d, pt);
}

/* Returns hit flag; out: t, bary[3] (weights of a,b,c), side, zero-edge mask. */
int orc_watertight_f32(const float* o, const float* dir, const float* a, const float* b, const float* c,
                       float exclusive_min_t, float* t_out, float* bary_out, int* side_out, int* mask_out) {
  *t_out = INFINITY;
  bary_out[0] = bary_out[1] = bary_out[2] = 0;
  *side_out = 0;
  *mask_out = 0;
  float ds = fmax3n(fabsf(dir[0]), fabsf(dir[1]), fabsf(dir[2]));
  if (!(ds > 0) || !isfinite(ds) || isnan(exclusive_min_t)) return 0;
  float d[3] = {dir[0] / ds, dir[1] / ds, dir[2] / ds};
  int kz = fabsf(d[1]) > fabsf(d[0]) ? 1 : 0;
  if (fabsf(d[2]) > fabsf(d[kz])) kz = 2;
  int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
  if (d[kz] < 0) { int x = kx; kx = ky; ky = x; }
  float sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = 1.0f / d[kz];
  float pa[3] = {a[0] - o[0], a[1] - o[1], a[2] - o[2]};
  float pb[3] = {b[0] - o[0], b[1] - o[1], b[2] - o[2]};
  float pc[3] = {c[0] - o[0], c[1] - o[1], c[2] - o[2]};
  float ap[2], bp[2], cp[2];
  { float m = sx * pa[kz]; ap[0] = pa[kx] - m; m = sy * pa[kz]; ap[1] = pa[ky] - m; }
  { float m = sx * pb[kz]; bp[0] = pb[kx] - m; m = sy * pb[kz]; bp[1] = pb[ky] - m; }
  { float m = sx * pc[kz]; cp[0] = pc[kx] - m; m = sy * pc[kz]; cp[1] = pc[ky] - m; }
  float e0 = edge_fn(bp, cp), e1 = edge_fn(cp, ap), e2 = edge_fn(ap, bp);
  float det = (e0 + e1) + e2;
  if (det == 0 || !isfinite(det)) return 0;
  int pos = det > 0;
  float n0 = pos ? e0 : -e0, n1 = pos ? e1 : -e1, n2 = pos ? e2 : -e2;
  if (n0 < 0 || n1 < 0 || n2 < 0) return 0;
  float az = pa[kz] * sz, bz = pb[kz] * sz, cz = pc[kz] * sz;
  float st;
  { float x0 = e0 * az, x1 = e1 * bz, x2 = e2 * cz; st = (x0 + x1) + x2; }
  float t = (st / det) / ds;
  float pt[3] = {0, 0, 0};
  int zc = (n0 == 0) + (n1 == 0) + (n2 == 0);
  if (zc >= 2) {
    if (n0 != 0) { memcpy(pt, a, 12); t = ray_param(o, dir, pt); }
    if (n1 != 0) { memcpy(pt, b, 12); t = ray_param(o, dir, pt); }
    if (n2 != 0) { memcpy(pt, c, 12); t = ray_param(o, dir, pt); }
  } else if (n0 == 0) {
    t = edge_ray_param(o, dir, b, c, bp, cp, pt);
  } else if (n1 == 0) {
    t = edge_ray_param(o, dir, c, a, cp, ap, pt);
  } else if (n2 == 0) {
    t = edge_ray_param(o, dir, a, b, ap, bp, pt);
  }
  float lo = exclusive_min_t > 0 ? exclusive_min_t : 0.0f;
  if (!(t > lo) || !isfinite(t)) return 0;
  float e1r[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  float e2r[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  float es = 0;
  for (int k = 0; k < 3; ++k) { es = fmaxf(es, fabsf(e1r[k])); }
  for (int k = 0; k < 3; ++k) { es = fmaxf(es, fabsf(e2r[k])); }
  if (!(es > 0) || !isfinite(es)) return 0;
  float s1[3] = {e1r[0] / es, e1r[1] / es, e1r[2] / es};
  float s2[3] = {e2r[0] / es, e2r[1] / es, e2r[2] / es};
  float nr[3];
  { float p = s1[1] * s2[2], q = s1[2] * s2[1]; nr[0] = p - q; }
  { float p = s1[2] * s2[0], q = s1[0] * s2[2]; nr[1] = p - q; }
  { float p = s1[0] * s2[1], q = s1[1] * s2[0]; nr[2] = p - q; }
  float ns = fmax3n(fabsf(nr[0]), fabsf(nr[1]), fabsf(nr[2]));
  if (!(ns > 0) || !isfinite(ns)) return 0;
  float nd[3] = {nr[0] / ns, nr[1] / ns, nr[2] / ns};
  float l0 = nd[0] * nd[0], l1 = nd[1] * nd[1], l2 = nd[2] * nd[2];
  float l2s = (l0 + l1) + l2;
  float nl = sqrtf(l2s);
  if (!(nl > 0) || !isfinite(nl)) return 0;
  float nn[3] = {nd[0] / nl, nd[1] / nl, nd[2] / nl};
  float q0 = d[0] * nn[0], q1 = d[1] * nn[1], q2 = d[2] * nn[2];
  float sd = -((q0 + q1) + q2);
  if (sd == 0 || !isfinite(sd)) return 0;
  *t_out = t;
  bary_out[0] = e0 / det; bary_out[1] = e1 / det; bary_out[2] = e2 / det;
  *side_out = sd > 0 ? 1 : -1;
  *mask_out = (n0 == 0 ? 1 : 0) | (n1 == 0 ? 2 : 0) | (n2 == 0 ? 4 : 0);
  return 1;
}

/* ------------------------------------------------------------------ */
/* first hit with the f32 watertight test over the same wide tree       */
/* ------------------------------------------------------------------ */
/* Same LIFO traversal as first_hit_one (FP64 slab tests on dequantised
 * bounds), triangles decided by orc_watertight_f32 with tmin exclusive and
 * strict t < closest in f32: the semantic of the device path. */
static void first_hit_wt_one(const orc_wide_t* W, const float* ry, int32_t* prim, float* t_out, float* bary_out) {
  double o[3] = {ry[0], ry[1], ry[2]}, d[3] = {ry[4], ry[5], ry[6]};
  float of[3] = {ry[0], ry[1], ry[2]}, df[3] = {ry[4], ry[5], ry[6]};
  float tmin = ry[3];
  float closest = ry[7];
  *prim = -1; *t_out = closest; bary_out[0] = bary_out[1] = bary_out[2] = 0;
  if (W->n_wide == 0) return;
  uint32_t stack[4096];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    uint32_t node = stack[--sp];
    uint32_t cnt = W->child_count[node];
    if (cnt > 8) return;
    for (uint32_t slot = 0; slot < cnt; ++slot) {
      const uint32_t* m = W->child_meta + (size_t)node * 24 + slot * 3;
      double mn[3], mx[3];
      child_box(W, node, (int)slot, mn, mx);
      /* widen the interval slightly: box culling must never decide a hit */
      if (!aabb_fp64(o, d, mn, mx, (double)tmin * (1 - 1e-9) - 1e-30, (double)closest * (1 + 1e-9) + 1e-30, NULL))
        continue;
      if (m[0] == 1) { if (sp < 4096) stack[sp++] = m[1]; continue; }
      for (uint32_t i = 0; i < m[2]; ++i) {
        uint32_t tri = m[1] + i;
        const uint32_t* ib = W->reordered_indices + (size_t)tri * W->idx_stride;
        float a[3], b[3], c[3], t, bary[3];
        int side, mask;
        for (int k = 0; k < 3; ++k) {
          a[k] = W->positions[(size_t)ib[0] * W->pos_stride + k];
          b[k] = W->positions[(size_t)ib[1] * W->pos_stride + k];
          c[k] = W->positions[(size_t)ib[2] * W->pos_stride + k];
        }
        if (orc_watertight_f32(of, df, a, b, c, tmin, &t, bary, &side, &mask) && t < closest) {
          closest = t;
          *prim = (int32_t)W->reordered_to_source[tri];
          *t_out = t;
          bary_out[0] = bary[0]; bary_out[1] = bary[1]; bary_out[2] = bary[2];
        }
      }
    }
  }
}

typedef struct {
  orc_wide_t W;
  const float* rays;
  int32_t* prim;
  float* t;
  float* bary;
} wt_ctx_t;

static void first_hit_wt_range(void* c, long b, long e, int worker) {
  wt_ctx_t* x = (wt_ctx_t*)c;
  (void)worker;
  for (long r = b; r < e; ++r) {
    float bary[3];
    first_hit_wt_one(&x->W, x->rays + r * 8, &x->prim[r], &x->t[r], bary);
    x->bary[3 * r] = bary[0]; x->bary[3 * r + 1] = bary[1]; x->bary[3 * r + 2] = bary[2];
  }
}

/* Batch first hit with the f32 watertight test.  bary: 3 floats per ray (a, b, c weights). */
int orc_first_hit_wt_batch(const float* node_bounds, const uint16_t* child_bounds, const uint32_t* child_meta,
                           const uint32_t* child_count, long n_wide, const float* positions, int pos_stride,
                           const uint32_t* reordered_indices, int idx_stride, const uint32_t* reordered_to_source,
                           long ntri, const float* rays, long nrays, int32_t* prim, float* t, float* bary,
                           int nthreads) {
  wt_ctx_t* x = (wt_ctx_t*)calloc(1, sizeof(wt_ctx_t));
  orc_wide_t W = {node_bounds, child_bounds, child_meta, child_count, n_wide, positions,
                  pos_stride, reordered_indices, idx_stride, reordered_to_source, ntri};
  x->W = W; x->rays = rays; x->prim = prim; x->t = t; x->bary = bary;
  parallel_for(nrays, 512, nthreads, first_hit_wt_range, x);
  free(x);
  return 0;
}

/* ------------------------------------------------------------------ */
/* TLAS build over instance AABBs (tlas.ts:257-989)                    */
/* ------------------------------------------------------------------ */
typedef struct {
  uint32_t orig;
  double cen[3], mn[3], mx[3];
} trec_t;

typedef struct {
  double mn[3], mx[3];
  uint32_t w6, w7;
} tnode_t;

typedef struct {
  tnode_t* nodes;
  long n, cap;
  uint32_t* perm;
  long np;
  int max_leaf, nbins, max_depth, err;
} tstate_t;

static double tsa(const double mn[3], const double mx[3]) { /* aabbSurfaceArea :265-273 */
  double dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  dx = jsmax(0, dx); dy = jsmax(0, dy); dz = jsmax(0, dz);
  return 2 * (dx * dy + dy * dz + dz * dx);
}

static int min_balanced_depth(long count, int max_leaf) { /* :423-426 */
  long leaves = (count + max_leaf - 1) / max_leaf;
  if (leaves <= 1) return 0;
  return (int)ceil(log2((double)leaves));
}

static const trec_t* g_tsort;
static int g_taxis;
static int cmp_tbal(const void* pa, const void* pb) {
  const trec_t* a = &g_tsort[*(const uint32_t*)pa];
  const trec_t* b = &g_tsort[*(const uint32_t*)pb];
  double d = a->cen[g_taxis] - b->cen[g_taxis];
  if (d != 0) return d < 0 ? -1 : 1;
  return a->orig < b->orig ? -1 : (a->orig > b->orig ? 1 : 0);
}

static long tpush(tstate_t* s) {
  if (s->n == s->cap) {
    s->cap = s->cap ? 2 * s->cap : 64;
    s->nodes = (tnode_t*)realloc(s->nodes, (size_t)s->cap * sizeof(tnode_t));
  }
  return s->n++;
}

static int tbin(double c, double cmin, double ext, int K) { /* Math.floor((c - cMin) / ext * K) clamped */
  double t = floor((c - cmin) / ext * K);
  if (t < 0) t = 0;
  if (t > K - 1) t = K - 1;
  return (int)t;
}

/* buildRecursive :467-579; sub holds record indices into R */
static long tbuild(tstate_t* s, const trec_t* R, uint32_t* sub, long cnt, int depth) {
  long me = s->n;
  if (cnt <= s->max_leaf) { /* buildLeaf :289-309 */
    long ni = tpush(s);
    tnode_t nd;
    for (int k = 0; k < 3; ++k) { nd.mn[k] = INFINITY; nd.mx[k] = -INFINITY; }
    for (long i = 0; i < cnt; ++i)
      for (int k = 0; k < 3; ++k) {
        if (R[sub[i]].mn[k] < nd.mn[k]) nd.mn[k] = R[sub[i]].mn[k];
        if (R[sub[i]].mx[k] > nd.mx[k]) nd.mx[k] = R[sub[i]].mx[k];
      }
    nd.w6 = (uint32_t)s->np;
    nd.w7 = ORC_LEAF_FLAG | (uint32_t)cnt;
    s->nodes[ni] = nd;
    for (long i = 0; i < cnt; ++i) s->perm[s->np++] = R[sub[i]].orig;
    return me;
  }
  if (depth >= s->max_depth || min_balanced_depth(cnt, s->max_leaf) > s->max_depth - depth) {
    s->err = 1;
    return me;
  }
  double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long i = 0; i < cnt; ++i) /* computeCentroidBounds :316-328 */
    for (int k = 0; k < 3; ++k) {
      if (R[sub[i]].cen[k] < cmn[k]) cmn[k] = R[sub[i]].cen[k];
      if (R[sub[i]].cen[k] > cmx[k]) cmx[k] = R[sub[i]].cen[k];
    }
  const int K = s->nbins;
  double ext[3] = {cmx[0] - cmn[0], cmx[1] - cmn[1], cmx[2] - cmn[2]};
  int have = 0, baxis = 0, bbin = 0;
  double bcost = 0;
  if (!(ext[0] <= 0 && ext[1] <= 0 && ext[2] <= 0)) { /* pickSplit :330-393 */
    double (*bmn)[3] = malloc(sizeof(double[3]) * K), (*bmx)[3] = malloc(sizeof(double[3]) * K);
    long* bc = malloc(sizeof(long) * K);
    double *lsa = malloc(sizeof(double) * K), *rsa = malloc(sizeof(double) * K);
    long *lc = malloc(sizeof(long) * K), *rc = malloc(sizeof(long) * K);
    for (int axis = 0; axis < 3; ++axis) {
      if (ext[axis] <= 0) continue;
      for (int b = 0; b < K; ++b) {
        for (int k = 0; k < 3; ++k) { bmn[b][k] = INFINITY; bmx[b][k] = -INFINITY; }
        bc[b] = 0;
      }
      for (long i = 0; i < cnt; ++i) {
        const trec_t* r = &R[sub[i]];
        int b = tbin(r->cen[axis], cmn[axis], ext[axis], K);
        for (int k = 0; k < 3; ++k) {
          if (r->mn[k] < bmn[b][k]) bmn[b][k] = r->mn[k];
          if (r->mx[k] > bmx[b][k]) bmx[b][k] = r->mx[k];
        }
        bc[b] += 1;
      }
      double lmn[3] = {INFINITY, INFINITY, INFINITY}, lmx[3] = {-INFINITY, -INFINITY, -INFINITY};
      long lcount = 0;
      for (int b = 0; b < K; ++b) { /* unionBinInto skips empty bins :279-288 */
        if (bc[b]) {
          for (int k = 0; k < 3; ++k) {
            if (bmn[b][k] < lmn[k]) lmn[k] = bmn[b][k];
            if (bmx[b][k] > lmx[k]) lmx[k] = bmx[b][k];
          }
          lcount += bc[b];
        }
        lsa[b] = tsa(lmn, lmx);
        lc[b] = lcount;
      }
      double rmn[3] = {INFINITY, INFINITY, INFINITY}, rmx[3] = {-INFINITY, -INFINITY, -INFINITY};
      long rcount = 0;
      for (int b = K - 1; b >= 0; --b) {
        if (bc[b]) {
          for (int k = 0; k < 3; ++k) {
            if (bmn[b][k] < rmn[k]) rmn[k] = bmn[b][k];
            if (bmx[b][k] > rmx[k]) rmx[k] = bmx[b][k];
          }
          rcount += bc[b];
        }
        rsa[b] = tsa(rmn, rmx);
        rc[b] = rcount;
      }
      double total = lsa[K - 1];
      if (total <= 0) continue;
      for (int b = 0; b < K - 1; ++b) {
        if (lc[b] == 0 || rc[b + 1] == 0) continue;
        double sah = ((double)lc[b] * lsa[b] + (double)rc[b + 1] * rsa[b + 1]) / total;
        if (!have || sah < bcost) { have = 1; baxis = axis; bbin = b; bcost = sah; }
      }
    }
    free(bmn); free(bmx); free(bc); free(lsa); free(rsa); free(lc); free(rc);
  }
  int axis = have ? baxis : 0;
  uint32_t* left = malloc(sizeof(uint32_t) * (size_t)cnt);
  uint32_t* right = malloc(sizeof(uint32_t) * (size_t)cnt);
  long nl = 0, nr = 0;
  int fallback = 0;
  if (!have) fallback = 1;
  else if (bcost >= (double)cnt) fallback = 1;
  else {
    for (long i = 0; i < cnt; ++i) { /* partitionByBin :395-413 */
      int b = tbin(R[sub[i]].cen[baxis], cmn[baxis], ext[baxis], K);
      if (b <= bbin) left[nl++] = sub[i]; else right[nr++] = sub[i];
    }
    if (nl == 0 || nr == 0) fallback = 1;
    else if (min_balanced_depth(nl, s->max_leaf) > s->max_depth - (depth + 1) ||
             min_balanced_depth(nr, s->max_leaf) > s->max_depth - (depth + 1))
      fallback = 1;
  }
  if (fallback) { /* balancedPartition :429-451 */
    axis = 0;
    if (ext[1] > ext[axis]) axis = 1;
    if (ext[2] > ext[axis]) axis = 2;
    uint32_t* ord = malloc(sizeof(uint32_t) * (size_t)cnt);
    memcpy(ord, sub, sizeof(uint32_t) * (size_t)cnt);
    g_tsort = R;
    g_taxis = axis;
    qsort(ord, (size_t)cnt, sizeof(uint32_t), cmp_tbal);
    long mid = cnt / 2;
    nl = mid; nr = cnt - mid;
    memcpy(left, ord, sizeof(uint32_t) * (size_t)nl);
    memcpy(right, ord + mid, sizeof(uint32_t) * (size_t)nr);
    free(ord);
  }
  long ni = tpush(s);
  s->nodes[ni].w7 = (uint32_t)axis;
  tbuild(s, R, left, nl, depth + 1);
  long ri = tbuild(s, R, right, nr, depth + 1);
  free(left);
  free(right);
  tnode_t* me_n = &s->nodes[ni];
  const tnode_t* L = &s->nodes[ni + 1];
  const tnode_t* Rn = &s->nodes[ri];
  me_n->w6 = (uint32_t)(ri - ni);
  for (int k = 0; k < 3; ++k) {
    me_n->mn[k] = jsmin(L->mn[k], Rn->mn[k]);
    me_n->mx[k] = jsmax(L->mx[k], Rn->mx[k]);
  }
  return me;
}

/*
 * buildTlas (tlas.ts:859).  aabb: 6 doubles per instance (min xyz, max xyz).
 * Outputs packed nodes (8 u32 each, f32 bounds) and instanceIndices.
 * Returns node count or -1.
 */
long orc_build_tlas(const double* aabb, long n, int max_leaf, int nbins, int max_depth, uint32_t* out_nodes,
                    uint32_t* out_perm) {
  if (n <= 0) return fail("buildTlas: instances list is empty");
  trec_t* R = (trec_t*)malloc(sizeof(trec_t) * (size_t)n);
  for (long i = 0; i < n; ++i) {
    R[i].orig = (uint32_t)i;
    for (int k = 0; k < 3; ++k) {
      R[i].mn[k] = aabb[6 * i + k];
      R[i].mx[k] = aabb[6 * i + 3 + k];
      R[i].cen[k] = (R[i].mn[k] + R[i].mx[k]) * 0.5; /* aabbCentroid :187-193 */
    }
  }
  tstate_t s;
  memset(&s, 0, sizeof s);
  s.perm = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  s.max_leaf = max_leaf;
  s.nbins = nbins;
  s.max_depth = max_depth;
  uint32_t* all = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  for (long i = 0; i < n; ++i) all[i] = (uint32_t)i;
  long result = -1;
  if (min_balanced_depth(n, max_leaf) <= max_depth) {
    tbuild(&s, R, all, n, 0);
    if (!s.err) {
      for (long i = 0; i < s.n; ++i) { /* flattenNodes :581-598 */
        float f[6];
        for (int k = 0; k < 3; ++k) { f[k] = (float)s.nodes[i].mn[k]; f[3 + k] = (float)s.nodes[i].mx[k]; }
        memcpy(out_nodes + 8 * i, f, 24);
        out_nodes[8 * i + 6] = s.nodes[i].w6;
        out_nodes[8 * i + 7] = s.nodes[i].w7;
      }
      memcpy(out_perm, s.perm, sizeof(uint32_t) * (size_t)n);
      result = s.n;
    }
  }
  if (result < 0) fail("buildTlas: cannot encode the instances within the traversal-safe depth");
  free(all);
  free(R);
  free(s.nodes);
  free(s.perm);
  return result;
}
