/*
 * lt_oracle.c -- CPU restatement of the reference's light tree.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the device light tree).
 *
 * Follows packages/shared-samplers/src/lightTree.ts:
 *   buildSubtree (median split on the widest centroid axis, ties by emitter
 *   index; by descending power when all centroids lie within 1e-4)   :350-454
 *   mergeCones (Conty Estevez & Kulla 2018 cone union)                 :250-307
 *   packLightTreeForGPU (16 floats per node)                           :611-737
 *   conservativeConeCosineThreshold / representedLightTreePower        :193-224
 *   packedDist2ToAabbCPU / packedConeFactorCPU /
 *   packedNodeImportanceUnchecked (every stage rounded to f32)         :938-1151
 *   allocateLeftBuckets / samplePackedLightTreeCPU /
 *   packedLightTreePdfCPU (24-bit bucket descent, exact PMF)           :1177-1408
 * (orc_lt_sample / orc_lt_pdf exactly so; orc_lt_select, the integrator's
 * selection, reserves more buckets per leaf and keeps distant lights outside).
 * The JS Math.fround(Math.log2(x)) and 2 ** x stages are (float)log2((double)x)
 * and (float)exp2((double)x) here.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LT_FLOATS 16
#define LT_BUCKETS 16777216u
#define LT_PI 3.14159265358979323846
#define F32_MAX 3.4028234663852886e38f
#define F32_MIN_NORMAL 1.1754943508222875e-38f

typedef struct { double axis[3], theta_o, theta_e; } lt_cone;
typedef struct { int emitter; double power, c[3], mn[3], mx[3]; lt_cone cone; } lt_item;
typedef struct { int emitter, left, right; double power, mn[3], mx[3]; lt_cone cone; } lt_node;

static const lt_cone LT_FULL = {{0, 0, 0}, LT_PI, LT_PI};

static double lt_vlen(const double* v) {
  double s = fmax(fabs(v[0]), fmax(fabs(v[1]), fabs(v[2])));
  if (s == 0.0) return 0.0;
  double x = v[0] / s, y = v[1] / s, z = v[2] / s;
  return s * sqrt(x * x + y * y + z * z);
}

static lt_cone lt_merge(lt_cone a, lt_cone b) {
  double la = lt_vlen(a.axis), lb = lt_vlen(b.axis);
  if (la == 0.0 || lb == 0.0 || a.theta_o >= LT_PI || b.theta_o >= LT_PI) {
    lt_cone r = {{0, 0, 0}, LT_PI, fmin(LT_PI, fmax(a.theta_e, b.theta_e))};
    return r;
  }
  lt_cone A = a, B = b;
  if (B.theta_o > A.theta_o) { A = b; B = a; }
  double lA = lt_vlen(A.axis), lB = lt_vlen(B.axis);
  double ax[3] = {A.axis[0] / lA, A.axis[1] / lA, A.axis[2] / lA};
  double bx[3] = {B.axis[0] / lB, B.axis[1] / lB, B.axis[2] / lB};
  double cd = fmax(-1.0, fmin(1.0, ax[0] * bx[0] + ax[1] * bx[1] + ax[2] * bx[2]));
  double dth = acos(cd);
  double te = fmin(LT_PI, fmax(A.theta_e, B.theta_e));
  if (fmin(dth + B.theta_o, LT_PI) <= A.theta_o) {
    lt_cone r = {{ax[0], ax[1], ax[2]}, A.theta_o, te};
    return r;
  }
  double to = (A.theta_o + dth + B.theta_o) * 0.5;
  if (to >= LT_PI) { lt_cone r = {{0, 0, 0}, LT_PI, te}; return r; }
  double rot = to - A.theta_o;
  double t[3] = {bx[0] - cd * ax[0], bx[1] - cd * ax[1], bx[2] - cd * ax[2]};
  double tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  if (tl < 1e-8) { lt_cone r = {{0, 0, 0}, LT_PI, te}; return r; }
  for (int k = 0; k < 3; ++k) t[k] /= tl;
  double cr = cos(rot), sr = sin(rot);
  lt_cone r = {{ax[0] * cr + t[0] * sr, ax[1] * cr + t[1] * sr, ax[2] * cr + t[2] * sr}, to, te};
  return r;
}

static int g_sort_axis;
static int cmp_centroid(const void* pa, const void* pb) {
  const lt_item* a = (const lt_item*)pa;
  const lt_item* b = (const lt_item*)pb;
  double d = a->c[g_sort_axis] - b->c[g_sort_axis];
  if (d < 0) return -1;
  if (d > 0) return 1;
  return (a->emitter > b->emitter) - (a->emitter < b->emitter);
}
static int cmp_power_desc(const void* pa, const void* pb) {
  const lt_item* a = (const lt_item*)pa;
  const lt_item* b = (const lt_item*)pb;
  double d = b->power - a->power;
  if (d < 0) return -1;
  if (d > 0) return 1;
  return (a->emitter > b->emitter) - (a->emitter < b->emitter);
}

static int lt_build(const lt_item* items, long n, lt_node* nodes, long* count) {
  int idx = (int)(*count)++;
  lt_node* nd = &nodes[idx];
  memset(nd, 0, sizeof *nd);
  nd->left = nd->right = -1;
  nd->emitter = -1;
  if (n == 1) {
    nd->emitter = items[0].emitter;
    nd->power = items[0].power;
    memcpy(nd->mn, items[0].mn, sizeof nd->mn);
    memcpy(nd->mx, items[0].mx, sizeof nd->mx);
    nd->cone = items[0].cone;
    return idx;
  }
  double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) { cmn[k] = fmin(cmn[k], items[i].c[k]); cmx[k] = fmax(cmx[k], items[i].c[k]); }
  double sx = cmx[0] - cmn[0], sy = cmx[1] - cmn[1], sz = cmx[2] - cmn[2];
  lt_item* sorted = (lt_item*)malloc(sizeof(lt_item) * (size_t)n);
  memcpy(sorted, items, sizeof(lt_item) * (size_t)n);
  if (fmax(sx, fmax(sy, sz)) < 1e-4) {
    qsort(sorted, (size_t)n, sizeof(lt_item), cmp_power_desc);
  } else {
    g_sort_axis = (sx >= sy && sx >= sz) ? 0 : (sy >= sz ? 1 : 2);
    qsort(sorted, (size_t)n, sizeof(lt_item), cmp_centroid);
  }
  long mid = n / 2;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY}, total = 0.0;
  for (long i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) { mn[k] = fmin(mn[k], items[i].mn[k]); mx[k] = fmax(mx[k], items[i].mx[k]); }
    total += items[i].power;
  }
  int l = lt_build(sorted, mid, nodes, count);
  int r = lt_build(sorted + mid, n - mid, nodes, count);
  free(sorted);
  nd = &nodes[idx];
  nd->power = total;
  memcpy(nd->mn, mn, sizeof mn);
  memcpy(nd->mx, mx, sizeof mx);
  nd->left = l;
  nd->right = r;
  nd->cone = lt_merge(nodes[l].cone, nodes[r].cone);
  return idx;
}

static float lt_next_down(float v) {
  if (isnan(v) || v == -INFINITY) return v;
  if (v == 0.0f) return -1.40129846e-45f;
  uint32_t b;
  memcpy(&b, &v, 4);
  b = v > 0.0f ? b - 1u : b + 1u;
  memcpy(&v, &b, 4);
  return v;
}
static float lt_cone_cos(double angle) {
  float r = (float)cos(fmin(LT_PI, angle)), t = r;
  for (int s = 0; s < 64; ++s) t = lt_next_down(t);
  float a = (float)((double)r - 3.814697265625e-06);
  return fmaxf(-1.0f, fminf(t, a));
}

/*
 * Build and pack.  Per emitter: power, centroid xyz, aabb (min xyz, max xyz),
 * cone (axis xyz, thetaO, thetaE, oriented flag).  Returns the node count
 * (out holds 16 floats per node; cap in nodes), or -1.
 */
long orc_lt_build(const double* power, const double* centroid, const double* aabb, const double* cone, long n,
                  float* out, long cap) {
  if (n <= 0 || 2 * n - 1 > cap) return -1;
  lt_item* items = (lt_item*)calloc((size_t)n, sizeof(lt_item));
  for (long i = 0; i < n; ++i) {
    items[i].emitter = (int)i;
    items[i].power = power[i];
    for (int k = 0; k < 3; ++k) {
      items[i].c[k] = centroid[3 * i + k];
      items[i].mn[k] = aabb[6 * i + k];
      items[i].mx[k] = aabb[6 * i + 3 + k];
    }
    const double* c = cone + 6 * i;
    double l = lt_vlen(c);
    if (c[5] == 0.0 || l == 0.0) {
      items[i].cone = LT_FULL;
    } else {
      lt_cone q = {{c[0] / l, c[1] / l, c[2] / l}, c[3], fmin(LT_PI, c[4])};
      items[i].cone = q;
    }
  }
  lt_node* nodes = (lt_node*)calloc((size_t)(2 * n), sizeof(lt_node));
  long count = 0;
  lt_build(items, n, nodes, &count);
  double maxp = 0.0;
  for (long i = 0; i < count; ++i) maxp = fmax(maxp, nodes[i].power);
  for (long i = 0; i < count; ++i) {
    const lt_node* nd = &nodes[i];
    float* o = out + LT_FLOATS * i;
    o[0] = (float)nd->emitter;
    float rp = 0.0f;
    if (nd->power > 0.0 && maxp > 0.0) {
      double ratio = nd->power / maxp;
      rp = ratio > 0.0 ? (float)ratio : F32_MIN_NORMAL;
      if (!(rp > F32_MIN_NORMAL)) rp = F32_MIN_NORMAL;
    }
    o[1] = rp;
    o[2] = (float)nd->left;
    o[3] = (float)nd->right;
    for (int k = 0; k < 3; ++k) { o[4 + k] = (float)nd->mn[k]; o[7 + k] = (float)nd->mx[k]; }
    double al = lt_vlen(nd->cone.axis);
    for (int k = 0; k < 3; ++k) o[10 + k] = al > 0.0 ? (float)(nd->cone.axis[k] / al) : 0.0f;
    o[13] = lt_cone_cos(nd->cone.theta_o);
    o[14] = lt_cone_cos(nd->cone.theta_o + nd->cone.theta_e);
  }
  for (long i = count - 1; i >= 0; --i) {
    float* o = out + LT_FLOATS * i;
    o[15] = nodes[i].left < 0 ? 1.0f : out[LT_FLOATS * nodes[i].left + 15] + out[LT_FLOATS * nodes[i].right + 15];
  }
  free(items);
  free(nodes);
  return count;
}

/* Cone of a group: the parts' cones (6 doubles each as above) merged in order. */
void orc_lt_merge_cones(const double* cones, long n, double* out6) {
  lt_cone c = LT_FULL;
  for (long i = 0; i < n; ++i) {
    const double* q = cones + 6 * i;
    double l = lt_vlen(q);
    lt_cone x = LT_FULL;
    if (q[5] != 0.0 && l != 0.0) { lt_cone y = {{q[0] / l, q[1] / l, q[2] / l}, q[3], fmin(LT_PI, q[4])}; x = y; }
    c = i == 0 ? x : lt_merge(c, x);
  }
  int oriented = lt_vlen(c.axis) > 0.0 && c.theta_o < LT_PI;
  for (int k = 0; k < 3; ++k) out6[k] = oriented ? c.axis[k] : 0.0;
  out6[3] = c.theta_o;
  out6[4] = c.theta_e;
  out6[5] = oriented ? 1.0 : 0.0;
}

/* ---- f32 importance ---- */
static float flog2(float a) { return (float)log2((double)a); }
static float fexp2(float a) { return (float)exp2((double)a); }
static float fdot(float ax, float ay, float az, float bx, float by, float bz) {
  float x = ax * bx, y = ay * by, z = az * bz;
  float s = x + y;
  return s + z;
}
static float fmax3a(float a, float b, float c) { return fmaxf(fabsf(a), fmaxf(fabsf(b), fabsf(c))); }

static float lt_dist2(float px, float py, float pz, const float* b) {
  float hx = fmaxf(fmaxf(0.5f * b[0] - 0.5f * px, 0.0f), 0.5f * px - 0.5f * b[3]);
  float hy = fmaxf(fmaxf(0.5f * b[1] - 0.5f * py, 0.0f), 0.5f * py - 0.5f * b[4]);
  float hz = fmaxf(fmaxf(0.5f * b[2] - 0.5f * pz, 0.0f), 0.5f * pz - 0.5f * b[5]);
  float hs = fmax3a(hx, hy, hz);
  if (!(hs >= F32_MIN_NORMAL)) return 0.0f;
  if (hs > 0.5f * F32_MAX) return F32_MAX;
  float sx = hx / hs, sy = hy / hs, sz = hz / hs;
  float ss = fdot(sx, sy, sz, sx, sy, sz);
  float s = 2.0f * hs;
  float lim = sqrtf(F32_MAX / ss);
  if (s >= lim) return F32_MAX;
  float r = (s * s) * ss;
  return fminf(F32_MAX, r);
}

static float lt_cone_factor(const float* n, float px, float py, float pz) {
  float axs = fmax3a(n[10], n[11], n[12]);
  if (!(axs > 0.0f) || axs > F32_MAX) return 1.0f;
  float ax = n[10] / axs, ay = n[11] / axs, az = n[12] / axs;
  float al = sqrtf(fdot(ax, ay, az, ax, ay, az));
  const float *mn = n + 4, *mx = n + 7;
  float dvx = (0.5f * px - 0.25f * mn[0]) - 0.25f * mx[0];
  float dvy = (0.5f * py - 0.25f * mn[1]) - 0.25f * mx[1];
  float dvz = (0.5f * pz - 0.25f * mn[2]) - 0.25f * mx[2];
  float rx = 0.25f * mx[0] - 0.25f * mn[0], ry = 0.25f * mx[1] - 0.25f * mn[1], rz = 0.25f * mx[2] - 0.25f * mn[2];
  float ds = fmax3a(dvx, dvy, dvz);
  if (!(ds >= F32_MIN_NORMAL) || ds > F32_MAX) return 1.0f;
  float sdx = dvx / ds, sdy = dvy / ds, sdz = dvz / ds;
  float sdl = sqrtf(fdot(sdx, sdy, sdz, sdx, sdy, sdz));
  float rs = fmax3a(rx, ry, rz), rod = 0.0f;
  if (rs >= F32_MIN_NORMAL) {
    float srx = rx / rs, sry = ry / rs, srz = rz / rs;
    float srl = sqrtf(fdot(srx, sry, srz, srx, sry, srz));
    float lr = ((flog2(rs) + flog2(srl)) - flog2(ds)) - flog2(sdl);
    if (lr >= 0.0f) return 1.0f;
    rod = fexp2(fmaxf(lr, -126.0f));
  }
  float dx = sdx / sdl, dy = sdy / sdl, dz = sdz / sdl;
  float nx = ax / al, ny = ay / al, nz = az / al;
  float ct = fmaxf(-1.0f, fminf(1.0f, fdot(nx, ny, nz, dx, dy, dz)));
  float stu = fmaxf(0.0f, fminf(1.0f, rod));
  float ctu = sqrtf(fmaxf(0.0f, 1.0f - stu * stu));
  float ca = 1.0f;
  if (ct < ctu) {
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float a = ct * ctu, b = st * stu;
    ca = fmaxf(-1.0f, fminf(1.0f, a + b));
  }
  if (ca < n[14]) return 0.0f;
  if (ca >= n[13]) return 1.0f;
  float span = n[13] - n[14];
  if (!(span > 0.0f)) return 1.0f;
  return fmaxf(F32_MIN_NORMAL, fminf(1.0f, (ca - n[14]) / span));
}

/*
 * The integrator's importance (device light_tree.cuh importance()): the same
 * quantity as orc_lt_importance -- power / max(dist^2 to the box, floor) times
 * the orientation cone's bound -- times the receiver term for the unit normal
 * nrm (Conty Estevez & Kulla 2018's bound cos(max(0, theta_i - theta_u)) on
 * the shading cosine; NULL or zero: none), evaluated directly in f32 rather
 * than in the reference's scale-safe log form: one reciprocal square root
 * serves both bounds, and the packed cone axis is unit (the build normalises
 * it).  Each operation is rounded on its own, as on the device.
 */
static float lt_bound_cos(float c, float cu, float su) {
  if (c >= cu) return 1.0f;
  float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
  float a = c * cu, b = s * su;
  return fmaxf(-1.0f, fminf(1.0f, a + b));
}

float orc_lt_importance_direct(const float* tree, long idx, const float* p, const float* nrm, float floor_d2) {
  const float* n = tree + LT_FLOATS * idx;
  float power = n[1];
  if (!(power > 0.0f)) return 0.0f;
  const float *mn = n + 4, *mx = n + 7;
  float ex = fmaxf(fmaxf(mn[0] - p[0], 0.0f), p[0] - mx[0]);
  float ey = fmaxf(fmaxf(mn[1] - p[1], 0.0f), p[1] - mx[1]);
  float ez = fmaxf(fmaxf(mn[2] - p[2], 0.0f), p[2] - mx[2]);
  float d2 = fmaxf(fdot(ex, ey, ez, ex, ey, ez), floor_d2);
  float vx = p[0] - 0.5f * (mn[0] + mx[0]), vy = p[1] - 0.5f * (mn[1] + mx[1]), vz = p[2] - 0.5f * (mn[2] + mx[2]);
  float hx = 0.5f * (mx[0] - mn[0]), hy = 0.5f * (mx[1] - mn[1]), hz = 0.5f * (mx[2] - mn[2]);
  float r2 = fdot(hx, hy, hz, hx, hy, hz), l2 = fdot(vx, vy, vz, vx, vy, vz);
  float w = 1.0f;
  if (l2 > r2 && l2 <= F32_MAX) { /* p outside the bounding sphere */
    float inv = (float)(1.0 / sqrt((double)l2));
    float su = fminf(1.0f, sqrtf(r2) * inv);
    float cu = sqrtf(fmaxf(0.0f, 1.0f - su * su));
    if (n[10] != 0.0f || n[11] != 0.0f || n[12] != 0.0f) {
      float ca = lt_bound_cos(fmaxf(-1.0f, fminf(1.0f, fdot(n[10], n[11], n[12], vx, vy, vz) * inv)), cu, su);
      if (ca < n[14]) return 0.0f;
      if (ca < n[13]) {
        float span = n[13] - n[14];
        if (span > 0.0f) w = fmaxf(F32_MIN_NORMAL, (ca - n[14]) / span);
      }
    }
    if (nrm && (nrm[0] != 0.0f || nrm[1] != 0.0f || nrm[2] != 0.0f)) {
      float ci = lt_bound_cos(fmaxf(-1.0f, fminf(1.0f, -(fdot(nrm[0], nrm[1], nrm[2], vx, vy, vz) * inv))), cu, su);
      if (!(ci > 0.0f)) return 0.0f;
      w = w * ci;
    }
  }
  float imp = (power * w) / d2;
  if (!(imp <= F32_MAX)) return F32_MAX;
  return fmaxf(F32_MIN_NORMAL, imp);
}

float orc_lt_importance(const float* tree, long idx, const float* p, float floor_d2) {
  const float* n = tree + LT_FLOATS * idx;
  float power = n[1];
  if (!(power > 0.0f)) return 0.0f;
  float d2 = fmaxf(fmaxf(lt_dist2(p[0], p[1], p[2], n + 4), floor_d2), F32_MIN_NORMAL);
  float cone = lt_cone_factor(n, p[0], p[1], p[2]);
  if (!(cone > 0.0f)) return 0.0f;
  float li = (flog2(power) - flog2(d2)) + flog2(fmaxf(cone, F32_MIN_NORMAL));
  if (li >= 127.99999f) return F32_MAX;
  if (li <= -126.0f) return F32_MIN_NORMAL;
  return fmaxf(F32_MIN_NORMAL, fminf(F32_MAX, fexp2(li)));
}

static uint32_t lt_left_buckets(uint32_t cur, uint32_t ll, uint32_t rl, float a, float b, uint32_t reserve) {
  ll *= reserve;
  rl *= reserve;
  uint32_t remaining = cur - (ll + rl);
  float pl = 0.5f;
  if (!(a == 0.0f && b == 0.0f)) {
    float s = fmaxf(a, b), l = a / s, r = b / s;
    pl = l / (l + r);
  }
  float ideal = (float)remaining * pl;
  float extra = floorf(ideal + 0.5f);
  uint32_t e = extra <= 0.0f ? 0u : (uint32_t)fminf(extra, (float)remaining);
  return ll + (e > remaining ? remaining : e);
}

/* direct: the integrator's importance (orc_lt_importance_direct with nrm), else the reference's */
static float lt_descend(const float* tree, long nodes, const float* p, const float* nrm, int direct, float floor_d2,
                        uint32_t cur, uint32_t bucket, uint32_t reserve, int* emitter) {
  long node = 0;
  *emitter = -1;
  for (long guard = 0; guard <= nodes; ++guard) {
    const float* n = tree + LT_FLOATS * node;
    if (n[2] < 0.0f) {
      *emitter = (int)n[0];
      return (float)cur / (float)LT_BUCKETS;
    }
    long l = (long)n[2], r = (long)n[3];
    float il = direct ? orc_lt_importance_direct(tree, l, p, nrm, floor_d2) : orc_lt_importance(tree, l, p, floor_d2);
    float ir = direct ? orc_lt_importance_direct(tree, r, p, nrm, floor_d2) : orc_lt_importance(tree, r, p, floor_d2);
    uint32_t lb = lt_left_buckets(cur, (uint32_t)tree[LT_FLOATS * l + 15], (uint32_t)tree[LT_FLOATS * r + 15], il, ir,
                                  reserve);
    if (bucket < lb) { cur = lb; node = l; }
    else { bucket -= lb; cur -= lb; node = r; }
  }
  return 0.0f;
}

/* Entry for point p from the 24-bit draw `bucket`; returns its PMF (0: none). */
float orc_lt_sample(const float* tree, long nodes, const float* p, float floor_d2, uint32_t bucket, int* emitter) {
  *emitter = -1;
  if (nodes <= 0) return 0.0f;
  return lt_descend(tree, nodes, p, NULL, 0, floor_d2, LT_BUCKETS, bucket, 1u, emitter);
}

/*
 * The integrator's selection: entries 0 .. n_pos-1 by the tree over the
 * positional entries (tree NULL: a single one), entries n_pos .. n_pos+n_dist-1
 * (distant lights) evenly within n_dist / (n_dist + 1) of the 2^24 buckets.
 * In the tree's descent every leaf keeps a defensive reserve of half the
 * tree's buckets split evenly (the reference keeps one bucket per leaf); the
 * other half follows orc_lt_importance_direct for the unit normal nrm (NULL
 * or zero: no receiver term).
 */
float orc_lt_select(const float* tree, long nodes, uint32_t n_pos, uint32_t n_dist, const float* p, const float* nrm,
                    float floor_d2, uint32_t bucket, int* emitter) {
  uint32_t D = n_dist == 0 ? 0u : (n_pos == 0 ? LT_BUCKETS : (uint32_t)(((uint64_t)LT_BUCKETS * n_dist) / (n_dist + 1u)));
  *emitter = -1;
  if (bucket < D) {
    uint32_t j = (uint32_t)(((uint64_t)bucket * n_dist) / D);
    uint64_t lo = ((uint64_t)j * D + n_dist - 1u) / n_dist, hi = ((uint64_t)(j + 1u) * D + n_dist - 1u) / n_dist;
    *emitter = (int)(n_pos + j);
    return (float)(hi - lo) / (float)LT_BUCKETS;
  }
  if (n_pos == 0) return 0.0f;
  if (!tree || nodes <= 1) { *emitter = 0; return (float)(LT_BUCKETS - D) / (float)LT_BUCKETS; }
  /* defensive half: each leaf keeps (buckets / 2) / leaves of the tree's buckets */
  uint32_t reserve = (LT_BUCKETS - D) / (2u * (uint32_t)tree[15]);
  if (reserve < 1u) reserve = 1u;
  return lt_descend(tree, nodes, p, nrm, 1, floor_d2, LT_BUCKETS - D, bucket - D, reserve, emitter);
}

/* PMF of one emitter at point p (the deterministic inverse of orc_lt_sample). */
float orc_lt_pdf(const float* tree, long nodes, const float* p, float floor_d2, int emitter) {
  if (nodes <= 0 || emitter < 0) return 0.0f;
  uint8_t* contains = (uint8_t*)calloc((size_t)nodes, 1);
  for (long i = nodes - 1; i >= 0; --i) {
    const float* n = tree + LT_FLOATS * i;
    contains[i] = n[2] < 0.0f ? (n[0] == (float)emitter) : (contains[(long)n[2]] || contains[(long)n[3]]);
  }
  float out = 0.0f;
  if (contains[0]) {
    long node = 0;
    uint32_t cur = LT_BUCKETS;
    for (long guard = 0; guard <= nodes; ++guard) {
      const float* n = tree + LT_FLOATS * node;
      if (n[2] < 0.0f) { out = n[0] == (float)emitter ? (float)cur / (float)LT_BUCKETS : 0.0f; break; }
      long l = (long)n[2], r = (long)n[3];
      uint32_t lb = lt_left_buckets(cur, (uint32_t)tree[LT_FLOATS * l + 15], (uint32_t)tree[LT_FLOATS * r + 15],
                                    orc_lt_importance(tree, l, p, floor_d2), orc_lt_importance(tree, r, p, floor_d2),
                                    1u);
      if (contains[l]) { cur = lb; node = l; }
      else { cur -= lb; node = r; }
    }
  }
  free(contains);
  return out;
}
