/* Plain-C restatement of the reference renderer's path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load this (oracle/_port/libxyzport.so); the CUDA product
 * never does.  It is pinned to the reference itself: tests compare it with the
 * reference's own code compiled from its sources (oracle/_ref, ref_harness.cpp)
 * and with golden fixtures generated from that build (tests/golden/).
 *
 * What it restates, step for step and with the reference's float/double
 * promotions (hi::basic_vector3 arithmetic promotes float x double to double,
 * libhi/hi/math/vector3.hpp:75-94, promote_traits.hpp:45-50):
 *   kd-tree build     KDTree::Build           xyz/geom/kdtree.cpp:207-357
 *   kd-tree traversal KDNode/KDLeaf/KDTree    xyz/geom/kdtree.cpp:82-150,366-372
 *   ray/triangle      FindIntersectionDF      xyz/geom/triangle.cpp:127-165
 *   shading basis     Triangle::ShadingBasis  xyz/geom/triangle.cpp:194-219
 *   light sampling    Scene::SampleLightPosition xyz/core/scene.cpp:42-78,
 *                     Triangle::Sample        xyz/geom/triangle.cpp:232-263
 *   camera            ThinLensCamera          xyz/core/thinlenscamera.cpp:71-205
 *   estimator         Scene::EvalutePathTracing xyz/core/scene_pathtracing.cpp:11-144
 *   NEE               Lambert::CalculateWeightedDirectLighting xyz/bsdf/lambert.cpp:125-173
 *   BSDF sampling     Lambert::NextScatteringDirection xyz/bsdf/lambert.cpp:176-187,
 *                     ComputeDiffusedVector   xyz/stdafx.hpp:50-63
 *   film              PathTracer::run         xyz/integrator/integrator.cpp:119-128
 *
 * Random numbers: the Philox stream of philox.h, read in the order the
 * reference consumes IPrimarySample::next() when built with g++.  g++ evaluates
 * the two `sample.next()` arguments of SampleLightPosition,
 * SampleLensPosition and ComputeDiffusedVector right to left, so the first draw
 * feeds the second parameter.
 *
 * Extensions beyond the reference (off by default, used to check the CUDA
 * path's options): `rr_start` (first vertex index that plays Russian roulette;
 * the reference plays it from vertex 1), a run-time pinhole switch (the
 * reference selects it at compile time, CONFIG_PINHOLE_CAMERA_MODEL), and a
 * per-material emission scale of the light power (1 = the reference).
 *
 * Gradients (xyzo_adjoint): for the differentiable-rendering check, every
 * contribution C = Phi * e * prod_j albedo_j * r * w of a path (r the Russian
 * roulette scale, w the geometric / MIS weight) is differentiated directly:
 * dC/d albedo_j = C without albedo_j's factor (product of the others), dC/de =
 * C at e = 1.  This per-contribution form is independent of the CUDA adjoint's
 * suffix-sum replay.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "philox.h"

#define XYZO_EPSILON 1e-6f                 /* xyz/stdafx.hpp:36 */
#define XYZO_TMIN 1e-5f                    /* xyz/geom/intersection.hpp:12 */
#define XYZO_M_1_PI 0.318309886183790671538 /* M_1_PI (double) */
#define XYZO_M_PI 3.14159265358979323846

typedef struct {
  float x, y, z;
} f3;

static inline f3 mk(float x, float y, float z) {
  f3 r = {x, y, z};
  return r;
}
static inline float at3(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
static inline f3 add3(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub3(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 mul3(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline f3 scale3(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline f3 neg3(f3 a) { return mk(-a.x, -a.y, -a.z); }
/* hi::dot (vector3.hpp:120): a0*b0 + a1*b1 + a2*b2, left to right. */
static inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* hi::cross (vector3.hpp:126-131). */
static inline f3 cross3(f3 a, f3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* hi::normalize = a * rsqrt(length_squared(a)), rsqrt = 1/sqrt (math.hpp:155). */
static inline f3 normalize3(f3 a) {
  float const r = 1.0f / sqrtf(dot3(a, a));
  return scale3(a, r);
}

/* ------------------------------------------------------------------ scene */
typedef struct {
  int nt, nm, nl;
  f3 *v0, *e1, *e2, *ng, *n0, *s1, *s2;
  int *mat;
  f3 *albedo;
  int *is_light;
  int *lights;   /* light triangle ids in triangle order */
  float *cdf;    /* nl + 1 entries, cdf[0] = 0 */
  f3 power;      /* Phi, XYZ */
  float *spd;    /* 31 albedo bins per material (spectral estimator), or NULL */
  float *emission; /* per-material emission scale, or NULL (all 1) */
  float light_spd[31];
  /* kd-tree (reference structure: interior / leaf / null nodes) */
  int nnodes, cap_nodes;
  int *kaxis;    /* 0..2 interior, -1 leaf, -2 null */
  float *kvalue;
  int *kchild;   /* 2 per node */
  int *kbegin, *kcount;
  int *refs;
  int nrefs, cap_refs, kmaxdepth_seen;
  f3 kmin, kmax;
  size_t max_bucket, max_depth;
} scene_t;

typedef struct {
  f3 eye, at;
  float film, focal, fnum, aspect;
  float L, V, R;
  f3 right, up, back;
  int pinhole, W, H;
} camera_t;

static scene_t S;
static camera_t CAM;
static size_t KMAX = 16;
static float RR_THRESHOLD = 0.2f;
static int RR_START = 1;

/* Triangle::min(k)/max(k) without cached bounds (triangle.hpp:142-156). */
static inline float tmin_k(int i, int k) {
  float a = at3(S.v0[i], k), b = a + at3(S.e1[i], k), c = a + at3(S.e2[i], k);
  float m = a;
  if (b < m) m = b;
  if (c < m) m = c;
  return m;
}
static inline float tmax_k(int i, int k) {
  float a = at3(S.v0[i], k), b = a + at3(S.e1[i], k), c = a + at3(S.e2[i], k);
  float m = a;
  if (b > m) m = b;
  if (c > m) m = c;
  return m;
}

/* ---------------------------------------------------------- kd-tree build */
typedef struct {
  int type; /* 0 open, 1 close */
  float value;
} event_t;

static int event_cmp(const void *pa, const void *pb) {
  const event_t *a = (const event_t *)pa, *b = (const event_t *)pb;
  if (a->value < b->value) return -1;
  if (a->value > b->value) return 1;
  return a->type - b->type; /* open < close on ties */
}

static int new_node(void) {
  if (S.nnodes == S.cap_nodes) {
    S.cap_nodes = S.cap_nodes ? 2 * S.cap_nodes : 1024;
    S.kaxis = (int *)realloc(S.kaxis, sizeof(int) * S.cap_nodes);
    S.kvalue = (float *)realloc(S.kvalue, sizeof(float) * S.cap_nodes);
    S.kchild = (int *)realloc(S.kchild, sizeof(int) * 2 * S.cap_nodes);
    S.kbegin = (int *)realloc(S.kbegin, sizeof(int) * S.cap_nodes);
    S.kcount = (int *)realloc(S.kcount, sizeof(int) * S.cap_nodes);
  }
  int n = S.nnodes++;
  S.kaxis[n] = -2;
  S.kvalue[n] = 0;
  S.kchild[2 * n] = S.kchild[2 * n + 1] = -1;
  S.kbegin[n] = S.kcount[n] = 0;
  return n;
}

static int add_leaf(const int *set, int n) {
  int node = new_node();
  if (n == 0) return node; /* KDNull */
  if (S.nrefs + n > S.cap_refs) {
    while (S.nrefs + n > S.cap_refs) S.cap_refs = S.cap_refs ? 2 * S.cap_refs : 4096;
    S.refs = (int *)realloc(S.refs, sizeof(int) * S.cap_refs);
  }
  S.kaxis[node] = -1;
  S.kbegin[node] = S.nrefs;
  S.kcount[node] = n;
  memcpy(S.refs + S.nrefs, set, sizeof(int) * n);
  S.nrefs += n;
  return node;
}

/* KDTree::Build(set, min, max, depth), xyz/geom/kdtree.cpp:226-357. */
static int build_rec(const int *set, int n, f3 bmin, f3 bmax, size_t depth) {
  if (depth > (size_t)S.kmaxdepth_seen) S.kmaxdepth_seen = (int)depth;
  if ((size_t)n <= S.max_bucket || depth > S.max_depth) return add_leaf(set, n);
  depth++;
  f3 const range = sub3(bmax, bmin);
  int axis = -1;
  float value = NAN;
  float min_cost = 3.402823466e+38f; /* numeric_limits<float>::max() */
  event_t *ev = (event_t *)malloc(sizeof(event_t) * 2 * (size_t)n);
  for (int k = 0; k < 3; ++k) {
    for (int i = 0; i < n; ++i) {
      ev[i].type = 0;
      ev[i].value = tmin_k(set[i], k);
      ev[i + n].type = 1;
      ev[i + n].value = tmax_k(set[i], k) + XYZO_EPSILON;
    }
    qsort(ev, 2 * (size_t)n, sizeof(event_t), event_cmp);
    float const a = at3(range, (k + 1) % 3) * at3(range, (k + 2) % 3);
    float const b = at3(range, (k + 1) % 3) + at3(range, (k + 2) % 3);
    size_t n_left = 0, n_right = (size_t)n;
#define XYZO_UPDATE(vv)                                                     \
  do {                                                                      \
    float const r = (vv) - at3(bmin, k);                                    \
    float const sa_left = a + b * r;                                        \
    float const sa_right = a + b * (at3(range, k) - r);                     \
    float const cost = (float)n_left * sa_left + (float)n_right * sa_right; \
    if (min_cost > cost) {                                                  \
      min_cost = cost;                                                      \
      axis = k;                                                             \
      value = (vv);                                                         \
    }                                                                       \
  } while (0)
    {
      float const v = ev[0].value - XYZO_EPSILON;
      XYZO_UPDATE(v);
    }
    size_t const size = 2 * (size_t)n;
    for (size_t i = 0; i < size; ++i) {
      if (ev[i].type) {
        n_right--;
      } else {
        n_left++;
      }
      float v = ev[i].value;
      if (i + 1 < size) {
        if (v == ev[i + 1].value) continue;
      } else {
        v += XYZO_EPSILON;
      }
      XYZO_UPDATE(v);
    }
#undef XYZO_UPDATE
  }
  free(ev);
  int *left = (int *)malloc(sizeof(int) * (size_t)n);
  int *right = (int *)malloc(sizeof(int) * (size_t)n);
  int nl = 0, nr = 0;
  for (int i = 0; i < n; ++i) {
    /* Triangle::Overlap (triangle.cpp:75-85) */
    if (tmax_k(set[i], axis) < value) {
      left[nl++] = set[i];
    } else if (value <= tmin_k(set[i], axis)) {
      right[nr++] = set[i];
    } else {
      left[nl++] = set[i];
      right[nr++] = set[i];
    }
  }
  int node = new_node();
  S.kaxis[node] = axis;
  S.kvalue[node] = value;
  f3 max_left = bmax, min_right = bmin;
  if (axis == 0) max_left.x = value, min_right.x = value;
  if (axis == 1) max_left.y = value, min_right.y = value;
  if (axis == 2) max_left.z = value, min_right.z = value;
  int c0 = build_rec(left, nl, bmin, max_left, depth);
  S.kchild[2 * node] = c0;
  free(left);
  int c1 = build_rec(right, nr, min_right, bmax, depth);
  S.kchild[2 * node + 1] = c1;
  free(right);
  return node;
}

static void kd_build(void) {
  S.nnodes = 0;
  S.nrefs = 0;
  S.kmaxdepth_seen = 0;
  f3 mn = mk(INFINITY, INFINITY, INFINITY), mx = mk(-INFINITY, -INFINITY, -INFINITY);
  for (int i = 0; i < S.nt; ++i) {
    float v;
    v = tmin_k(i, 0); if (mn.x > v) mn.x = v;
    v = tmin_k(i, 1); if (mn.y > v) mn.y = v;
    v = tmin_k(i, 2); if (mn.z > v) mn.z = v;
    v = tmax_k(i, 0); if (mx.x < v) mx.x = v;
    v = tmax_k(i, 1); if (mx.y < v) mx.y = v;
    v = tmax_k(i, 2); if (mx.z < v) mx.z = v;
  }
  mx = add3(mx, scale3(sub3(mx, mn), 1e-5f)); /* kdtree.cpp:215-216 */
  S.kmin = mn;
  S.kmax = mx;
  int *all = (int *)malloc(sizeof(int) * (size_t)(S.nt > 0 ? S.nt : 1));
  for (int i = 0; i < S.nt; ++i) all[i] = i;
  build_rec(all, S.nt, mn, mx, 0);
  free(all);
}

/* ------------------------------------------------------------- traversal */
typedef struct {
  float tmin, tmax, f, g;
  int back;
} isect_t;

/* Triangle::FindIntersectionDF, xyz/geom/triangle.cpp:127-165. */
static inline int tri_hit(int i, f3 o, f3 d, isect_t *p) {
  f3 const e2xe1 = cross3(S.e2[i], S.e1[i]);
  float const det = dot3(d, e2xe1);
  if (fabsf(det) < XYZO_EPSILON) return 0;
  float const inv_det = 1.0f / det;
  f3 const vmo = sub3(S.v0[i], o);
  float const t = inv_det * dot3(vmo, e2xe1);
  if ((t < p->tmin) || (p->tmax < t)) return 0;
  f3 const dxvmo = cross3(d, vmo);
  float const f = inv_det * dot3(S.e2[i], dxvmo);
  if ((f < 0) || (f > 1)) return 0;
  float const g = inv_det * -dot3(S.e1[i], dxvmo);
  if ((g < 0) || ((f + g) > 1)) return 0;
  p->tmax = t;
  p->f = f;
  p->g = g;
  p->back = det > 0;
  return 1;
}

static int find_rec(int node, f3 o, f3 d, isect_t *p) {
  int const ax = S.kaxis[node];
  if (ax == -2) return -1;
  if (ax == -1) {
    int s = -1;
    for (int j = 0; j < S.kcount[node]; ++j) {
      int const i = S.refs[S.kbegin[node] + j];
      if (tri_hit(i, o, d, p)) s = i;
    }
    return s;
  }
  float const v = S.kvalue[node];
  float const e = (v - at3(o, ax)) / at3(d, ax);
  int const side = at3(o, ax) < v;
  int const nearc = S.kchild[2 * node + (1 - side)];
  int const farc = S.kchild[2 * node + side];
  if ((e > p->tmax) || (e < 0)) {
    return find_rec(nearc, o, d, p);
  } else if (e < p->tmin) {
    return find_rec(farc, o, d, p);
  } else {
    float const tmax = p->tmax;
    p->tmax = e;
    int const s = find_rec(nearc, o, d, p);
    if (s >= 0) return s;
    p->tmin = e;
    p->tmax = tmax;
    return find_rec(farc, o, d, p);
  }
}

static int find_intersection(f3 o, f3 d, isect_t *p) {
  p->tmin = XYZO_TMIN;
  p->tmax = INFINITY;
  if (S.nnodes == 0) return -1;
  return find_rec(0, o, d, p);
}

/* ---------------------------------------------------------------- camera */
static void camera_reset(void) {
  f3 const view = sub3(CAM.eye, CAM.at);
  CAM.L = sqrtf(dot3(view, view));
  CAM.V = CAM.L * CAM.focal / (CAM.L - CAM.focal);
  CAM.R = CAM.focal / (2 * CAM.fnum);
  CAM.back = normalize3(view);
  CAM.right = normalize3(cross3(mk(0, 1, 0), CAM.back));
  CAM.up = cross3(CAM.back, CAM.right);
}

/* ------------------------------------------------------------- estimator */
typedef struct {
  f3 pos, sn, gn, tan, bin;
} frame_t;

/* Triangle::ShadingBasis (triangle.cpp:194-219). */
static void shading_basis(int i, float f, float g, int back, frame_t *fr) {
  f3 sn = normalize3(add3(add3(S.n0[i], scale3(S.s1[i], f)), scale3(S.s2[i], g)));
  f3 gn = S.ng[i];
  if (back) {
    gn = neg3(gn);
    sn = neg3(sn);
  }
  f3 t = mk(-sn.z, 0, sn.x);
  float const l2 = dot3(t, t);
  if (l2 > 0) {
    t = scale3(t, 1.0f / sqrtf(l2));
    fr->bin = cross3(t, sn);
  } else {
    fr->bin = mk(0, 0, (sn.y > 0) ? 1.0f : -1.0f);
    t = cross3(sn, fr->bin);
  }
  fr->tan = t;
  fr->sn = sn;
  fr->gn = gn;
}

static float light_area(void) { return S.cdf[S.nl]; }

/* float3 * double (promoted) accumulated into a float3 with per-component
 * narrowing, as `*pColor += vector3<double>` does. */
static inline void acc_d(f3 *c, double x, double y, double z) {
  c->x += (float)x;
  c->y += (float)y;
  c->z += (float)z;
}

/* Optional per-path recorder for debugging: every traced segment's ray, hit
 * triangle and kind (0 extension, 1 shadow). */
typedef struct {
  int n, cap;
  float *rays;  /* 6 per segment: origin, direction */
  int *tri, *kind;
  float *t;
} recorder_t;
static __thread recorder_t *REC = NULL;

static inline void rec_seg(f3 o, f3 d, int tri, float t, int kind) {
  if (!REC || REC->n >= REC->cap) return;
  int const i = REC->n++;
  REC->rays[6 * i + 0] = o.x;
  REC->rays[6 * i + 1] = o.y;
  REC->rays[6 * i + 2] = o.z;
  REC->rays[6 * i + 3] = d.x;
  REC->rays[6 * i + 4] = d.y;
  REC->rays[6 * i + 5] = d.z;
  REC->tri[i] = tri;
  REC->t[i] = t;
  REC->kind[i] = kind;
}

/* Gradient context of one thread (xyzo_adjoint). */
#define XYZO_MAX_VERT 1024
typedef struct {
  const float *dfilm;  /* 3 per pixel */
  double *g_alb, *g_em;
  size_t pix;
  int nv;
  int vm[XYZO_MAX_VERT];  /* materials of the vertices whose albedo is in beta */
  double r[3];            /* Russian roulette scale in beta */
} grad_t;
static __thread grad_t *GRAD = NULL;

static inline float emission_of(int m) { return S.emission ? S.emission[m] : 1.0f; }

/* Adds dfilm . dC/dparams for a contribution C_c = phi_w[c] * e * r_c * prod a_c. */
static void grad_contrib(const double phi_w[3], int light_m) {
  grad_t *g = GRAD;
  float const *df = g->dfilm + 3 * g->pix;
  double const e = (double)emission_of(light_m);
  double cu = 0;
  for (int c = 0; c < 3; ++c) {
    double prod = g->r[c];
    for (int j = 0; j < g->nv; ++j) prod *= (double)at3(S.albedo[g->vm[j]], c);
    cu += (double)df[c] * phi_w[c] * prod;
    for (int j = 0; j < g->nv; ++j) {
      double others = g->r[c] * e * phi_w[c];
      for (int i = 0; i < g->nv; ++i)
        if (i != j) others *= (double)at3(S.albedo[g->vm[i]], c);
      g->g_alb[3 * g->vm[j] + c] += (double)df[c] * others;
    }
  }
  g->g_em[light_m] += cu;
}

/* importance-driven mode (defined with the importon map below) */
#define XYZO_IMP_N 16
static int IMP_ON, IMP_BOUNCES;
static void imp_hist(f3 pos, f3 sn, f3 tan, f3 bin, float c[XYZO_IMP_N + 1]);
static float imp_density(const float c[XYZO_IMP_N + 1], f3 dir, f3 sn, f3 tan, f3 bin);

static int eval_path(int px, int py, int s, uint64_t seed, f3 *color) {
  xyzo_stream st;
  xyzo_stream_init(&st, seed, (uint32_t)(py * CAM.W + px), (uint32_t)s, 0u);
  float const jx = xyzo_stream_next(&st);
  float const jy = xyzo_stream_next(&st);
  float const x = ((float)px + jx) / (float)CAM.W;
  float const y = ((float)py + jy) / (float)CAM.H;
  *color = mk(0, 0, 0);

  /* SampleLightPosition(s = second draw, t = first draw) */
  float const lt = xyzo_stream_next(&st);
  float const ls = xyzo_stream_next(&st);
  int has_light = S.nl > 0;
  f3 lpos = mk(0, 0, 0), lsn = mk(0, 0, 0), lgn = mk(0, 0, 0);
  int lmat = 0;
  if (has_light) {
    float const u = ls * S.cdf[S.nl];
    int lo = 0, hi = S.nl + 1; /* upper_bound over cdf[0..nl] */
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (!(u < S.cdf[mid])) lo = mid + 1; else hi = mid;
    }
    int const n = lo - 1;
    float const v = (u - S.cdf[n]) / (S.cdf[n + 1] - S.cdf[n]);
    int const li = S.lights[n];
    float const ss = sqrtf(v);
    float const tt = lt;
    float const uu = ss * (1 - tt);
    float const vv = ss * tt;
    lpos = add3(add3(S.v0[li], scale3(S.e1[li], uu)), scale3(S.e2[li], vv));
    lsn = normalize3(add3(add3(S.n0[li], scale3(S.s1[li], uu)), scale3(S.s2[li], vv)));
    lgn = S.ng[li];
    lmat = S.mat[li];
  }
  f3 const lpow = S.power;
  if (GRAD) {
    GRAD->pix = (size_t)py * (size_t)CAM.W + (size_t)px;
    GRAD->nv = 0;
    GRAD->r[0] = GRAD->r[1] = GRAD->r[2] = 1.0;
  }

  /* camera vertex */
  f3 pos, dir;
  f3 beta = mk(1, 1, 1);
  int specular = 1;
  float fSamplingNext = 0;
  if (CAM.pinhole) {
    pos = CAM.eye;
    float const lx = (float)(((double)x - 0.5) * (double)CAM.film * (double)CAM.aspect);
    float const ly = (float)(((double)y - 0.5) * (double)CAM.film);
    float const lz = -CAM.V;
    dir = normalize3(add3(add3(scale3(CAM.right, lx), scale3(CAM.up, ly)), scale3(CAM.back, lz)));
  } else {
    float const ct = xyzo_stream_next(&st);
    float const cs = xyzo_stream_next(&st);
    /* SampleDisk (thinlenscamera.cpp:4-15): the angle is stored as float */
    float const radius = CAM.R * sqrtf(cs);
    float const ang = (float)((2 * XYZO_M_PI) * (double)ct);
    float const lensx = radius * cosf(ang);
    float const lensy = radius * sinf(ang);
    pos = add3(add3(CAM.eye, scale3(CAM.right, lensx)), scale3(CAM.up, lensy));
    float const fps = CAM.film * CAM.L / CAM.V;
    float const lx = (float)(((double)x - 0.5) * (double)fps * (double)CAM.aspect - (double)lensx);
    float const ly = (float)(((double)y - 0.5) * (double)fps - (double)lensy);
    float const lz = -CAM.L;
    dir = normalize3(add3(add3(scale3(CAM.right, lx), scale3(CAM.up, ly)), scale3(CAM.back, lz)));
  }

  float const A = light_area();
  for (size_t k = 1;;) {
    isect_t p;
    int const tri = find_intersection(pos, dir, &p);
    rec_seg(pos, dir, tri, tri >= 0 ? p.tmax : 0.0f, 0);
    if (tri < 0) break;
    frame_t fr;
    shading_basis(tri, p.f, p.g, p.back, &fr);
    if (-dot3(dir, fr.sn) <= 0) break;
    pos = add3(pos, scale3(dir, p.tmax));
    int const m = S.mat[tri];
    if (S.is_light[m] && !p.back) {
      f3 const pb = scale3(mul3(lpow, beta), emission_of(m));
      double wt;
      if (specular) {
        double const w = XYZO_M_1_PI / (double)A;
        acc_d(color, (double)pb.x * w, (double)pb.y * w, (double)pb.z * w);
        wt = w;
      } else {
        float const cosv = fabsf(dot3(dir, fr.sn));
        float const d2 = p.tmax * p.tmax;
        float const dimp = fSamplingNext * cosv / d2;
        float const dexp = 1.0f / A;
        float const dens = dexp / dimp;
        double const w = XYZO_M_1_PI / (double)A;
        float const mis = 1.0f / (1 + dens * dens);
        acc_d(color, (double)pb.x * w * (double)mis, (double)pb.y * w * (double)mis,
              (double)pb.z * w * (double)mis);
        wt = w * (double)mis;
      }
      if (GRAD) {
        double const pw[3] = {(double)lpow.x * wt, (double)lpow.y * wt, (double)lpow.z * wt};
        grad_contrib(pw, m);
      }
      break;
    }
    if (++k >= KMAX) break;

    /* importance-driven mode: the histogram of this Lambert vertex
     * (kNN_query, scene_importancedrivenpathtracing.cpp:121-123) */
    int const imp = IMP_ON && !S.is_light[m] && (int)k - 2 < IMP_BOUNCES;
    float ic[XYZO_IMP_N + 1];
    if (imp) imp_hist(pos, fr.sn, fr.tan, fr.bin, ic);

    /* NEE (Lambert::CalculateWeightedDirectLighting); a light's NEE is zero
     * and leaves the throughput alone (xyz/bsdf/light.cpp:18-25). */
    if (!S.is_light[m]) {
      beta = mul3(beta, S.albedo[m]);
      if (GRAD && GRAD->nv < XYZO_MAX_VERT) GRAD->vm[GRAD->nv++] = m;
    }
    if (has_light && !S.is_light[m]) {
      f3 const vin = normalize3(sub3(pos, lpos));
      float const nk3 = dot3(vin, lgn);
      if (!((nk3 <= 0) || (dot3(vin, lsn) <= 0))) {
        float const nk2 = -dot3(vin, fr.sn);
        if (!((nk2 <= 0) || (-dot3(vin, fr.gn) <= 0))) {
          isect_t q;
          int const sh = find_intersection(lpos, vin, &q);
          rec_seg(lpos, vin, sh, sh >= 0 ? q.tmax : 0.0f, 1);
          if (sh == tri) {
            float const G = nk2 * nk3 / (q.tmax * q.tmax);
            /* importance-driven: M_1_PI * G * GetDensity (lambert.cpp:210-212) */
            float const dimp = imp ? (float)(XYZO_M_1_PI * (double)G *
                                             (double)imp_density(ic, vin, fr.sn, fr.tan, fr.bin))
                                   : (float)(XYZO_M_1_PI * (double)G);
            float const dexp = 1.0f / A;
            float const dens = dimp / dexp;
            double const w =
                ((double)G * (XYZO_M_1_PI * XYZO_M_1_PI)) * (double)(1.0f / (1 + dens * dens));
            f3 const pb = scale3(mul3(lpow, beta), emission_of(lmat));
            f3 const c = mk((float)((double)pb.x * w), (float)((double)pb.y * w),
                            (float)((double)pb.z * w));
            *color = add3(*color, c);
            if (GRAD) {
              double const pw[3] = {(double)lpow.x * w, (double)lpow.y * w, (double)lpow.z * w};
              grad_contrib(pw, lmat);
            }
          }
        }
      }
    }

    /* Russian roulette */
    if ((int)k - 1 >= RR_START) {
      float const t = beta.y;
      if (t < RR_THRESHOLD) {
        float const q = t / RR_THRESHOLD;
        if (xyzo_stream_next(&st) >= q) break;
        beta = scale3(beta, 1.0f / q);
        if (GRAD)
          for (int c = 0; c < 3; ++c) GRAD->r[c] *= (double)(1.0f / q);
      }
    }

    /* Light::NextScatteringDirection ends the path (xyz/bsdf/light.cpp:27-31). */
    if (S.is_light[m]) break;

    if (imp) {
      /* Lambert::NextScatteringDirection with importons (lambert.cpp:243-257)
       * -> ImportanceQuery::SetDiffusedVector (photonmap.cpp:403-439): a bin
       * by the cumulative counts, (cos^2 theta, phi) uniform in it; the
       * throughput is divided by the bin's density. */
      float const value = ic[XYZO_IMP_N] * xyzo_stream_next(&st);
      int lo = 0, hi = XYZO_IMP_N + 1; /* upper_bound over c[0..16] */
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (!(value < ic[mid])) lo = mid + 1; else hi = mid;
      }
      int const n = lo - 1;
      int const u = n / 8, v = n % 8;
      float const mu_u = ((float)u + xyzo_stream_next(&st)) / 2;
      float const mu_v = ((float)v + xyzo_stream_next(&st)) / 8;
      float const cos_t = sqrtf(mu_u);
      float const sin_t = sqrtf(1 - mu_u);
      float const phi = (float)(2 * XYZO_M_PI) * mu_v;
      dir = add3(add3(scale3(fr.tan, sin_t * cosf(phi)), scale3(fr.bin, sin_t * sinf(phi))),
                 scale3(fr.sn, cos_t));
      float const dens = XYZO_IMP_N * (ic[n + 1] - ic[n]) / ic[XYZO_IMP_N];
      fSamplingNext = (float)((double)(dens * cos_t) * XYZO_M_1_PI);
      beta = scale3(beta, 1.0f / dens);
      specular = 0;
      if (!(dot3(dir, fr.gn) > 0)) break;
      continue;
    }

    /* Lambert::NextScatteringDirection: fMuPhi = first draw, fMuTheta = second */
    float const mu_phi = xyzo_stream_next(&st);
    float const mu_theta = xyzo_stream_next(&st);
    specular = 0;
    float const phi = (float)(2 * XYZO_M_PI) * mu_phi;
    float const cos_t = sqrtf(mu_theta);
    float const sin_t = sqrtf(1 - mu_theta);
    dir = add3(add3(scale3(fr.tan, sin_t * cosf(phi)), scale3(fr.bin, sin_t * sinf(phi))),
               scale3(fr.sn, cos_t));
    fSamplingNext = (float)(XYZO_M_1_PI * (double)cos_t);
    if (!(dot3(dir, fr.gn) > 0)) break;
  }
  return (int)st.dim;
}

/* ------------------------------------------------- spectral estimator */
/* The reference's spectral estimator, tgir::Scene::EvaluteRussianRoulette
 * (renderer/core/SceneStrategy.cpp:11-149), with H hero wavelengths and the
 * Philox stream; same geometry as eval_path.  Differences from the xyz
 * estimator, as in that source: next-event estimation (renderer/bsdf/
 * Lambert.cpp:98-137) comes before the depth cap; Russian roulette tests the
 * first wavelength's throughput; the film gets XYZ = L * 31 * CMF[bin]
 * (libhi/hi/image/spectrum.cpp:561-567).  Wavelength draw: the dimension after
 * the camera's.  mode 1: 31 equal-probability bins over 400..700 nm;
 * mode 2: 380..720 nm with basic_spectrum::Sample interpolation
 * (spectrum.cpp:148-165). */
static const double CMF_RAW[3][31] = {
    {0.014, 0.044, 0.134, 0.284, 0.348, 0.336, 0.291, 0.195, 0.096, 0.032, 0.005, 0.009, 0.063, 0.166,
     0.290, 0.433, 0.595, 0.762, 0.916, 1.026, 1.062, 1.003, 0.854, 0.642, 0.448, 0.284, 0.165, 0.087,
     0.047, 0.023, 0.011},
    {0.000, 0.001, 0.004, 0.012, 0.023, 0.038, 0.060, 0.091, 0.139, 0.208, 0.323, 0.503, 0.710, 0.862,
     0.954, 0.995, 0.995, 0.952, 0.870, 0.757, 0.631, 0.503, 0.381, 0.265, 0.175, 0.107, 0.061, 0.032,
     0.017, 0.008, 0.004},
    {0.068, 0.207, 0.646, 1.386, 1.747, 1.772, 1.669, 1.288, 0.813, 0.465, 0.272, 0.158, 0.078, 0.042,
     0.020, 0.009, 0.004, 0.002, 0.002, 0.001, 0.001, 0.000, 0.000, 0.000, 0.000, 0.000, 0.000, 0.000,
     0.000, 0.000, 0.000}};

static float cmf(int c, int i) { return (float)(CMF_RAW[c][i] / 9.80328); }

static float spd_sample(const float *t, float p) {
  p *= 31.0f;
  p -= 0.5f;
  if (p <= 0.0f) return t[0];
  if (p >= 30.0f) return t[30];
  int const k = (int)p;
  p -= (float)k;
  return t[k] + (t[k + 1] - t[k]) * p;
}

static float cmf_sample(int c, float p) {
  float t[31];
  for (int i = 0; i < 31; ++i) t[i] = cmf(c, i);
  return spd_sample(t, p);
}

typedef struct {
  int bin[4];
  float p[4];
} hero_t;

static float spd_at(const float *t, const hero_t *hs, int k, int mode) {
  return mode == 1 ? t[hs->bin[k]] : spd_sample(t, hs->p[k]);
}

static int eval_path_spectral(int px, int py, int s, uint64_t seed, int mode, int H, f3 *color) {
  xyzo_stream st;
  xyzo_stream_init(&st, seed, (uint32_t)(py * CAM.W + px), (uint32_t)s, 0u);
  float const jx = xyzo_stream_next(&st);
  float const jy = xyzo_stream_next(&st);
  float const x = ((float)px + jx) / (float)CAM.W;
  float const y = ((float)py + jy) / (float)CAM.H;
  *color = mk(0, 0, 0);
  float const lt = xyzo_stream_next(&st);
  float const ls = xyzo_stream_next(&st);
  int has_light = S.nl > 0 && S.cdf[S.nl] > 0;
  f3 lpos = mk(0, 0, 0), lsn = mk(0, 0, 0), lgn = mk(0, 0, 0);
  int lmat = 0;
  if (has_light) {
    float const u = ls * S.cdf[S.nl];
    int lo = 0, hi = S.nl + 1;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (!(u < S.cdf[mid])) lo = mid + 1; else hi = mid;
    }
    int n = lo - 1;
    if (n < 0) n = 0;
    if (n > S.nl - 1) n = S.nl - 1;
    float const v = (u - S.cdf[n]) / (S.cdf[n + 1] - S.cdf[n]);
    int const li = S.lights[n];
    float const ss = sqrtf(v), uu = ss * (1 - lt), vv = ss * lt;
    lpos = add3(add3(S.v0[li], scale3(S.e1[li], uu)), scale3(S.e2[li], vv));
    lsn = normalize3(add3(add3(S.n0[li], scale3(S.s1[li], uu)), scale3(S.s2[li], vv)));
    lgn = S.ng[li];
    lmat = S.mat[li];
  }
  f3 pos, dir;
  if (CAM.pinhole) {
    pos = CAM.eye;
    float const lx = (float)(((double)x - 0.5) * (double)CAM.film * (double)CAM.aspect);
    float const ly = (float)(((double)y - 0.5) * (double)CAM.film);
    dir = normalize3(add3(add3(scale3(CAM.right, lx), scale3(CAM.up, ly)), scale3(CAM.back, -CAM.V)));
  } else {
    float const ct = xyzo_stream_next(&st);
    float const cs = xyzo_stream_next(&st);
    float const radius = CAM.R * sqrtf(cs);
    float const ang = (float)((2 * XYZO_M_PI) * (double)ct);
    float const lensx = radius * cosf(ang), lensy = radius * sinf(ang);
    pos = add3(add3(CAM.eye, scale3(CAM.right, lensx)), scale3(CAM.up, lensy));
    float const fps = CAM.film * CAM.L / CAM.V;
    float const lx = (float)(((double)x - 0.5) * (double)fps * (double)CAM.aspect - (double)lensx);
    float const ly = (float)(((double)y - 0.5) * (double)fps - (double)lensy);
    dir = normalize3(add3(add3(scale3(CAM.right, lx), scale3(CAM.up, ly)), scale3(CAM.back, -CAM.L)));
  }
  /* hero wavelengths */
  float const uh = xyzo_stream_next(&st);
  hero_t hs;
  for (int k = 0; k < 4; ++k) {
    float u = uh + (float)k / (float)H;
    if (u >= 1.0f) u -= 1.0f;
    int b = (int)(u * 31.0f);
    hs.bin[k] = b > 30 ? 30 : b;
    float const lambda = 380.0f + 340.0f * u;
    hs.p[k] = (lambda - 395.0f) / 310.0f;
  }
  float phi[4] = {0, 0, 0, 0}, beta[4] = {1, 1, 1, 1}, L[4] = {0, 0, 0, 0};
  for (int k = 0; k < H; ++k) phi[k] = spd_at(S.light_spd, &hs, k, mode);
  int specular = 1;
  float fsn = 0;
  float const A = light_area();
  for (size_t k = 1;;) {
    isect_t p;
    int const tri = find_intersection(pos, dir, &p);
    if (tri < 0) break;
    frame_t fr;
    shading_basis(tri, p.f, p.g, p.back, &fr);
    if (-dot3(dir, fr.sn) <= 0) break;
    pos = add3(pos, scale3(dir, p.tmax));
    int const m = S.mat[tri];
    if (S.is_light[m] && !p.back) {
      double const wl = XYZO_M_1_PI / (double)A;
      double mis = 1.0;
      if (!specular) {
        float const cosv = fabsf(dot3(dir, fr.sn));
        float const dimp = fsn * cosv / (p.tmax * p.tmax);
        float const dens = (1.0f / A) / dimp;
        mis = (double)(1.0f / (1 + dens * dens));
      }
      float const e = emission_of(m);
      for (int j = 0; j < 4; ++j) L[j] += (float)((double)(phi[j] * beta[j] * e) * wl * mis);
      break;
    }
    if (!S.is_light[m]) {
      for (int j = 0; j < 4; ++j) beta[j] *= j < H ? spd_at(S.spd + 31 * m, &hs, j, mode) : 0.0f;
      if (has_light) {
        f3 const vin = normalize3(sub3(pos, lpos));
        float const nk3 = dot3(vin, lgn);
        if (!((nk3 <= 0) || (dot3(vin, lsn) <= 0))) {
          float const nk2 = -dot3(vin, fr.sn);
          if (!((nk2 <= 0) || (-dot3(vin, fr.gn) <= 0))) {
            isect_t q;
            if (find_intersection(lpos, vin, &q) == tri) {
              float const G = (nk2 * nk3) / (q.tmax * q.tmax);
              float const dimp = (float)(XYZO_M_1_PI * (double)G);
              float const dens = dimp / (1.0f / A);
              double const w = ((double)G * (XYZO_M_1_PI * XYZO_M_1_PI)) * (double)(1.0f / (1 + dens * dens));
              float const e = emission_of(lmat);
              for (int j = 0; j < 4; ++j) L[j] += (float)((double)(phi[j] * beta[j] * e) * w);
            }
          }
        }
      }
    }
    if (++k >= KMAX) break;
    if ((int)k - 1 >= RR_START) {
      float const t = beta[0];
      if (t < RR_THRESHOLD) {
        float const q = t / RR_THRESHOLD;
        if (xyzo_stream_next(&st) >= q) break;
        float const r = 1.0f / q;
        for (int j = 0; j < 4; ++j) beta[j] *= r;
      }
    }
    if (S.is_light[m]) break;
    float const mu_phi = xyzo_stream_next(&st);
    float const mu_theta = xyzo_stream_next(&st);
    specular = 0;
    float const ph = (float)(2 * XYZO_M_PI) * mu_phi;
    float const cos_t = sqrtf(mu_theta), sin_t = sqrtf(1 - mu_theta);
    dir = add3(add3(scale3(fr.tan, sin_t * cosf(ph)), scale3(fr.bin, sin_t * sinf(ph))), scale3(fr.sn, cos_t));
    fsn = (float)(XYZO_M_1_PI * (double)cos_t);
    if (!(dot3(dir, fr.gn) > 0)) break;
  }
  float const scale = mode == 1 ? 31.0f : 34.0f;
  float acc[3] = {0, 0, 0};
  for (int j = 0; j < H; ++j) {
    float const v = L[j] * scale;
    for (int c = 0; c < 3; ++c) acc[c] += v * (mode == 1 ? cmf(c, hs.bin[j]) : cmf_sample(c, hs.p[j]));
  }
  color->x = acc[0] / (float)H;
  color->y = acc[1] / (float)H;
  color->z = acc[2] / (float)H;
  return (int)st.dim;
}

/* --------------------------------------------------------------- C API */
static void free_scene(void) {
  free(S.v0); free(S.e1); free(S.e2); free(S.ng); free(S.n0); free(S.s1); free(S.s2);
  free(S.mat); free(S.albedo); free(S.is_light); free(S.lights); free(S.cdf);
  free(S.kaxis); free(S.kvalue); free(S.kchild); free(S.kbegin); free(S.kcount); free(S.refs);
  free(S.spd);
  free(S.emission);
  memset(&S, 0, sizeof(S));
}

int xyzo_scene_create(int nv, const float *pos, const float *nrm, int nt, const int *tri,
                      const int *tri_mat, int nm, const float *albedo, const int *is_light,
                      const float *power, int kd_max_bucket, int kd_max_depth) {
  free_scene();
  S.nt = nt;
  S.nm = nm;
  S.v0 = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.e1 = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.e2 = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.ng = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.n0 = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.s1 = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.s2 = (f3 *)malloc(sizeof(f3) * (size_t)(nt + 1));
  S.mat = (int *)malloc(sizeof(int) * (size_t)(nt + 1));
  S.albedo = (f3 *)malloc(sizeof(f3) * (size_t)(nm + 1));
  S.is_light = (int *)malloc(sizeof(int) * (size_t)(nm + 1));
  S.lights = (int *)malloc(sizeof(int) * (size_t)(nt + 1));
  S.cdf = (float *)malloc(sizeof(float) * (size_t)(nt + 2));
  for (int m = 0; m < nm; ++m) {
    S.albedo[m] = mk(albedo[3 * m], albedo[3 * m + 1], albedo[3 * m + 2]);
    S.is_light[m] = is_light[m] != 0;
  }
  S.cdf[0] = 0;
  S.nl = 0;
  for (int i = 0; i < nt; ++i) {
    int const a = tri[3 * i], b = tri[3 * i + 1], c = tri[3 * i + 2];
    int const m = tri_mat[i];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv || m < 0 || m >= nm) {
      free_scene();
      return -1;
    }
    f3 const p0 = mk(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
    f3 const p1 = mk(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
    f3 const p2 = mk(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
    S.v0[i] = p0;
    S.e1[i] = sub3(p1, p0);
    S.e2[i] = sub3(p2, p0);
    S.ng[i] = normalize3(cross3(S.e2[i], S.e1[i])); /* NormalVector (triangle.hpp:202) */
    if (nrm) {
      f3 const m0 = mk(nrm[3 * a], nrm[3 * a + 1], nrm[3 * a + 2]);
      f3 const m1 = mk(nrm[3 * b], nrm[3 * b + 1], nrm[3 * b + 2]);
      f3 const m2 = mk(nrm[3 * c], nrm[3 * c + 1], nrm[3 * c + 2]);
      S.n0[i] = m0;
      S.s1[i] = sub3(m1, m0);
      S.s2[i] = sub3(m2, m0);
    } else {
      S.n0[i] = S.ng[i];
      S.s1[i] = mk(0, 0, 0);
      S.s2[i] = mk(0, 0, 0);
    }
    S.mat[i] = m;
    if (S.is_light[m]) {
      f3 const cr = cross3(S.e2[i], S.e1[i]);
      float const area = sqrtf(dot3(cr, cr)) * 0.5f; /* Triangle::area */
      S.lights[S.nl] = i;
      S.cdf[S.nl + 1] = S.cdf[S.nl] + area;
      S.nl++;
    }
  }
  S.power = mk(power[0], power[1], power[2]);
  S.max_bucket = (size_t)kd_max_bucket;
  S.max_depth = (size_t)kd_max_depth;
  kd_build();
  return S.nl;
}

void xyzo_scene_destroy(void) { free_scene(); }

/* Spectral data of the current scene: 31 albedo bins per material, light SPD. */
void xyzo_scene_set_spectra(const float *albedo_spd, const float *light_spd) {
  free(S.spd);
  S.spd = (float *)malloc(sizeof(float) * 31 * (size_t)(S.nm > 0 ? S.nm : 1));
  memcpy(S.spd, albedo_spd, sizeof(float) * 31 * (size_t)S.nm);
  memcpy(S.light_spd, light_spd, sizeof(float) * 31);
}

/* Replaces the albedos (3 per material) and / or sets the per-material
 * emission scale (NULL leaves a table unchanged). */
void xyzo_set_materials(const float *albedo, const float *emission) {
  if (albedo)
    for (int m = 0; m < S.nm; ++m) S.albedo[m] = mk(albedo[3 * m], albedo[3 * m + 1], albedo[3 * m + 2]);
  if (emission) {
    if (!S.emission) S.emission = (float *)malloc(sizeof(float) * (size_t)(S.nm > 0 ? S.nm : 1));
    memcpy(S.emission, emission, sizeof(float) * (size_t)S.nm);
  }
}

static int SPEC_MODE = 0, SPEC_H = 1;
void xyzo_set_spectral(int mode, int hero) {
  SPEC_MODE = mode;
  SPEC_H = hero;
}

float xyzo_light_area(void) { return S.nl ? S.cdf[S.nl] : 0.0f; }

void xyzo_light_power_xyz(float *out) {
  out[0] = S.power.x;
  out[1] = S.power.y;
  out[2] = S.power.z;
}

void xyzo_set_path_params(int kmax, float rr_threshold, int rr_start) {
  KMAX = (size_t)kmax;
  RR_THRESHOLD = rr_threshold;
  RR_START = rr_start;
}

void xyzo_set_camera_full(const float *eye, const float *at, float film, float focal, float fnum,
                          int W, int H, int pinhole) {
  CAM.eye = mk(eye[0], eye[1], eye[2]);
  CAM.at = mk(at[0], at[1], at[2]);
  CAM.film = film;
  CAM.focal = focal;
  CAM.fnum = fnum;
  CAM.W = W;
  CAM.H = H;
  CAM.aspect = (float)W / (float)H; /* Scene::SetDimension (scene.hpp:226-230) */
  CAM.pinhole = pinhole;
  camera_reset();
}

void xyzo_set_camera(const float *eye, const float *at, float film, float focal, float fnum, int W,
                     int H) {
  xyzo_set_camera_full(eye, at, film, focal, fnum, W, H, 0);
}

float xyzo_philox_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t dim) {
  return xyzo_stream_at(seed, pixel, sample, dim);
}

/* nodes, leaves, empty leaves, leaf references, max depth, triangles */
void xyzo_kdtree_stats(int64_t *out) {
  int64_t leaves = 0, empty = 0;
  for (int i = 0; i < S.nnodes; ++i) {
    if (S.kaxis[i] == -1) leaves++;
    if (S.kaxis[i] == -2) empty++;
  }
  out[0] = S.nnodes;
  out[1] = leaves;
  out[2] = empty;
  out[3] = S.nrefs;
  out[4] = S.kmaxdepth_seen;
  out[5] = S.nt;
  out[6] = 0;
  out[7] = 0;
}

/* ------------------------------------------------------ threaded drivers */
typedef struct {
  int mode; /* 0 trace, 1 render */
  int lo, hi, chunk;
  volatile int next;
  pthread_mutex_t mu;
  /* trace */
  const float *org, *dir;
  int *tri;
  float *t, *f, *g;
  int *back;
  /* render */
  int s;
  uint64_t seed;
  float *film;
  /* adjoint: samples [s, s + spp) of rows [lo, hi), gradients summed under mu */
  int spp;
  const float *dfilm;
  double *g_alb, *g_em;
  /* pixels: samples [s, s + spp) of pixels [lo, hi) of the list px, py */
  const int *px, *py;
  double *acc;
} job_t;

static int job_take(job_t *j, int *b, int *e) {
  pthread_mutex_lock(&j->mu);
  int const x = j->next;
  j->next = x + j->chunk;
  pthread_mutex_unlock(&j->mu);
  if (x >= j->hi) return 0;
  *b = x;
  *e = x + j->chunk < j->hi ? x + j->chunk : j->hi;
  return 1;
}

static void *adjoint_worker(job_t *j) {
  size_t const na = 3 * (size_t)S.nm, ne = (size_t)S.nm;
  grad_t *g = (grad_t *)calloc(1, sizeof(grad_t));
  g->dfilm = j->dfilm;
  g->g_alb = (double *)calloc(na + 1, sizeof(double));
  g->g_em = (double *)calloc(ne + 1, sizeof(double));
  GRAD = g;
  int b, e;
  while (job_take(j, &b, &e))
    for (int y = b; y < e; ++y)
      for (int s = j->s; s < j->s + j->spp; ++s)
        for (int x = 0; x < CAM.W; ++x) {
          f3 c;
          eval_path(x, y, s, j->seed, &c);
        }
  GRAD = NULL;
  pthread_mutex_lock(&j->mu);
  for (size_t i = 0; i < na; ++i) j->g_alb[i] += g->g_alb[i];
  for (size_t i = 0; i < ne; ++i) j->g_em[i] += g->g_em[i];
  pthread_mutex_unlock(&j->mu);
  free(g->g_alb);
  free(g->g_em);
  free(g);
  return NULL;
}

static void *pixels_worker(job_t *j) {
  int b, e;
  while (job_take(j, &b, &e))
    for (int i = b; i < e; ++i) {
      double sx = 0, sy = 0, sz = 0, syy = 0;
      for (int s = j->s; s < j->s + j->spp; ++s) {
        f3 c;
        eval_path(j->px[i], j->py[i], s, j->seed, &c);
        sx += c.x;
        sy += c.y;
        sz += c.z;
        syy += (double)c.y * c.y;
      }
      double *a = j->acc + 4 * (size_t)i;
      a[0] += sx;
      a[1] += sy;
      a[2] += sz;
      a[3] += syy;
    }
  return NULL;
}

static void *job_worker(void *arg) {
  job_t *j = (job_t *)arg;
  if (j->mode == 2) return adjoint_worker(j);
  if (j->mode == 3) return pixels_worker(j);
  int b, e;
  while (job_take(j, &b, &e)) {
    for (int i = b; i < e; ++i) {
      if (j->mode == 0) {
        isect_t p;
        f3 const o = mk(j->org[3 * i], j->org[3 * i + 1], j->org[3 * i + 2]);
        f3 const d = mk(j->dir[3 * i], j->dir[3 * i + 1], j->dir[3 * i + 2]);
        int const t = find_intersection(o, d, &p);
        j->tri[i] = t;
        j->t[i] = t >= 0 ? p.tmax : 0;
        j->f[i] = t >= 0 ? p.f : 0;
        j->g[i] = t >= 0 ? p.g : 0;
        j->back[i] = t >= 0 ? p.back : 0;
      } else {
        int const y = i;
        for (int x = 0; x < CAM.W; ++x) {
          f3 c;
          if (SPEC_MODE)
            eval_path_spectral(x, y, j->s, j->seed, SPEC_MODE, SPEC_H, &c);
          else
            eval_path(x, y, j->s, j->seed, &c);
          float *fp = j->film + 3 * ((size_t)y * CAM.W + x);
          fp[0] += c.x;
          fp[1] += c.y;
          fp[2] += c.z;
        }
      }
    }
  }
  return NULL;
}

static int default_threads(int n) {
  if (n > 0) return n;
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

static void run_job(job_t *j, int nthreads) {
  nthreads = default_threads(nthreads);
  pthread_mutex_init(&j->mu, NULL);
  j->next = j->lo;
  if (nthreads == 1) {
    job_worker(j);
  } else {
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, job_worker, j);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th);
  }
  pthread_mutex_destroy(&j->mu);
}

void xyzo_trace(int n, const float *org, const float *dir, int *tri, float *t, float *f, float *g,
                int *back, int nthreads) {
  job_t j;
  memset(&j, 0, sizeof(j));
  j.mode = 0;
  j.lo = 0;
  j.hi = n;
  j.chunk = 256;
  j.org = org;
  j.dir = dir;
  j.tri = tri;
  j.t = t;
  j.f = f;
  j.g = g;
  j.back = back;
  run_job(&j, nthreads);
}

int xyzo_eval_path(int px, int py, int s, uint64_t seed, float *out) {
  f3 c;
  int const dims = SPEC_MODE ? eval_path_spectral(px, py, s, seed, SPEC_MODE, SPEC_H, &c)
                             : eval_path(px, py, s, seed, &c);
  out[0] = c.x;
  out[1] = c.y;
  out[2] = c.z;
  return dims;
}

/* eval_path with every traced segment recorded (debugging aid). */
int xyzo_eval_path_record(int px, int py, int s, uint64_t seed, float *out, int cap, float *rays,
                          int *tri, float *t, int *kind, int *n_seg) {
  recorder_t r = {0, cap, rays, tri, kind, t};
  REC = &r;
  f3 c;
  int const dims = eval_path(px, py, s, seed, &c);
  REC = NULL;
  out[0] = c.x;
  out[1] = c.y;
  out[2] = c.z;
  *n_seg = r.n;
  return dims;
}

/* PathTracer::run's loop for samples [s0, s0+spp), rows [y0, y1): film += color
 * per sample in sample order (sum, not mean). */
void xyzo_render(int s0, int spp, uint64_t seed, int y0, int y1, float *film, int nthreads) {
  for (int s = s0; s < s0 + spp; ++s) {
    job_t j;
    memset(&j, 0, sizeof(j));
    j.mode = 1;
    j.lo = y0;
    j.hi = y1;
    j.chunk = 1;
    j.s = s;
    j.seed = seed;
    j.film = film;
    run_job(&j, nthreads);
  }
}

/* Per-pixel statistics in double for reference images (test and benchmark
 * infrastructure): for each listed pixel (px[i], py[i]), the samples
 * [s0, s0 + spp) of PathTracer::run's estimator are evaluated and
 * acc[4 i .. 4 i + 3] += (sum X, sum Y, sum Z, sum Y^2), summed in double. */
void xyzo_render_pixels(int n, const int *px, const int *py, int s0, int spp, uint64_t seed, double *acc,
                        int nthreads) {
  job_t j;
  memset(&j, 0, sizeof(j));
  j.mode = 3;
  j.lo = 0;
  j.hi = n;
  j.chunk = 1;
  j.s = s0;
  j.spp = spp;
  j.seed = seed;
  j.px = px;
  j.py = py;
  j.acc = acc;
  run_job(&j, nthreads);
}

int xyzo_max_threads(void) { return default_threads(0); }

/* Gradient of sum_p dfilm[p] . film[p] (the film of xyzo_render over samples
 * [s0, s0 + spp)) with respect to the albedos (3 per material) and emission
 * scales (1 per material), added to g_alb / g_em.  XYZ estimator only. */
void xyzo_adjoint(int s0, int spp, uint64_t seed, const float *dfilm, double *g_alb, double *g_em,
                  int nthreads) {
  job_t j;
  memset(&j, 0, sizeof(j));
  j.mode = 2;
  j.lo = 0;
  j.hi = CAM.H;
  j.chunk = 1;
  j.s = s0;
  j.spp = spp;
  j.seed = seed;
  j.dfilm = dfilm;
  j.g_alb = g_alb;
  j.g_em = g_em;
  run_job(&j, nthreads);
}

/* ------------------------------------------------------------------ film output
 * CCIR601_1_XYZ2RGB (libhi/hi/image/color_space.hpp:69-79) in float. */
static void ccir601_xyz2rgb(const float xyz[3], float rgb[3]) {
  rgb[0] = 1.9104f * xyz[0] - 0.5338f * xyz[1] - 0.2891f * xyz[2];
  rgb[1] = -0.9844f * xyz[0] + 1.9985f * xyz[1] - 0.0279f * xyz[2];
  rgb[2] = 0.0585f * xyz[0] - 0.1187f * xyz[1] + 0.9017f * xyz[2];
}

/* static_cast<unsigned char>(float) as the reference's x86-64 build performs it:
 * truncation towards zero to a 32-bit integer, low byte kept. */
static unsigned char byte_of(float v) { return (unsigned char)(unsigned int)(int)v; }

/* hdr_encode (xyz/core/imagefilm_hdr.cpp:14-31). */
static void rgbe_of(const float c[3], unsigned char out[4]) {
  float d = c[0] > c[1] ? c[0] : c[1];
  d = d > c[2] ? d : c[2];
  if ((double)d <= 1e-32) {
    out[0] = out[1] = out[2] = out[3] = 0;
    return;
  }
  int e;
  float const m = frexpf(d, &e);
  float const f = (float)((double)m * 255.9999 / (double)d);
  out[0] = byte_of(c[0] * f);
  out[1] = byte_of(c[1] * f);
  out[2] = byte_of(c[2] * f);
  out[3] = (unsigned char)(e + 128);
}

/* The pixels of ImageFilm::SaveAsHdr (imagefilm_hdr.cpp:124-183) in file order:
 * film * scale, CCIR 601-1 RGB with non-finite pixels as 0, scanlines from the
 * top row down; xyze: XYZ, scanlines from the bottom row up (CONFIG_HDR_STRICT). */
void xyzo_encode_rgbe(const float *film, int W, int H, float scale, int xyze, unsigned char *out) {
  for (int row = 0; row < H; ++row) {
    int const y = xyze ? row : H - 1 - row;
    for (int x = 0; x < W; ++x) {
      const float *f = film + 3 * ((size_t)y * W + x);
      float xyz[3] = {f[0] * scale, f[1] * scale, f[2] * scale}, c[3];
      if (xyze) {
        c[0] = xyz[0], c[1] = xyz[1], c[2] = xyz[2];
      } else {
        ccir601_xyz2rgb(xyz, c);
        if (!isfinite(c[0]) || !isfinite(c[1]) || !isfinite(c[2])) c[0] = c[1] = c[2] = 0.0f;
      }
      rgbe_of(c, out + 4 * ((size_t)row * W + x));
    }
  }
}

/* tonemap() and clamp() of float2bmp/main.cpp:69-118 with the operator chosen
 * at run time (0 film 1 - exp(-e L), the tool's; 1 linear; 2 Reinhard; 3
 * Reinhard with white). */
static unsigned char tone_one(float light, int op, float exposure, float white, float gamma) {
  if (light <= 0) return 0;
  float v;
  switch (op) {
    case 1: v = exposure * light; break;
    case 2: v = exposure * light / (1 + light); break;
    case 3: v = exposure * light * (1 + light / (white * white)) / (1 + light); break;
    default: v = 1.0f - expf(-exposure * light); break;
  }
  v = powf(v, gamma);
  if (v <= 0) return 0;
  if (v >= 1) return 255;
  return (unsigned char)(v * 256);
}

/* float2bmp's image loop (main.cpp:186-214): white <= 0 takes the maximum of
 * 0.6069 c0 + 0.1735 c1 + 0.2003 c2; BGR bytes, rows from the bottom padded to
 * 4 bytes. */
void xyzo_tonemap(const float *film, int W, int H, float scale, int op, float exposure, float white,
                  float dst_gamma, float src_gamma, int rgb, unsigned char *out) {
  size_t const n = (size_t)W * H, stride = ((size_t)3 * W + 3) & ~(size_t)3;
  float const gamma = src_gamma / dst_gamma;
  if (op == 3 && !(white > 0)) {
    white = 0;
    for (size_t p = 0; p < n; ++p) {
      float c[3] = {film[3 * p] * scale, film[3 * p + 1] * scale, film[3 * p + 2] * scale};
      if (rgb) {
        float const xyz[3] = {c[0], c[1], c[2]};
        ccir601_xyz2rgb(xyz, c);
      }
      float const l = 0.6069f * c[0] + 0.1735f * c[1] + 0.2003f * c[2];
      if (white < l) white = l;
    }
  }
  for (size_t p = 0; p < n; ++p) {
    float c[3] = {film[3 * p] * scale, film[3 * p + 1] * scale, film[3 * p + 2] * scale};
    if (rgb) {
      float const xyz[3] = {c[0], c[1], c[2]};
      ccir601_xyz2rgb(xyz, c);
    }
    unsigned char *o = out + (p / W) * stride + 3 * (p % W);
    o[2] = tone_one(c[0], op, exposure, white, gamma);
    o[1] = tone_one(c[1], op, exposure, white, gamma);
    o[0] = tone_one(c[2], op, exposure, white, gamma);
  }
}

/* ------------------------------------------------ importance-driven tracing
 * The reference's importance-driven path tracer (Scene::
 * EvaluteImportanceDrivenPathTracing, xyz/core/scene_importancedrivenpathtracing
 * .cpp:11-180) with its light-importance map (Scene::CreateLightImportanceMap,
 * xyz/core/scene_photonmap.cpp:272-330) and histogram guide (ImportanceQuery,
 * xyz/core/photonmap.cpp:321-494), as the variants that act in scenes of
 * Lambert surfaces only: importons are kept at every Lambert hit from bounce
 * `min_depth` on (the source's commented `depth > 0` test; its active test
 * also wants a specular bounce first) and the histogram guides every Lambert
 * vertex of the first `guide_bounces` (the source's "[TEST]" condition).
 *
 * Particle p reads the Philox stream (pixel = p, sample = 0xffffffff): two
 * draws for the light point (as SampleLightPosition), two for a cosine
 * direction about the light's geometric normal, then per Lambert hit one
 * roulette draw (survival albedo.y, Lambert::BoundsImportance,
 * xyz/bsdf/lambert.cpp:16-42) and two for the next cosine direction about the
 * hit's geometric normal. */
#define XYZO_IMP_U 2  /* CONFIG_U_SIZE (photonmap.hpp:9) */
#define XYZO_IMP_V 8  /* CONFIG_V_SIZE (photonmap.hpp:10); XYZO_IMP_N = U * V */

static float *IMP_P = NULL, *IMP_D = NULL; /* 3 floats each per importon */
static int IMP_N = 0;
static float IMP_R2 = 0.01f;               /* CONFIG_SEARCH_RADIUS^2 in float */
/* uniform grid over the importons (any structure finds the same set) */
static f3 IMP_LO;
static float IMP_CS = 1.0f;
static int IMP_G[3] = {1, 1, 1};
static int *IMP_START = NULL, *IMP_IDX = NULL;

/* Light point from two draws (SampleLightPosition + Triangle::Sample). */
static void light_point(float lt, float ls, f3 *pos, f3 *sn, f3 *gn, int *mat) {
  float const u = ls * S.cdf[S.nl];
  int lo = 0, hi = S.nl + 1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (!(u < S.cdf[mid])) lo = mid + 1; else hi = mid;
  }
  int const n = lo - 1;
  float const v = (u - S.cdf[n]) / (S.cdf[n + 1] - S.cdf[n]);
  int const li = S.lights[n];
  float const ss = sqrtf(v);
  float const uu = ss * (1 - lt), vv = ss * lt;
  *pos = add3(add3(S.v0[li], scale3(S.e1[li], uu)), scale3(S.e2[li], vv));
  *sn = normalize3(add3(add3(S.n0[li], scale3(S.s1[li], uu)), scale3(S.s2[li], vv)));
  *gn = S.ng[li];
  *mat = S.mat[li];
}

/* Tangent frame about a normal as Triangle::GeometricBasis builds it
 * (xyz/geom/triangle.cpp:181-191). */
static void frame_about(f3 n, f3 *t, f3 *b) {
  f3 tt = mk(-n.z, 0, n.x);
  float const l2 = dot3(tt, tt);
  if (l2 > 0) {
    tt = scale3(tt, 1.0f / sqrtf(l2));
    *b = cross3(tt, n);
  } else {
    *b = mk(0, 0, (n.y > 0) ? 1.0f : -1.0f);
    tt = cross3(n, *b);
  }
  *t = tt;
}

static f3 cosine_dir(f3 t, f3 b, f3 n, float mu_phi, float mu_theta) {
  float const phi = (float)(2 * XYZO_M_PI) * mu_phi;
  float const cos_t = sqrtf(mu_theta), sin_t = sqrtf(1 - mu_theta);
  return add3(add3(scale3(t, sin_t * cosf(phi)), scale3(b, sin_t * sinf(phi))), scale3(n, cos_t));
}

/* Emits `particles` light particles; writes up to `cap` importons (position,
 * incoming direction: 6 floats each) in particle order, returns how many
 * there are in all. */
int xyzo_importons_emit(int particles, int max_depth, int min_depth, uint64_t seed, float *out, int cap) {
  int count = 0;
  if (S.nl <= 0) return 0;
  for (int pi = 0; pi < particles; ++pi) {
    xyzo_stream st;
    xyzo_stream_init(&st, seed, (uint32_t)pi, 0xffffffffu, 0u);
    float const lt = xyzo_stream_next(&st);
    float const ls = xyzo_stream_next(&st);
    f3 pos, lsn, lgn, t, b;
    int lmat;
    light_point(lt, ls, &pos, &lsn, &lgn, &lmat);
    frame_about(lgn, &t, &b);
    float const mp = xyzo_stream_next(&st);
    float const mt = xyzo_stream_next(&st);
    f3 dir = cosine_dir(t, b, lgn, mp, mt);
    for (int depth = 0; depth < max_depth; ++depth) {
      isect_t p;
      int const tri = find_intersection(pos, dir, &p);
      if (tri < 0) break;
      int const m = S.mat[tri];
      if (S.is_light[m]) break; /* Light::BoundsImportance */
      f3 sn = normalize3(add3(add3(S.n0[tri], scale3(S.s1[tri], p.f)), scale3(S.s2[tri], p.g)));
      f3 gn = S.ng[tri];
      if (p.back) {
        gn = neg3(gn);
        sn = neg3(sn);
      }
      pos = add3(pos, scale3(dir, p.tmax));
      if (depth >= min_depth) {
        if (count < cap) {
          float *o = out + 6 * (size_t)count;
          o[0] = pos.x, o[1] = pos.y, o[2] = pos.z, o[3] = dir.x, o[4] = dir.y, o[5] = dir.z;
        }
        ++count;
      }
      if (-dot3(dir, sn) <= 0) break;
      if (xyzo_stream_next(&st) >= S.albedo[m].y) break;
      frame_about(gn, &t, &b);
      float const a = xyzo_stream_next(&st);
      float const c = xyzo_stream_next(&st);
      dir = cosine_dir(t, b, gn, a, c);
    }
  }
  return count;
}

static int imp_cell(float v, int k) {
  int c = (int)floorf((v - at3(IMP_LO, k)) / IMP_CS);
  return c < 0 ? 0 : (c >= IMP_G[k] ? IMP_G[k] - 1 : c);
}

/* Loads an importon map (6 floats per importon) with search radius r. */
void xyzo_importons_set(const float *pd, int n, float radius, int enable, int guide_bounces) {
  free(IMP_P);
  free(IMP_D);
  free(IMP_START);
  free(IMP_IDX);
  IMP_P = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
  IMP_D = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
  IMP_N = n;
  IMP_R2 = radius * radius;
  IMP_ON = enable;
  IMP_BOUNCES = guide_bounces;
  f3 lo = mk(INFINITY, INFINITY, INFINITY), hi = mk(-INFINITY, -INFINITY, -INFINITY);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      IMP_P[3 * i + k] = pd[6 * i + k];
      IMP_D[3 * i + k] = pd[6 * i + 3 + k];
    }
    lo = mk(fminf(lo.x, pd[6 * i]), fminf(lo.y, pd[6 * i + 1]), fminf(lo.z, pd[6 * i + 2]));
    hi = mk(fmaxf(hi.x, pd[6 * i]), fmaxf(hi.y, pd[6 * i + 1]), fmaxf(hi.z, pd[6 * i + 2]));
  }
  if (n == 0) lo = hi = mk(0, 0, 0);
  IMP_LO = lo;
  IMP_CS = radius > 0 ? radius : 1.0f;
  size_t cells = 1;
  for (int k = 0; k < 3; ++k) {
    IMP_G[k] = (int)((at3(hi, k) - at3(lo, k)) / IMP_CS) + 1;
    if (IMP_G[k] > 1024) IMP_G[k] = 1024;
    cells *= (size_t)IMP_G[k];
  }
  if (cells > ((size_t)1 << 24)) { /* coarser cells for very spread maps */
    IMP_CS *= cbrtf((float)cells / (float)(1 << 24)) + 1.0f;
    cells = 1;
    for (int k = 0; k < 3; ++k) {
      IMP_G[k] = (int)((at3(hi, k) - at3(lo, k)) / IMP_CS) + 1;
      cells *= (size_t)IMP_G[k];
    }
  }
  IMP_START = (int *)calloc(cells + 1, sizeof(int));
  IMP_IDX = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int *key = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) {
    key[i] = (imp_cell(IMP_P[3 * i + 2], 2) * IMP_G[1] + imp_cell(IMP_P[3 * i + 1], 1)) * IMP_G[0] +
             imp_cell(IMP_P[3 * i], 0);
    IMP_START[key[i] + 1]++;
  }
  for (size_t c = 0; c < cells; ++c) IMP_START[c + 1] += IMP_START[c];
  int *fill = (int *)malloc(sizeof(int) * (cells + 1));
  memcpy(fill, IMP_START, sizeof(int) * (cells + 1));
  for (int i = 0; i < n; ++i) IMP_IDX[fill[key[i]]++] = i;
  free(fill);
  free(key);
}

/* ImportanceQuery over a fixed-radius neighbourhood (begin_query, push_back,
 * end_query: photonmap.cpp:321-373): 16 (cos^2 theta, phi) bins that start at
 * 16 counts each, one count per importon within the radius whose direction
 * arrives from above the shading normal and whose point, moved along that
 * direction onto the tangent plane, is within the radius; c[0] = 0 and c[i]
 * the cumulative counts. */
static void imp_hist(f3 pos, f3 sn, f3 tan, f3 bin, float c[XYZO_IMP_N + 1]) {
  c[0] = 0;
  for (int i = 1; i <= XYZO_IMP_N; ++i) c[i] = (float)XYZO_IMP_N;
  int lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = imp_cell(at3(pos, k) - IMP_CS, k);
    hi[k] = imp_cell(at3(pos, k) + IMP_CS, k);
  }
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int y = lo[1]; y <= hi[1]; ++y)
      for (int x = lo[0]; x <= hi[0]; ++x) {
        int const cell = (z * IMP_G[1] + y) * IMP_G[0] + x;
        for (int q = IMP_START[cell]; q < IMP_START[cell + 1]; ++q) {
          int const j = IMP_IDX[q];
          f3 const d = mk(IMP_P[3 * j] - pos.x, IMP_P[3 * j + 1] - pos.y, IMP_P[3 * j + 2] - pos.z);
          if (!(dot3(d, d) < IMP_R2)) continue;
          f3 const dir = mk(IMP_D[3 * j], IMP_D[3 * j + 1], IMP_D[3 * j + 2]);
          float const cs = -dot3(dir, sn);
          if (cs <= 0) continue;
          f3 const vp = add3(d, scale3(dir, dot3(d, sn)));
          if (dot3(vp, vp) >= IMP_R2) continue;
          int u = (int)(cs * cs * XYZO_IMP_U);
          if (u >= XYZO_IMP_U) u = XYZO_IMP_U - 1;
          float phi = 0.5f * atan2f(-dot3(dir, bin), -dot3(dir, tan));
          if (phi < 0) phi = (float)((double)phi + XYZO_M_PI);
          int v = (int)((double)phi * (XYZO_IMP_V * XYZO_M_1_PI));
          if (v >= XYZO_IMP_V) v = XYZO_IMP_V - 1;
          c[1 + u * XYZO_IMP_V + v] += 1;
        }
      }
  for (int i = 2; i <= XYZO_IMP_N; ++i) c[i] += c[i - 1];
}

/* ImportanceQuery::GetDensity (photonmap.cpp:375-401). */
static float imp_density(const float c[XYZO_IMP_N + 1], f3 dir, f3 sn, f3 tan, f3 bin) {
  float const cs = -dot3(dir, sn);
  if (cs <= 0) return 0.0f;
  int u = (int)(cs * cs * XYZO_IMP_U);
  if (u >= XYZO_IMP_U) u = XYZO_IMP_U - 1;
  float phi = 0.5f * atan2f(-dot3(dir, bin), -dot3(dir, tan));
  if (phi < 0) phi = (float)((double)phi + XYZO_M_PI);
  int v = (int)((double)phi * (XYZO_IMP_V * XYZO_M_1_PI));
  if (v >= XYZO_IMP_V) v = XYZO_IMP_V - 1;
  int const n = u * XYZO_IMP_V + v;
  return XYZO_IMP_N * (c[n + 1] - c[n]) / c[XYZO_IMP_N];
}

/* Histograms (16 cumulative counts c[1..16]) for n frames given as 12 floats:
 * position, tangent, binormal, shading normal. */
void xyzo_importons_query(const float *fr, int n, float *out) {
  for (int i = 0; i < n; ++i) {
    const float *q = fr + 12 * (size_t)i;
    float c[XYZO_IMP_N + 1];
    imp_hist(mk(q[0], q[1], q[2]), mk(q[9], q[10], q[11]), mk(q[3], q[4], q[5]), mk(q[6], q[7], q[8]), c);
    memcpy(out + XYZO_IMP_N * (size_t)i, c + 1, sizeof(float) * XYZO_IMP_N);
  }
}
