/*
 * kdop_oracle.c -- CPU restatement of the reference's kDOP BVH collision path
 * (refit, tandem traversal, MOST_OPPOSING tet-tet contacts).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA library: tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py call it; the
 * product never does.  Its results are pinned against the reference's own
 * code (oracle/_ref, built by oracle/Makefile from the reference's sources)
 * and against tests/golden/.
 *
 * Reference files followed (paths inside the reference project):
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/types/geometry_direction_table.h:54-176
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/types/geometry_dop.h:49-74
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/geometry_make_union.h:10-24
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/overlap/geometry_overlap_dop_dop.h:13-25
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/overlap/geometry_overlap_interval_interval.h:12-20
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/overlap/geometry_overlap_tetrahedron_tetrahedron.h:14-290
 *   FOUNDATION/GEOMETRY/GEOMETRY/include/contacts/geometry_contacts_tetrahedron_tetrahedron.h:31-157,465-681,1313-1345
 *   FOUNDATION/MESH_ARRAY/MESH_ARRAY/include/mesh_array_compute_surface_map.h:41-76
 *   FOUNDATION/TINY/TINY/include/tiny_vector_ops_policy.h:33-76
 *   FOUNDATION/TINY/TINY/include/tiny_quaternion_functions.h:137-152
 *   SIMULATION/KDOP/KDOP/include/kdop_mesh_reorder.h:173-353
 *   SIMULATION/KDOP/KDOP/include/kdop_make_tree.h:58-121
 *   SIMULATION/KDOP/KDOP/include/kdop_refit_tree.h:24-115
 *   SIMULATION/KDOP/KDOP/include/kdop_tandem_traversal.h:19-196
 */
#define _POSIX_C_SOURCE 200809L
#include "kdop_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define REAL float
#define SUF _f
#include "kdop_oracle_impl.h"
#undef REAL
#undef SUF
#define REAL double
#define SUF _d
#include "kdop_oracle_impl.h"
#undef REAL
#undef SUF

int or_contacts_dd(const double* xyzA, const uint32_t* tetsA, const uint8_t* surfA, const double* xyzB,
                   const uint32_t* tetsB, const uint8_t* surfB, int64_t n_pairs, const uint32_t* pairs,
                   int64_t cap, double* out, int64_t* n_out, or_record* rec) {
  return contacts_generic_d(xyzA, xyzB, 1, tetsA, surfA, tetsB, surfB, n_pairs, pairs, cap, out, n_out, rec);
}

/* ---- Morton order (kdop_mesh_reorder.h:173-353) ----------------------------- */
typedef struct {
  unsigned long long code;
  uint32_t idx;
} or_mc;

static int or_mc_cmp(const void* a, const void* b) {
  const or_mc* x = (const or_mc*)a;
  const or_mc* y = (const or_mc*)b;
  if (x->code != y->code) return x->code < y->code ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

int or_morton_order(const float* xyz, int64_t nv, int64_t nt, const uint32_t* tets, uint32_t* perm) {
  (void)nv;
  if (nt <= 0) return 0;
  float* c = (float*)malloc(sizeof(float) * 3 * (size_t)nt);
  or_mc* mc = (or_mc*)malloc(sizeof(or_mc) * (size_t)nt);
  if (!c || !mc) { free(c); free(mc); return -1; }
  float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float mx[3] = {FLT_MIN, FLT_MIN, FLT_MIN}; /* numeric_limits<float>::min(), as the reference */
  for (int64_t t = 0; t < nt; ++t) {
    const uint32_t* q = tets + 4 * t;
    for (int d = 0; d < 3; ++d) {
      float s = xyz[3 * q[0] + d] + xyz[3 * q[1] + d];
      s = s + xyz[3 * q[2] + d];
      s = s + xyz[3 * q[3] + d];
      float v = (float)(0.25 * (double)s);
      c[3 * t + d] = v;
      mn[d] = (v < mn[d]) ? v : mn[d];
      mx[d] = (mx[d] < v) ? v : mx[d];
    }
  }
  const int K = (int)(sizeof(unsigned long long) * 8) / 3;
  int scale = (int)((float)((1 << K) - 1) / (mx[0] - mn[0]));
  int sy = (int)((float)((1 << K) - 1) / (mx[1] - mn[1]));
  int sz = (int)((float)((1 << K) - 1) / (mx[2] - mn[2]));
  scale = sy < scale ? sy : scale;
  scale = sz < scale ? sz : scale;
  for (int64_t t = 0; t < nt; ++t) {
    unsigned long long x = (unsigned long long)(float)(int)((c[3 * t + 0] - mn[0]) * (float)scale);
    unsigned long long y = (unsigned long long)(float)(int)((c[3 * t + 1] - mn[1]) * (float)scale);
    unsigned long long z = (unsigned long long)(float)(int)((c[3 * t + 2] - mn[2]) * (float)scale);
    unsigned long long code = 0;
    for (unsigned long k = 0; k < (unsigned long)K; ++k) {
      code |= ((x >> k) & 1ull) << (3 * k);
      code |= ((y >> k) & 1ull) << (3 * k + 1);
      code |= ((z >> k) & 1ull) << (3 * k + 2);
    }
    mc[t].code = code;
    mc[t].idx = (uint32_t)t;
  }
  qsort(mc, (size_t)nt, sizeof(or_mc), or_mc_cmp);
  for (int64_t t = 0; t < nt; ++t) perm[t] = mc[t].idx;
  free(c);
  free(mc);
  return 0;
}

/* ---- median-split tree (kdop_make_tree.h:58-121), one chunk ---------------- */
typedef struct {
  int64_t* left;
  int64_t* right;
  int64_t* tet;
  const uint32_t* perm;
  int64_t free_idx;
} or_builder;

static void or_build_rec(or_builder* b, int64_t node, int64_t first, int64_t last) {
  if (last - first + 1 > 1) {
    int64_t l = b->free_idx, r = b->free_idx + 1;
    b->free_idx += 2;
    b->left[node] = l;
    b->right[node] = r;
    b->tet[node] = -1;
    int64_t mid = (int64_t)floor((double)(first + last) / 2.0);
    or_build_rec(b, l, first, mid);
    or_build_rec(b, r, mid + 1, last);
  } else {
    b->left[node] = b->right[node] = -1;
    b->tet[node] = b->perm[first];
  }
}

int64_t or_build_tree(int64_t nt, const uint32_t* perm, int64_t* left, int64_t* right, int64_t* tet) {
  if (nt <= 0) return 0;
  or_builder b;
  b.left = left;
  b.right = right;
  b.tet = tet;
  b.perm = perm;
  b.free_idx = 1;
  or_build_rec(&b, 0, 0, nt - 1);
  return b.free_idx;
}

/* ---- refit (kdop_refit_tree.h:24-115): children have larger indices --------- */
void or_refit_f(int K, const float* xyz, const uint32_t* tets, int64_t nnodes, const int64_t* left,
                const int64_t* right, const int64_t* tet, float* vol) {
  float D[39];
  int N = or_dirs_f(K, D);
  for (int64_t i = nnodes - 1; i >= 0; --i) {
    float* o = vol + (size_t)i * K;
    if (left[i] < 0) {
      tet_dop_f(N, D, xyz, tets + 4 * (size_t)tet[i], o);
    } else {
      const float* a = vol + (size_t)left[i] * K;
      const float* c = vol + (size_t)right[i] * K;
      for (int s = 0; s < N; ++s) {
        o[2 * s] = rmin_f(a[2 * s], c[2 * s]);         /* min(A.lo, B.lo) */
        o[2 * s + 1] = rmax_f(a[2 * s + 1], c[2 * s + 1]); /* max(A.hi, B.hi) */
      }
    }
  }
}

/* ---- tandem traversal (kdop_tandem_traversal.h:19-157) --------------------- */
typedef struct {
  int K;
  const float *volA, *volB;
  const int64_t *leftA, *rightA, *tetA, *leftB, *rightB, *tetB;
  const uint8_t *surfA, *surfB;
  int64_t cap, npairs, tests, leaf_overlaps;
  uint32_t* out;
  int over;
} or_trav;

static int or_overlap_f(const float* a, const float* b, int K) {
  for (int s = 0; s < K / 2; ++s) {
    if (a[2 * s + 1] < b[2 * s]) return 0;     /* A.upper < B.lower */
    if (b[2 * s + 1] < a[2 * s]) return 0;     /* B.upper < A.lower */
  }
  return 1;
}

static void or_trav_rec(or_trav* t, int64_t a, int64_t b) {
  ++t->tests;
  if (!or_overlap_f(t->volA + (size_t)a * t->K, t->volB + (size_t)b * t->K, t->K)) return;
  int la = t->leftA[a] < 0, lb = t->leftB[b] < 0;
  if (la && lb) {
    ++t->leaf_overlaps;
    int64_t ta = t->tetA[a], tb = t->tetB[b];
    if (!t->surfA[ta] || !t->surfB[tb]) return; /* :56-88 */
    if (t->npairs < t->cap) {
      t->out[2 * t->npairs] = (uint32_t)ta;
      t->out[2 * t->npairs + 1] = (uint32_t)tb;
    } else {
      t->over = 1;
    }
    ++t->npairs;
  } else if (!la && !lb) {
    or_trav_rec(t, t->leftA[a], t->leftB[b]);
    or_trav_rec(t, t->leftA[a], t->rightB[b]);
    or_trav_rec(t, t->rightA[a], t->leftB[b]);
    or_trav_rec(t, t->rightA[a], t->rightB[b]);
  } else if (!la && lb) {
    or_trav_rec(t, t->leftA[a], b);
    or_trav_rec(t, t->rightA[a], b);
  } else {
    or_trav_rec(t, a, t->leftB[b]);
    or_trav_rec(t, a, t->rightB[b]);
  }
}

int or_traverse_f(int K, const float* volA, const int64_t* leftA, const int64_t* rightA, const int64_t* tetA,
                  const uint8_t* surfA, const float* volB, const int64_t* leftB, const int64_t* rightB,
                  const int64_t* tetB, const uint8_t* surfB, int64_t cap, uint32_t* out_pairs,
                  int64_t* npairs, int64_t* tests, int64_t* leaf_overlaps) {
  or_trav t;
  memset(&t, 0, sizeof(t));
  t.K = K;
  t.volA = volA; t.volB = volB;
  t.leftA = leftA; t.rightA = rightA; t.tetA = tetA;
  t.leftB = leftB; t.rightB = rightB; t.tetB = tetB;
  t.surfA = surfA; t.surfB = surfB;
  t.cap = cap;
  t.out = out_pairs;
  /* root test of kdop_tandem_traversal.h:164 (the tree root equals node 0) */
  t.tests = 1;
  if (or_overlap_f(volA, volB, K)) or_trav_rec(&t, 0, 0);
  *npairs = t.npairs;
  *tests = t.tests;
  *leaf_overlaps = t.leaf_overlaps;
  return t.over ? -1 : 0;
}

int or_run_pair_f(int K, int64_t nvA, const float* xyzA, const float* restA, int64_t ntA, const uint32_t* tetsA,
                  const uint8_t* surfA, int64_t nvB, const float* xyzB, const float* restB, int64_t ntB,
                  const uint32_t* tetsB, const uint8_t* surfB, int64_t cap, uint32_t* out_pairs, int64_t* npairs,
                  int64_t* tests, int64_t* leaf_overlaps) {
  *npairs = *tests = *leaf_overlaps = 0;
  if (ntA <= 0 || ntB <= 0) return 0;
  int64_t nnA = 2 * ntA - 1, nnB = 2 * ntB - 1;
  uint32_t* pA = (uint32_t*)malloc(4 * (size_t)ntA);
  uint32_t* pB = (uint32_t*)malloc(4 * (size_t)ntB);
  int64_t* tA = (int64_t*)malloc(8 * 3 * (size_t)nnA);
  int64_t* tB = (int64_t*)malloc(8 * 3 * (size_t)nnB);
  float* vA = (float*)malloc(4 * (size_t)K * (size_t)nnA);
  float* vB = (float*)malloc(4 * (size_t)K * (size_t)nnB);
  int rc = -2;
  if (pA && pB && tA && tB && vA && vB) {
    or_morton_order(restA ? restA : xyzA, nvA, ntA, tetsA, pA);
    or_morton_order(restB ? restB : xyzB, nvB, ntB, tetsB, pB);
    or_build_tree(ntA, pA, tA, tA + nnA, tA + 2 * nnA);
    or_build_tree(ntB, pB, tB, tB + nnB, tB + 2 * nnB);
    or_refit_f(K, xyzA, tetsA, nnA, tA, tA + nnA, tA + 2 * nnA, vA);
    or_refit_f(K, xyzB, tetsB, nnB, tB, tB + nnB, tB + 2 * nnB, vB);
    rc = or_traverse_f(K, vA, tA, tA + nnA, tA + 2 * nnA, surfA, vB, tB, tB + nnB, tB + 2 * nnB, surfB, cap,
                       out_pairs, npairs, tests, leaf_overlaps);
  }
  free(pA); free(pB); free(tA); free(tB); free(vA); free(vB);
  return rc;
}

/* ---- many pairs on a thread pool ------------------------------------------- */
typedef struct {
  int K;
  const int64_t *v_off, *t_off;
  const float* xyz;
  const float* rest;
  const uint32_t* tets;
  const uint8_t* surf;
  const uint32_t* pairs;
  int64_t n_pairs;
  int64_t next;
  pthread_mutex_t mu;
  uint32_t** res;
  int64_t *npp, *tpp;
  int err;
} or_pool;

static void* or_pool_worker(void* arg) {
  or_pool* P = (or_pool*)arg;
  for (;;) {
    pthread_mutex_lock(&P->mu);
    int64_t p = P->next++;
    pthread_mutex_unlock(&P->mu);
    if (p >= P->n_pairs) break;
    uint32_t a = P->pairs[2 * p], b = P->pairs[2 * p + 1];
    int64_t ntA = P->t_off[a + 1] - P->t_off[a], ntB = P->t_off[b + 1] - P->t_off[b];
    int64_t cap = 1024;
    for (;;) {
      uint32_t* buf = (uint32_t*)malloc(8 * (size_t)cap);
      int64_t np = 0, tests = 0, lo = 0;
      int rc = or_run_pair_f(P->K, P->v_off[a + 1] - P->v_off[a], P->xyz + 3 * P->v_off[a],
                             P->rest ? P->rest + 3 * P->v_off[a] : NULL, ntA, P->tets + 4 * P->t_off[a],
                             P->surf + P->t_off[a], P->v_off[b + 1] - P->v_off[b], P->xyz + 3 * P->v_off[b],
                             P->rest ? P->rest + 3 * P->v_off[b] : NULL, ntB, P->tets + 4 * P->t_off[b],
                             P->surf + P->t_off[b], cap, buf, &np, &tests, &lo);
      if (rc == -1) {
        free(buf);
        cap = np + 16;
        continue;
      }
      if (rc != 0) P->err = rc;
      P->res[p] = buf;
      P->npp[p] = np;
      P->tpp[p] = tests;
      break;
    }
  }
  return NULL;
}

int or_run_pairs_f(int K, int n_meshes, const int64_t* v_off, const float* xyz, const float* rest, const int64_t* t_off,
                   const uint32_t* tets, const uint8_t* surf, int64_t n_pairs, const uint32_t* pairs,
                   int threads, int64_t cap, uint32_t* out_pairs, int64_t* npairs, int64_t* tests_per_pair,
                   int64_t* pairs_per_pair) {
  (void)n_meshes;
  or_pool P;
  memset(&P, 0, sizeof(P));
  P.K = K; P.v_off = v_off; P.t_off = t_off; P.xyz = xyz; P.rest = rest; P.tets = tets; P.surf = surf;
  P.pairs = pairs; P.n_pairs = n_pairs;
  pthread_mutex_init(&P.mu, NULL);
  P.res = (uint32_t**)calloc((size_t)(n_pairs > 0 ? n_pairs : 1), sizeof(uint32_t*));
  P.npp = pairs_per_pair;
  P.tpp = tests_per_pair;
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, or_pool_worker, &P);
  for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
  int64_t n = 0;
  int over = 0;
  for (int64_t p = 0; p < n_pairs; ++p) {
    for (int64_t i = 0; i < P.npp[p]; ++i, ++n) {
      if (n < cap) {
        out_pairs[3 * n] = (uint32_t)p;
        out_pairs[3 * n + 1] = P.res[p][2 * i];
        out_pairs[3 * n + 2] = P.res[p][2 * i + 1];
      } else {
        over = 1;
      }
    }
    free(P.res[p]);
  }
  free(P.res);
  pthread_mutex_destroy(&P.mu);
  *npairs = n;
  if (P.err) return P.err;
  return over ? -1 : 0;
}

/* ---- surface map (mesh_array_compute_surface_map.h:41-76) ------------------ */
typedef struct {
  uint32_t v[3];
  int64_t tet;
  int face;
} or_face;

static int or_face_cmp(const void* a, const void* b) {
  const or_face* x = (const or_face*)a;
  const or_face* y = (const or_face*)b;
  for (int i = 0; i < 3; ++i)
    if (x->v[i] != y->v[i]) return x->v[i] < y->v[i] ? -1 : 1;
  return 0;
}

int or_surface_map(int64_t nv, int64_t nt, const uint32_t* tets, uint8_t* surf) {
  (void)nv;
  or_face* f = (or_face*)malloc(sizeof(or_face) * 4 * (size_t)(nt > 0 ? nt : 1));
  if (!f) return -1;
  for (int64_t t = 0; t < nt; ++t) {
    surf[t] = 0;
    for (int k = 0; k < 4; ++k) {
      or_face* g = &f[4 * t + k];
      int n = 0;
      for (int v = 0; v < 4; ++v)
        if (v != k) g->v[n++] = tets[4 * t + v];
      /* sort the three ids */
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2 - i; ++j)
          if (g->v[j] > g->v[j + 1]) { uint32_t s = g->v[j]; g->v[j] = g->v[j + 1]; g->v[j + 1] = s; }
      g->tet = t;
      g->face = k;
    }
  }
  qsort(f, 4 * (size_t)nt, sizeof(or_face), or_face_cmp);
  int64_t i = 0, n = 4 * nt;
  while (i < n) {
    int64_t j = i + 1;
    while (j < n && or_face_cmp(&f[i], &f[j]) == 0) ++j;
    if (j - i == 1) surf[f[i].tet] |= (uint8_t)(1u << f[i].face);
    i = j;
  }
  free(f);
  return 0;
}

/* ---- rigid pose (tiny_quaternion_functions.h:137-152) ----------------------- */
void or_rotate_f(const float* q, const float* p, int64_t nv, const float* xyz, float* out) {
  float s = q[0];
  v3_f v = mk_f(q[1], q[2], q[3]);
  v3_f nv3 = mk_f(-q[1], -q[2], -q[3]);
  for (int64_t i = 0; i < nv; ++i) {
    v3_f r = mk_f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    /* prod(q, r) = (-q.v . r, q.v x r + r q.s) */
    float a = -dot_f(v, r);
    v3_f c = cross_f(v, r);
    v3_f A = mk_f(c.x + r.x * s, c.y + r.y * s, c.z + r.z * s);
    /* prod(qr, conj q).imag = a B + A b + A x B with b = q.s, B = -q.v */
    v3_f x = cross_f(A, nv3);
    v3_f im = mk_f((a * nv3.x + A.x * s) + x.x, (a * nv3.y + A.y * s) + x.y, (a * nv3.z + A.z * s) + x.z);
    out[3 * i] = im.x + p[0];
    out[3 * i + 1] = im.y + p[1];
    out[3 * i + 2] = im.z + p[2];
  }
}

/* ---- the project's own single-precision sine --------------------------------
 * Cody-Waite reduction by 2 pi (split constant 6.28125 + remainder), fold into
 * [-pi/2, pi/2], then the Taylor series of sin to degree 11.  Every operation
 * is a separately rounded float op, so the CUDA kernels reproduce it bit for
 * bit. */
float or_sin_f(float x) {
  const float inv2pi = 0.159154936671257019f;
  const float c1 = 6.28125f;
  const float c2 = 0.00193530717f;
  const float pi = 3.14159274101257324f;
  const float hpi = 1.57079637050628662f;
  float k = rintf(x * inv2pi);
  float r = x - k * c1;
  r = r - k * c2;
  if (r > hpi) r = pi - r;
  if (r < -hpi) r = -pi - r;
  float r2 = r * r;
  float s = -2.50521083854417188e-8f;        /* -1/11! */
  s = s * r2 + 2.75573192239858907e-6f;      /*  1/9!  */
  s = s * r2 + -1.98412698412698413e-4f;     /* -1/7!  */
  s = s * r2 + 8.33333333333333333e-3f;      /*  1/5!  */
  s = s * r2 + -1.66666666666666667e-1f;     /* -1/3!  */
  s = s * r2;
  return r + r * s;
}

void or_deform_f(float amp, float w, float phase, int64_t nv, const float* xyz, float* out) {
  for (int64_t i = 0; i < nv; ++i) {
    float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    float arg = (x + y) + z;
    arg = w * arg + phase;
    float d = amp * or_sin_f(arg);
    out[3 * i] = x + d;
    out[3 * i + 1] = y + d;
    out[3 * i + 2] = z + d;
  }
}

/* ---- frozen-decision depth and its gradient (double) ------------------------
 * In exact arithmetic the three corner cross products of make_unscaled_plane
 * are equal and every corner lies on the plane, so the frozen depth uses the
 * first corner throughout; it is smooth in the 8 vertices. */
typedef struct { double x, y, z; } gv;
static gv g_mk(double x, double y, double z) { gv r; r.x = x; r.y = y; r.z = z; return r; }
static gv g_sub(gv a, gv b) { return g_mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static gv g_add(gv a, gv b) { return g_mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static gv g_scl(gv a, double s) { return g_mk(a.x * s, a.y * s, a.z * s); }
static double g_dot(gv a, gv b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static gv g_cross(gv l, gv r) { return g_mk(l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x); }

static void g_load(const double* p12, gv* v) {
  for (int i = 0; i < 4; ++i) v[i] = g_mk(p12[3 * i], p12[3 * i + 1], p12[3 * i + 2]);
}

/* plane normal m of face f of tet T (unscaled), and its first corner */
static gv g_face_m(const gv* T, int f, gv* F0) {
  gv P0 = T[OR_FACE[f][0]], P1 = T[OR_FACE[f][1]], P2 = T[OR_FACE[f][2]];
  *F0 = P0;
  return g_cross(g_sub(P1, P0), g_sub(P2, P0));
}
/* adjoint of m = (P1-P0) x (P2-P0) for face f of T into gT */
static void g_face_m_adj(const gv* T, int f, gv gm, gv* gT) {
  int i0 = OR_FACE[f][0], i1 = OR_FACE[f][1], i2 = OR_FACE[f][2];
  gv u = g_sub(T[i1], T[i0]), w = g_sub(T[i2], T[i0]);
  gv gu = g_cross(w, gm), gw = g_cross(gm, u);
  gT[i1] = g_add(gT[i1], gu);
  gT[i2] = g_add(gT[i2], gw);
  gT[i0] = g_sub(gT[i0], g_add(gu, gw));
}

static gv g_cand(int c, const gv* A, const gv* B) {
  if (c < 8) return (c & 1) ? A[c >> 1] : B[c >> 1];
  int e = (c - 8) >> 3, p = ((c - 8) >> 1) & 3;
  const gv* E = (c & 1) ? A : B; /* edge owner */
  const gv* T = (c & 1) ? B : A; /* plane owner */
  gv a = E[OR_EDGE[e][0]], b = E[OR_EDGE[e][1]], F0;
  gv m = g_face_m(T, p, &F0);
  double dA = fabs(g_dot(m, g_sub(a, F0))), dB = fabs(g_dot(m, g_sub(b, F0)));
  double t = dA / (dA + dB);
  return g_add(a, g_scl(g_sub(b, a), t));
}

static void g_cand_adj(int c, const gv* A, const gv* B, gv gq, gv* gA, gv* gB) {
  if (c < 8) {
    gv* g = (c & 1) ? gA : gB;
    g[c >> 1] = g_add(g[c >> 1], gq);
    return;
  }
  int e = (c - 8) >> 3, p = ((c - 8) >> 1) & 3;
  const gv* E = (c & 1) ? A : B;
  const gv* T = (c & 1) ? B : A;
  gv* gE = (c & 1) ? gA : gB;
  gv* gT = (c & 1) ? gB : gA;
  int ia = OR_EDGE[e][0], ib = OR_EDGE[e][1];
  gv a = E[ia], b = E[ib], F0;
  gv m = g_face_m(T, p, &F0);
  double sA = g_dot(m, g_sub(a, F0)), sB = g_dot(m, g_sub(b, F0));
  double sgA = sA < 0 ? -1.0 : 1.0, sgB = sB < 0 ? -1.0 : 1.0;
  double dA = fabs(sA), dB = fabs(sB), S = dA + dB;
  double t = dA / S;
  /* q = a + (b - a) t */
  gE[ia] = g_add(gE[ia], g_scl(gq, 1.0 - t));
  gE[ib] = g_add(gE[ib], g_scl(gq, t));
  double gt = g_dot(gq, g_sub(b, a));
  double gdA = gt * dB / (S * S), gdB = -gt * dA / (S * S);
  /* dA = sgA m.(a - F0), dB = sgB m.(b - F0) */
  gE[ia] = g_add(gE[ia], g_scl(m, sgA * gdA));
  gE[ib] = g_add(gE[ib], g_scl(m, sgB * gdB));
  int f0 = OR_FACE[p][0];
  gT[f0] = g_sub(gT[f0], g_add(g_scl(m, sgA * gdA), g_scl(m, sgB * gdB)));
  gv gm = g_add(g_scl(g_sub(a, F0), sgA * gdA), g_scl(g_sub(b, F0), sgB * gdB));
  g_face_m_adj(T, p, gm, gT);
}

double or_frozen_depth_d(const double* a12, const double* b12, const or_record* rec, double* n_out) {
  gv A[4], B[4], F0;
  g_load(a12, A);
  g_load(b12, B);
  if (rec->face_a < 0 || rec->imin < 0) return 0.0;
  gv m = g_face_m(A, rec->face_a, &F0);
  gv n = g_scl(m, 1.0 / sqrt(g_dot(m, m)));
  if (n_out) { n_out[0] = n.x; n_out[1] = n.y; n_out[2] = n.z; }
  return g_dot(g_cand(rec->imin, A, B), n) - g_dot(g_cand(rec->imax, A, B), n);
}

void or_depth_grad_d(const double* a12, const double* b12, const or_record* rec, double gd, const double* gn,
                     double* g24) {
  gv A[4], B[4], gA[4], gB[4], F0;
  g_load(a12, A);
  g_load(b12, B);
  for (int i = 0; i < 4; ++i) gA[i] = gB[i] = g_mk(0, 0, 0);
  if (rec->face_a >= 0 && rec->imin >= 0) {
    gv m = g_face_m(A, rec->face_a, &F0);
    double len = sqrt(g_dot(m, m));
    gv n = g_scl(m, 1.0 / len);
    gv qmin = g_cand(rec->imin, A, B), qmax = g_cand(rec->imax, A, B);
    /* depth = qmin.n - qmax.n */
    g_cand_adj(rec->imin, A, B, g_scl(n, gd), gA, gB);
    g_cand_adj(rec->imax, A, B, g_scl(n, -gd), gA, gB);
    gv gnt = g_add(g_mk(gn[0], gn[1], gn[2]), g_scl(g_sub(qmin, qmax), gd));
    gv gm = g_scl(g_sub(gnt, g_scl(n, g_dot(n, gnt))), 1.0 / len);
    g_face_m_adj(A, rec->face_a, gm, gA);
  }
  for (int i = 0; i < 4; ++i) {
    g24[3 * i] = gA[i].x; g24[3 * i + 1] = gA[i].y; g24[3 * i + 2] = gA[i].z;
    g24[12 + 3 * i] = gB[i].x; g24[12 + 3 * i + 1] = gB[i].y; g24[12 + 3 * i + 2] = gB[i].z;
  }
}

void or_frozen_batch_d(int64_t n, const double* a12, const double* b12, const or_record* rec, double* depth,
                       double* normal) {
  for (int64_t i = 0; i < n; ++i)
    depth[i] = or_frozen_depth_d(a12 + 12 * i, b12 + 12 * i, rec + i, normal ? normal + 3 * i : NULL);
}

void or_depth_grad_batch_d(int64_t n, const double* a12, const double* b12, const or_record* rec, const double* gd,
                           const double* gn, double* g24) {
  for (int64_t i = 0; i < n; ++i) or_depth_grad_d(a12 + 12 * i, b12 + 12 * i, rec + i, gd[i], gn + 3 * i, g24 + 24 * i);
}
