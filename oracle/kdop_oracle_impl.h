/*
 * Precision-generic part of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 * Included twice by kdop_oracle.c with REAL = float / double and SUF = _f / _d.
 * Every floating-point expression keeps the reference's operation order so
 * that the float instantiation reproduces the reference's FP32 results bit for
 * bit (compiled with -ffp-contract=off: no FMA contraction).
 */
#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define F(name) OR_CAT(name, SUF)

typedef struct { REAL x, y, z; } F(v3);

static inline F(v3) F(mk)(REAL x, REAL y, REAL z) { F(v3) r; r.x = x; r.y = y; r.z = z; return r; }
static inline F(v3) F(sub)(F(v3) a, F(v3) b) { return F(mk)(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline F(v3) F(add)(F(v3) a, F(v3) b) { return F(mk)(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline F(v3) F(scl)(F(v3) a, REAL s) { return F(mk)(a.x * s, a.y * s, a.z * s); }
/* tiny_vector_ops_policy.h:33-45: ((0 + a0 b0) + a1 b1) + a2 b2 */
static inline REAL F(dot)(F(v3) a, F(v3) b) {
  REAL d = (REAL)0;
  d = d + a.x * b.x;
  d = d + a.y * b.y;
  d = d + a.z * b.z;
  return d;
}
/* tiny_vector_ops_policy.h:47-54 */
static inline F(v3) F(cross)(F(v3) l, F(v3) r) {
  return F(mk)(l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x);
}
/* tiny_vector_ops_policy.h:56-75: multiply by the reciprocal of the norm */
static inline F(v3) F(unit)(F(v3) m) {
  REAL l = (REAL)sqrt((double)F(dot)(m, m));
  if (sizeof(REAL) == 4) l = (REAL)sqrtf((float)F(dot)(m, m));
  if (l > (REAL)0) {
    REAL inv = (REAL)1 / l;
    m.x = m.x * inv;
    m.y = m.y * inv;
    m.z = m.z * inv;
  }
  return m;
}
static inline REAL F(rmin)(REAL a, REAL b) { return (b < a) ? b : a; } /* std::min */
static inline REAL F(rmax)(REAL a, REAL b) { return (a < b) ? b : a; } /* std::max */
static inline REAL F(rabs)(REAL a) { return a < (REAL)0 ? -a : (a == (REAL)0 ? (REAL)0 : a); }

/* ---- direction tables (geometry_direction_table.h:54-176) ------------------ */
static void F(set_dir)(REAL* o, int i, REAL x, REAL y, REAL z, int normalise) {
  F(v3) v = F(mk)(x, y, z);
  if (normalise) v = F(unit)(v);
  o[3 * i] = v.x; o[3 * i + 1] = v.y; o[3 * i + 2] = v.z;
}
static int F(dirs3)(REAL* o, int at) {
  F(set_dir)(o, at + 0, 1, 0, 0, 0); F(set_dir)(o, at + 1, 0, 1, 0, 0); F(set_dir)(o, at + 2, 0, 0, 1, 0);
  return at + 3;
}
static int F(dirs4)(REAL* o, int at) {
  F(set_dir)(o, at + 0, 1, 1, 1, 1); F(set_dir)(o, at + 1, 1, 1, -1, 1);
  F(set_dir)(o, at + 2, 1, -1, 1, 1); F(set_dir)(o, at + 3, 1, -1, -1, 1);
  return at + 4;
}
static int F(dirs6)(REAL* o, int at) {
  F(set_dir)(o, at + 0, 1, 1, 0, 1); F(set_dir)(o, at + 1, 1, -1, 0, 1); F(set_dir)(o, at + 2, 1, 0, 1, 1);
  F(set_dir)(o, at + 3, 0, 1, 1, 1); F(set_dir)(o, at + 4, -1, 0, 1, 1); F(set_dir)(o, at + 5, 0, -1, 1, 1);
  return at + 6;
}
int F(or_dirs)(int K, REAL* o) {
  switch (K) {
    case 6: return F(dirs3)(o, 0);
    case 8: return F(dirs4)(o, 0);
    case 12: return F(dirs6)(o, 0);
    case 14: return F(dirs4)(o, F(dirs3)(o, 0));
    case 18: return F(dirs6)(o, F(dirs3)(o, 0));
    case 20: return F(dirs6)(o, F(dirs4)(o, 0));
    case 26: return F(dirs6)(o, F(dirs4)(o, F(dirs3)(o, 0)));
  }
  return -1;
}

/* ---- make_dop over the 4 tet vertices (geometry_dop.h:49-74) --------------- */
static void F(tet_dop)(int N, const REAL* D, const float* xyz, const uint32_t* tet, REAL* out) {
  for (int k = 0; k < N; ++k) {
    F(v3) d = F(mk)(D[3 * k], D[3 * k + 1], D[3 * k + 2]);
    REAL lo = (sizeof(REAL) == 4) ? (REAL)FLT_MAX : (REAL)DBL_MAX;
    REAL hi = -lo;
    for (int v = 0; v < 4; ++v) {
      const float* p = xyz + 3 * (size_t)tet[v];
      REAL pr = F(dot)(d, F(mk)((REAL)p[0], (REAL)p[1], (REAL)p[2]));
      lo = F(rmin)(lo, pr);
      hi = F(rmax)(hi, pr);
    }
    out[2 * k] = lo;
    out[2 * k + 1] = hi;
  }
}

void F(or_leaf_dops)(int K, const float* xyz, int64_t nt, const uint32_t* tets, REAL* out) {
  REAL D[39];
  int N = F(or_dirs)(K, D);
  for (int64_t t = 0; t < nt; ++t) F(tet_dop)(N, D, xyz, tets + 4 * t, out + (size_t)t * K);
}

/* ---- tet-tet contacts, MOST_OPPOSING_SURFACES ------------------------------ */
typedef struct { F(v3) n; F(v3) p; } F(uplane);

#ifndef OR_TABLES_DEFINED
#define OR_TABLES_DEFINED
/* geometry_tetrahedron.h:231-257 (faces listed so the normal points out) */
static const int OR_FACE[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
/* geometry_contacts_tetrahedron_tetrahedron.h:584-591 */
static const int OR_EDGE[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
#endif

/* make_unscaled_plane (geometry_contacts_tetrahedron_tetrahedron.h:31-62):
 * the largest of the three corner cross products; later variants win ties. */
static F(uplane) F(unscaled_plane)(F(v3) p0, F(v3) p1, F(v3) p2) {
  F(uplane) pl;
  F(v3) m0 = F(cross)(F(sub)(p1, p0), F(sub)(p2, p0));
  F(v3) m1 = F(cross)(F(sub)(p2, p1), F(sub)(p0, p1));
  F(v3) m2 = F(cross)(F(sub)(p0, p2), F(sub)(p1, p2));
  REAL l0 = F(dot)(m0, m0), l1 = F(dot)(m1, m1), l2 = F(dot)(m2, m2);
  pl.n = m0; pl.p = p0;
  if (l0 >= l1 && l0 >= l2) { pl.n = m0; pl.p = p0; }
  if (l1 >= l0 && l1 >= l2) { pl.n = m1; pl.p = p1; }
  if (l2 >= l1 && l2 >= l0) { pl.n = m2; pl.p = p2; }
  return pl;
}
static inline REAL F(sdist)(F(v3) q, F(uplane) pl) { return F(dot)(pl.n, F(sub)(q, pl.p)); }
static int F(inside)(F(v3) q, const F(uplane)* pl) {
  REAL d0 = F(sdist)(q, pl[0]), d1 = F(sdist)(q, pl[1]), d2 = F(sdist)(q, pl[2]), d3 = F(sdist)(q, pl[3]);
  if (d0 > 0) return 0;
  if (d1 > 0) return 0;
  if (d2 > 0) return 0;
  if (d3 > 0) return 0;
  return 1;
}
static int F(crossing)(F(v3) a, F(v3) b, F(uplane) pl) {
  REAL dA = F(sdist)(a, pl), dB = F(sdist)(b, pl);
  if (dA >= 0 && dB >= 0) return 0;
  if (dA <= 0 && dB <= 0) return 0;
  return 1;
}
static F(v3) F(intersect)(F(v3) a, F(v3) b, F(uplane) pl) {
  REAL dA = F(rabs)(F(sdist)(a, pl));
  REAL dB = F(rabs)(F(sdist)(b, pl));
  REAL t = dA / (dA + dB);
  return F(add)(a, F(scl)(F(sub)(b, a), t));
}

/* Normalised plane of geometry_plane.h:102-111 and its signed distance :171-175 */
typedef struct { F(v3) n; REAL w; } F(nplane);
static F(nplane) F(make_plane)(F(v3) p0, F(v3) p1, F(v3) p2) {
  F(nplane) P;
  P.n = F(unit)(F(cross)(F(sub)(p1, p0), F(sub)(p2, p0)));
  P.w = F(dot)(p0, P.n);
  return P;
}
static inline REAL F(pdist)(F(v3) p, F(nplane) P) { return F(dot)(P.n, p) - P.w; }

/* SAT_line (geometry_overlap_tetrahedron_tetrahedron.h:14-47) */
static int F(sat_line)(F(v3) a0, F(v3) a1, F(v3) a2, F(v3) b0, F(v3) b1, F(v3) b2, F(v3) n) {
  REAL s0 = F(dot)(n, a0), s1 = F(dot)(n, a1), s2 = F(dot)(n, a2);
  REAL t0 = F(dot)(n, b0), t1 = F(dot)(n, b1), t2 = F(dot)(n, b2);
  REAL smin = F(rmin)(F(rmin)(s0, s1), s2), tmin = F(rmin)(F(rmin)(t0, t1), t2);
  REAL smax = F(rmax)(F(rmax)(s0, s1), s2), tmax = F(rmax)(F(rmax)(t0, t1), t2);
  return (smax < tmin) || (smin > tmax);
}

#ifndef OR_SAT_TABLE_DEFINED
#define OR_SAT_TABLE_DEFINED
/* The 36 edge-edge axes of geometry_overlap_tetrahedron_tetrahedron.h:109-287,
 * in their order.  Per entry: A edge, B edge, the A vertex left out of the
 * three projected A vertices, the B vertex left out. */
static const unsigned char OR_SAT_EDGE[36][4] = {
    {0, 0, 0, 0}, {0, 1, 0, 2}, {0, 2, 0, 3}, {0, 3, 0, 2}, {0, 4, 0, 3}, {0, 5, 0, 3},
    {1, 0, 0, 0}, {1, 1, 0, 0}, {1, 2, 0, 3}, {1, 3, 0, 2}, {1, 4, 0, 3}, {1, 5, 0, 3},
    {2, 0, 0, 0}, {2, 1, 0, 0}, {2, 2, 0, 0}, {2, 3, 0, 2}, {2, 4, 0, 3}, {2, 5, 0, 3},
    {3, 0, 2, 0}, {3, 1, 2, 0}, {3, 2, 2, 0}, {3, 3, 2, 2}, {3, 4, 2, 3}, {3, 5, 2, 3},
    {4, 0, 3, 0}, {4, 1, 3, 0}, {4, 2, 3, 0}, {4, 3, 3, 2}, {4, 4, 3, 3}, {4, 5, 3, 3},
    {5, 0, 3, 0}, {5, 1, 3, 0}, {5, 2, 3, 0}, {5, 3, 3, 2}, {5, 4, 3, 3}, {5, 5, 3, 3}};
#endif

/* overlap_tetrahedron_tetrahedron (geometry_overlap_tetrahedron_tetrahedron.h:51-290) */
static int F(tet_overlap)(const F(v3)* A, const F(v3)* B) {
  for (int i = 0; i < 4; ++i) {
    F(nplane) P = F(make_plane)(A[OR_FACE[i][0]], A[OR_FACE[i][1]], A[OR_FACE[i][2]]);
    REAL b0 = F(pdist)(B[0], P), b1 = F(pdist)(B[1], P), b2 = F(pdist)(B[2], P), b3 = F(pdist)(B[3], P);
    if (b0 > 0 && b1 > 0 && b2 > 0 && b3 > 0) return 0;
  }
  for (int i = 0; i < 4; ++i) {
    F(nplane) P = F(make_plane)(B[OR_FACE[i][0]], B[OR_FACE[i][1]], B[OR_FACE[i][2]]);
    REAL a0 = F(pdist)(A[0], P), a1 = F(pdist)(A[1], P), a2 = F(pdist)(A[2], P), a3 = F(pdist)(A[3], P);
    if (a0 > 0 && a1 > 0 && a2 > 0 && a3 > 0) return 0;
  }
  for (int e = 0; e < 36; ++e) {
    const unsigned char* s = OR_SAT_EDGE[e];
    F(v3) ea = F(sub)(A[OR_EDGE[s[0]][1]], A[OR_EDGE[s[0]][0]]);
    F(v3) eb = F(sub)(B[OR_EDGE[s[1]][1]], B[OR_EDGE[s[1]][0]]);
    F(v3) ax = F(cross)(ea, eb);
    F(v3) a3[3], b3[3];
    int na = 0, nb = 0;
    for (int v = 0; v < 4; ++v) {
      if (v != s[2]) a3[na++] = A[v];
      if (v != s[3]) b3[nb++] = B[v];
    }
    if (F(sat_line)(a3[0], a3[1], a3[2], b3[0], b3[1], b3[2], ax)) return 0;
  }
  return 1;
}

/* pick_most_opposing_surface_normal (…_tetrahedron_tetrahedron.h:465-533) */
static int F(pick_normal)(const F(v3)* A, const F(v3)* B, unsigned sa, unsigned sb, F(v3)* n, int* fa,
                          int* fb) {
  int found = 0;
  REAL best = 0;
  for (int a = 0; a < 4; ++a) {
    if (!((sa >> a) & 1)) continue;
    F(uplane) pA = F(unscaled_plane)(A[OR_FACE[a][0]], A[OR_FACE[a][1]], A[OR_FACE[a][2]]);
    F(v3) nA = F(unit)(pA.n);
    for (int b = 0; b < 4; ++b) {
      if (!((sb >> b) & 1)) continue;
      F(uplane) pB = F(unscaled_plane)(B[OR_FACE[b][0]], B[OR_FACE[b][1]], B[OR_FACE[b][2]]);
      F(v3) nB = F(unit)(pB.n);
      REAL test = F(dot)(nA, nB);
      if (test >= 0) continue;
      REAL testA = F(dot)(pA.n, F(sub)(B[b], pA.p));
      REAL testB = F(dot)(pB.n, F(sub)(A[a], pB.p));
      if (testA < 0) continue;
      if (testB < 0) continue;
      if (test < best) {
        *n = nA;
        best = test;
        found = 1;
        *fa = a;
        *fb = b;
      }
    }
  }
  return found;
}

/* Candidate code c (0..55) in the order of
 * generate_contacts_from_intersection (…_tetrahedron_tetrahedron.h:569-620):
 *   c < 8 : vertex v = c/2; c even: B.p(v) inside A, odd: A.p(v) inside B
 *   c >= 8: e = (c-8)/8, plane p = ((c-8)/2)%4; even: B edge e x plane p of A,
 *           odd: A edge e x plane p of B. */
static int F(candidate)(int c, const F(v3)* A, const F(v3)* B, const F(uplane)* PA, const F(uplane)* PB,
                        F(v3)* q) {
  if (c < 8) {
    int v = c >> 1;
    if (!(c & 1)) {
      if (!F(inside)(B[v], PA)) return 0;
      *q = B[v];
    } else {
      if (!F(inside)(A[v], PB)) return 0;
      *q = A[v];
    }
    return 1;
  }
  int e = (c - 8) >> 3, p = ((c - 8) >> 1) & 3;
  int i = OR_EDGE[e][0], j = OR_EDGE[e][1];
  if (!(c & 1)) {
    if (!F(crossing)(B[i], B[j], PA[p])) return 0;
    F(v3) qq = F(intersect)(B[i], B[j], PA[p]);
    if (!F(inside)(qq, PA)) return 0;
    *q = qq;
  } else {
    if (!F(crossing)(A[i], A[j], PB[p])) return 0;
    F(v3) qq = F(intersect)(A[i], A[j], PB[p]);
    if (!F(inside)(qq, PB)) return 0;
    *q = qq;
  }
  return 1;
}

/* contacts_tetrahedron_tetrahedron(..., MOST_OPPOSING_SURFACES) for one pair.
 * Writes up to OR_NCAND rows (p3 n3 d) into rows; returns the row count. */
static int F(pair_contacts)(const F(v3)* A, const F(v3)* B, unsigned sa, unsigned sb, REAL* rows,
                            or_record* rec) {
  rec->face_a = rec->face_b = -1;
  rec->imin = rec->imax = -1;
  rec->ncontacts = 0;
  rec->overlap = 0;
  rec->cand_mask = 0;
  if (!sa || !sb) return 0;
  if (!F(tet_overlap)(A, B)) return 0;
  rec->overlap = 1;
  F(v3) n = F(mk)(0, 0, 0);
  int fa = -1, fb = -1;
  if (!F(pick_normal)(A, B, sa, sb, &n, &fa, &fb)) return 0;
  rec->face_a = fa;
  rec->face_b = fb;
  F(uplane) PA[4], PB[4];
  for (int v = 0; v < 4; ++v) {
    PA[v] = F(unscaled_plane)(A[OR_FACE[v][0]], A[OR_FACE[v][1]], A[OR_FACE[v][2]]);
    PB[v] = F(unscaled_plane)(B[OR_FACE[v][0]], B[OR_FACE[v][1]], B[OR_FACE[v][2]]);
  }
  F(v3) q[OR_NCAND];
  int code[OR_NCAND];
  int nq = 0;
  for (int c = 0; c < OR_NCAND; ++c)
    if (F(candidate)(c, A, B, PA, PB, &q[nq])) {
      rec->cand_mask |= 1ull << c;
      code[nq++] = c;
    }
  if (!nq) return 0;
  REAL big = (sizeof(REAL) == 4) ? (REAL)FLT_MAX : (REAL)DBL_MAX;
  REAL mn = big, mx = -big;
  int imn = -1, imx = -1;
  for (int i = 0; i < nq; ++i) {
    REAL d = F(dot)(q[i], n);
    if (d < mn) { mn = d; imn = code[i]; }
    if (mx < d) { mx = d; imx = code[i]; }
  }
  rec->imin = imn;
  rec->imax = imx;
  REAL depth = mn - mx;
  REAL s = mx + mn;
  F(v3) mid = F(mk)((n.x * s) * (REAL)0.5, (n.y * s) * (REAL)0.5, (n.z * s) * (REAL)0.5);
  for (int i = 0; i < nq; ++i) {
    REAL k = F(dot)(n, F(sub)(q[i], mid));
    q[i] = F(sub)(q[i], F(mk)(k * n.x, k * n.y, k * n.z));
  }
  REAL eps = (sizeof(REAL) == 4) ? (REAL)(FLT_EPSILON * 10) : (REAL)(DBL_EPSILON * 10);
  int nr = 0;
  for (int i = 0; i < nq; ++i) {
    int unique = 1;
    for (int j = 0; j < i; ++j) {
      F(v3) d = F(sub)(q[j], q[i]);
      REAL m = F(rmax)(F(rmax)(F(rabs)(d.x), F(rabs)(d.y)), F(rabs)(d.z));
      if (m < eps) { unique = 0; break; }
    }
    if (unique) {
      REAL* r = rows + 7 * nr++;
      r[0] = q[i].x; r[1] = q[i].y; r[2] = q[i].z;
      r[3] = n.x; r[4] = n.y; r[5] = n.z;
      r[6] = depth;
    }
  }
  rec->ncontacts = nr;
  return nr;
}

#define OR_LOADTET(dst, xyz, tet)                                                            \
  for (int v_ = 0; v_ < 4; ++v_)                                                             \
    dst[v_] = F(mk)((REAL)(xyz)[3 * (size_t)(tet)[v_]], (REAL)(xyz)[3 * (size_t)(tet)[v_] + 1], \
                    (REAL)(xyz)[3 * (size_t)(tet)[v_] + 2]);

static int F(contacts_generic)(const void* xyzA_, const void* xyzB_, int in_double, const uint32_t* tetsA,
                               const uint8_t* surfA, const uint32_t* tetsB, const uint8_t* surfB,
                               int64_t n_pairs, const uint32_t* pairs, int64_t cap, REAL* out,
                               int64_t* n_out, or_record* rec) {
  int64_t n = 0;
  int over = 0;
  REAL rows[7 * OR_NCAND];
  for (int64_t i = 0; i < n_pairs; ++i) {
    uint32_t ta = pairs[2 * i], tb = pairs[2 * i + 1];
    F(v3) A[4], B[4];
    if (in_double) {
      const double* xa = (const double*)xyzA_;
      const double* xb = (const double*)xyzB_;
      OR_LOADTET(A, xa, tetsA + 4 * (size_t)ta);
      OR_LOADTET(B, xb, tetsB + 4 * (size_t)tb);
    } else {
      const float* xa = (const float*)xyzA_;
      const float* xb = (const float*)xyzB_;
      OR_LOADTET(A, xa, tetsA + 4 * (size_t)ta);
      OR_LOADTET(B, xb, tetsB + 4 * (size_t)tb);
    }
    or_record r;
    int nr = F(pair_contacts)(A, B, surfA[ta], surfB[tb], rows, &r);
    if (rec) rec[i] = r;
    for (int k = 0; k < nr; ++k, ++n) {
      if (n < cap) {
        for (int c = 0; c < 7; ++c) out[8 * n + c] = rows[7 * k + c];
        out[8 * n + 7] = (REAL)i;
      } else {
        over = 1;
      }
    }
  }
  *n_out = n;
  return over ? -1 : 0;
}

int F(or_contacts)(const float* xyzA, const uint32_t* tetsA, const uint8_t* surfA, const float* xyzB,
                   const uint32_t* tetsB, const uint8_t* surfB, int64_t n_pairs, const uint32_t* pairs,
                   int64_t cap, REAL* out, int64_t* n_out, or_record* rec) {
  return F(contacts_generic)(xyzA, xyzB, 0, tetsA, surfA, tetsB, surfB, n_pairs, pairs, cap, out, n_out, rec);
}

#undef F
#undef OR_CAT
#undef OR_CAT2
#undef OR_LOADTET
