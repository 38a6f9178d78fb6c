// kdop_contacts.cu -- tet-tet contact generation and its adjoint.
//
// Reference: contacts_tetrahedron_tetrahedron(A, B, cb, sA, sB,
// MOST_OPPOSING_SURFACES) (FOUNDATION/GEOMETRY/GEOMETRY/include/contacts/
// geometry_contacts_tetrahedron_tetrahedron.h:1313-1345), the default of
// kdop_select_contact_point_algorithm.h:30:
//   1. exact SAT overlap of the two tets (overlap/
//      geometry_overlap_tetrahedron_tetrahedron.h:51-290),
//   2. contact normal = unit normal of A's boundary face in the most opposing
//      pair of boundary faces (:465-533),
//   3. candidates = vertices of one tet inside the other and edge/face-plane
//      crossings inside the other tet (:544-620), depth = min - max of p.n over
//      all candidates, points projected on the mid plane, near-duplicates
//      (max-norm < 10 FLT_EPSILON) dropped, reported in order (:622-681).
//
// Three passes, a thread per candidate tet pair in each.  The first two run
// steps 1 and 2 up to the first separating axis or the first admissible face
// pair (almost all leaf pairs of a deep overlap stop there: no contact) --
// the 8 face axes of the SAT test in the first, the 36 edge axes and the
// face-pair search in the second, on the pairs the first lists densely -- and
// list the pairs that go on; the third runs step 2's argmin and step 3 for
// the listed pairs in the reference's order (face pairs, then the 56
// candidates in generation order), so the reported rows and every value equal
// the reference's FP32 results.  All passes evaluate the same functions on
// the same inputs, so their decisions agree.  Vertex positions are the world
// positions the last refit used (after a pose / deform refit, the array it
// computed).  (A warp-per-pair form, lanes over
// SAT axes, face pairs and candidates with ballots keeping the order, took
// 1.5x longer on contact-rich pairs: most phases kept few lanes busy.)
#include "kdop_device.cuh"

namespace kdop {

// geometry_tetrahedron.h:231-257: face opposite vertex v, outward for a
// positively oriented tet.
__constant__ int8_t c_face[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
// edge table of geometry_contacts_tetrahedron_tetrahedron.h:584-591
__constant__ int8_t c_edge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
// The face and edge tables as compile-time values, and the 36 edge x edge
// axes of geometry_overlap_tetrahedron_tetrahedron.h:109-287 in order (A
// edge, B edge, A vertex left out, B vertex left out of SAT_line): in loops
// unrolled over faces, edges or SAT axes the indices fold to constants, so a
// tet's vertices and planes stay in registers instead of an indexed array in
// local memory (the contact filter and edge passes: 0.17 -> 0.14 ms and 0.39
// -> 0.32 ms on config 3).
__device__ __forceinline__ int face_vtx(int f, int k) {
  constexpr int8_t t[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
  return t[f][k];
}
__device__ __forceinline__ int edge_vtx(int e, int k) {
  constexpr int8_t t[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  return t[e][k];
}
__device__ __forceinline__ int sat_entry(int e, int k) {
  constexpr int8_t t[36][4] = {
      {0, 0, 0, 0}, {0, 1, 0, 2}, {0, 2, 0, 3}, {0, 3, 0, 2}, {0, 4, 0, 3}, {0, 5, 0, 3},
      {1, 0, 0, 0}, {1, 1, 0, 0}, {1, 2, 0, 3}, {1, 3, 0, 2}, {1, 4, 0, 3}, {1, 5, 0, 3},
      {2, 0, 0, 0}, {2, 1, 0, 0}, {2, 2, 0, 0}, {2, 3, 0, 2}, {2, 4, 0, 3}, {2, 5, 0, 3},
      {3, 0, 2, 0}, {3, 1, 2, 0}, {3, 2, 2, 0}, {3, 3, 2, 2}, {3, 4, 2, 3}, {3, 5, 2, 3},
      {4, 0, 3, 0}, {4, 1, 3, 0}, {4, 2, 3, 0}, {4, 3, 3, 2}, {4, 4, 3, 3}, {4, 5, 3, 3},
      {5, 0, 3, 0}, {5, 1, 3, 0}, {5, 2, 3, 0}, {5, 3, 3, 2}, {5, 4, 3, 3}, {5, 5, 3, 3}};
  return t[e][k];
}

struct UPlane {
  f3 n, p;
};

// make_unscaled_plane (…_tetrahedron_tetrahedron.h:31-62)
__device__ __forceinline__ UPlane unscaled_plane(f3 p0, f3 p1, f3 p2) {
  f3 m0 = cross3(sub3(p1, p0), sub3(p2, p0));
  f3 m1 = cross3(sub3(p2, p1), sub3(p0, p1));
  f3 m2 = cross3(sub3(p0, p2), sub3(p1, p2));
  float l0 = dot3(m0, m0), l1 = dot3(m1, m1), l2 = dot3(m2, m2);
  UPlane pl{m0, p0};
  if (l0 >= l1 && l0 >= l2) pl = UPlane{m0, p0};
  if (l1 >= l0 && l1 >= l2) pl = UPlane{m1, p1};
  if (l2 >= l1 && l2 >= l0) pl = UPlane{m2, p2};
  return pl;
}
__device__ __forceinline__ float sdist(f3 q, const UPlane& pl) { return dot3(pl.n, sub3(q, pl.p)); }
__device__ __forceinline__ bool inside4(f3 q, const UPlane* pl) {
  float d0 = sdist(q, pl[0]), d1 = sdist(q, pl[1]), d2 = sdist(q, pl[2]), d3 = sdist(q, pl[3]);
  return !(d0 > 0.f) && !(d1 > 0.f) && !(d2 > 0.f) && !(d3 > 0.f);
}
__device__ __forceinline__ bool crossing(f3 a, f3 b, const UPlane& pl) {
  float dA = sdist(a, pl), dB = sdist(b, pl);
  if (dA >= 0.f && dB >= 0.f) return false;
  if (dA <= 0.f && dB <= 0.f) return false;
  return true;
}
__device__ __forceinline__ f3 intersect(f3 a, f3 b, const UPlane& pl) {
  float dA = fabsf(sdist(a, pl)), dB = fabsf(sdist(b, pl));
  float t = fdiv(dA, fadd(dA, dB));
  return add3(a, scl3(sub3(b, a), t));
}

// Contact candidate `c` (0..55) in the reference's generation order.
__device__ __forceinline__ bool candidate(int c, const f3* A, const f3* B, const UPlane* PA, const UPlane* PB,
                                          f3& q) {
  if (c < 8) {
    int v = c >> 1;
    if (!(c & 1)) {
      if (!inside4(B[v], PA)) return false;
      q = B[v];
    } else {
      if (!inside4(A[v], PB)) return false;
      q = A[v];
    }
    return true;
  }
  int e = (c - 8) >> 3, p = ((c - 8) >> 1) & 3;
  int i = c_edge[e][0], j = c_edge[e][1];
  if (!(c & 1)) {
    if (!crossing(B[i], B[j], PA[p])) return false;
    f3 x = intersect(B[i], B[j], PA[p]);
    if (!inside4(x, PA)) return false;
    q = x;
  } else {
    if (!crossing(A[i], A[j], PB[p])) return false;
    f3 x = intersect(A[i], A[j], PB[p]);
    if (!inside4(x, PB)) return false;
    q = x;
  }
  return true;
}

// One of the 44 SAT tests; true = separating.
__device__ __forceinline__ bool sat_test(int t, const f3* A, const f3* B) {
  if (t < 8) {
    const f3* X = (t < 4) ? A : B;  // plane owner
    const f3* Y = (t < 4) ? B : A;  // tested points
    int f = t & 3;
    f3 p0 = X[face_vtx(f, 0)], p1 = X[face_vtx(f, 1)], p2 = X[face_vtx(f, 2)];
    // make_plane (geometry_plane.h:102-111) and get_signed_distance (:171-175)
    f3 nrm = unit3(cross3(sub3(p1, p0), sub3(p2, p0)));
    float w = dot3(p0, nrm);
    float d0 = fsub(dot3(nrm, Y[0]), w), d1 = fsub(dot3(nrm, Y[1]), w);
    float d2 = fsub(dot3(nrm, Y[2]), w), d3 = fsub(dot3(nrm, Y[3]), w);
    return d0 > 0.f && d1 > 0.f && d2 > 0.f && d3 > 0.f;
  }
  int e = t - 8;
  int ea = sat_entry(e, 0), eb = sat_entry(e, 1), xa = sat_entry(e, 2), xb = sat_entry(e, 3);
  f3 axis = cross3(sub3(A[edge_vtx(ea, 1)], A[edge_vtx(ea, 0)]), sub3(B[edge_vtx(eb, 1)], B[edge_vtx(eb, 0)]));
  // SAT_line (geometry_overlap_tetrahedron_tetrahedron.h:14-47) over the 3
  // vertices of each tet other than the one left out, in index order
  float s[3], u[3];
  int k = 0;
#pragma unroll
  for (int v = 0; v < 4; ++v)
    if (v != xa) s[k++] = dot3(axis, A[v]);
  k = 0;
#pragma unroll
  for (int v = 0; v < 4; ++v)
    if (v != xb) u[k++] = dot3(axis, B[v]);
  float lo_s = smin(smin(s[0], s[1]), s[2]), hi_s = smax(smax(s[0], s[1]), s[2]);
  float lo_u = smin(smin(u[0], u[1]), u[2]), hi_u = smax(smax(u[0], u[1]), u[2]);
  return (hi_s < lo_u) || (lo_s > hi_u);
}

struct ContactArgs {
  const uint32_t* candA;
  const uint32_t* candB;
  const uint32_t* candP;
  uint32_t* surv;  // candidates past the pre-filter (n_surv of them)
  uint32_t* mid;   // candidates past the face axes of the SAT test (n_mid of them)
  unsigned cand_cap;
  const uint4* __restrict__ tets;
  const uint8_t* __restrict__ surf;
  VertexSource vs;
  kdop_contact* out;
  int4* rec;
  unsigned out_cap;
  TravCtl* ctl;
};

// Face pair (fa, fb) admissible as the most opposing pair (…_tetrahedron_
// tetrahedron.h:465-533): both boundary faces, opposing unit normals, and
// each tet's opposite vertex not behind the other's face plane.
__device__ __forceinline__ bool face_pair_ok(int fa, int fb, uint32_t sa, uint32_t sb, const UPlane* PA,
                                             const UPlane* PB, const f3* A, const f3* B, float& test, f3& nA) {
  if (!(((sa >> fa) & 1u) && ((sb >> fb) & 1u))) return false;
  const UPlane& pa = PA[fa];
  const UPlane& pb = PB[fb];
  nA = unit3(pa.n);
  f3 nB = unit3(pb.n);
  float t = dot3(nA, nB);
  if (!(t < 0.f)) return false;
  float tA = dot3(pa.n, sub3(B[fb], pa.p));
  float tB = dot3(pb.n, sub3(A[fa], pb.p));
  if ((tA < 0.f) || (tB < 0.f)) return false;
  test = t;
  return true;
}

// Tets ta and tb of a candidate, posed.
__device__ __forceinline__ void candidate_tets(const ContactArgs& a, uint32_t ta, uint32_t tb, f3* A, f3* B) {
  const uint4 qa = __ldg(a.tets + ta), qb = __ldg(a.tets + tb);
  A[0] = world_vertex(a.vs, qa.x);
  A[1] = world_vertex(a.vs, qa.y);
  A[2] = world_vertex(a.vs, qa.z);
  A[3] = world_vertex(a.vs, qa.w);
  B[0] = world_vertex(a.vs, qb.x);
  B[1] = world_vertex(a.vs, qb.y);
  B[2] = world_vertex(a.vs, qb.z);
  B[3] = world_vertex(a.vs, qb.w);
}

// Appends the warp's kept candidates to a list (one atomic per warp).
__device__ __forceinline__ void warp_append(bool keep, unsigned ci, unsigned* counter, uint32_t* list, int lane) {
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (m) {
    unsigned at = 0;
    if (lane == 0) at = atomicAdd(counter, (unsigned)__popc(m));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (keep) list[at + __popc(m & ((1u << lane) - 1u))] = ci;
  }
}

// Pass 1a: thread per candidate, the surface check and the 8 face axes of the
// SAT test.  A pair they reject gets its empty record here; the others are
// listed for pass 1b, so that the 36 edge axes run on dense warps.  The SAT
// verdict is an OR over all 44 axes, so splitting the axes leaves it as it is.
__global__ void __launch_bounds__(256) contacts_filter_kernel(ContactArgs a) {
  const int lane = threadIdx.x & 31;
  const unsigned n_cand = min(*(volatile unsigned*)&a.ctl->n_cand, a.cand_cap);
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_cand; base += stride) {
    const unsigned ci = base + lane;
    bool keep = false;
    if (ci < n_cand) {
      const uint32_t ta = a.candA[ci], tb = a.candB[ci];
      if (a.surf[ta] != 0u && a.surf[tb] != 0u) {
        f3 A[4], B[4];
        candidate_tets(a, ta, tb, A, B);
        bool sep = false;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (!sep) sep = sat_test(t, A, B);
        keep = !sep;
      }
      if (!keep) a.rec[ci] = make_int4(-1, -1, 0, 0);
    }
    warp_append(keep, ci, &a.ctl->n_mid, a.mid, lane);
  }
}

// Pass 1b: thread per candidate past the face axes: the 36 edge axes of the
// SAT test, then the search for an admissible face pair.  A pair that fails
// gets its empty record here; the others are listed for pass 2.
__global__ void __launch_bounds__(256) contacts_edge_kernel(ContactArgs a) {
  const int lane = threadIdx.x & 31;
  const unsigned n_mid = *(volatile unsigned*)&a.ctl->n_mid;
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_mid; base += stride) {
    const unsigned k = base + lane;
    bool keep = false;
    unsigned ci = 0;
    if (k < n_mid) {
      ci = a.mid[k];
      const uint32_t ta = a.candA[ci], tb = a.candB[ci];
      const uint32_t sa = a.surf[ta], sb = a.surf[tb];
      f3 A[4], B[4];
      candidate_tets(a, ta, tb, A, B);
      bool sep = false;
#pragma unroll
      for (int t = 8; t < 44; ++t)
        if (!sep) sep = sat_test(t, A, B);
      if (!sep) {
        UPlane PA[4], PB[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          PA[f] = unscaled_plane(A[face_vtx(f, 0)], A[face_vtx(f, 1)], A[face_vtx(f, 2)]);
          PB[f] = unscaled_plane(B[face_vtx(f, 0)], B[face_vtx(f, 1)], B[face_vtx(f, 2)]);
        }
        float test;
        f3 nA;
#pragma unroll
        for (int l = 0; l < 16; ++l)
          if (!keep) keep = face_pair_ok(l >> 2, l & 3, sa, sb, PA, PB, A, B, test, nA);
      }
      if (!keep) a.rec[ci] = make_int4(-1, -1, 0, 0);
    }
    warp_append(keep, ci, &a.ctl->n_surv, a.surv, lane);
  }
}

// Pass 2, thread per listed pair: the argmin over the 16 face pairs by a
// strict < in loop order (first occurrence), the 56 candidates in generation
// order with running min / max of p.n (first occurrence), projection on the
// mid plane, and the duplicate test of each candidate against every earlier
// one.  Rows of a warp are placed with one atomic.
__global__ void __launch_bounds__(128) contacts_thread_kernel(ContactArgs a) {
  const int lane = threadIdx.x & 31;
  const unsigned n_surv = *(volatile unsigned*)&a.ctl->n_surv;
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_surv; base += stride) {
    const unsigned k = base + lane;
    const bool act = k < n_surv;
    unsigned ci = 0;
    int4 record = make_int4(-1, -1, 0, 0);
    int nq = 0, nu = 0;
    float depth = 0.f;
    f3 n = mk3(0.f, 0.f, 0.f);
    float px[56], py[56], pz[56];
    uint64_t kept = 0;
    if (act) {
      ci = a.surv[k];
      const uint32_t ta = a.candA[ci], tb = a.candB[ci];
      const uint32_t sa = a.surf[ta], sb = a.surf[tb];
      const uint4 qa = __ldg(a.tets + ta), qb = __ldg(a.tets + tb);
      f3 A[4] = {world_vertex(a.vs, qa.x), world_vertex(a.vs, qa.y), world_vertex(a.vs, qa.z),
                 world_vertex(a.vs, qa.w)};
      f3 B[4] = {world_vertex(a.vs, qb.x), world_vertex(a.vs, qb.y), world_vertex(a.vs, qb.z),
                 world_vertex(a.vs, qb.w)};
      UPlane PA[4], PB[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        PA[f] = unscaled_plane(A[c_face[f][0]], A[c_face[f][1]], A[c_face[f][2]]);
        PB[f] = unscaled_plane(B[c_face[f][0]], B[c_face[f][1]], B[c_face[f][2]]);
      }
      float bv = 3.0e38f;
      int bl = -1;
      for (int l = 0; l < 16; ++l) {
        float t;
        f3 nA;
        if (face_pair_ok(l >> 2, l & 3, sa, sb, PA, PB, A, B, t, nA) && t < bv) {
          bv = t;
          bl = l;
          n = nA;
        }
      }
      if (bl >= 0) {
        record.x = bl >> 2;
        record.y = 0;
        float mnv = 0.f, mxv = 0.f;
        int mnc = -1, mxc = -1;
        for (int c = 0; c < 56; ++c) {
          f3 q;
          if (!candidate(c, A, B, PA, PB, q)) continue;
          const float d = dot3(q, n);
          if (nq == 0 || d < mnv) { mnv = d; mnc = c; }
          if (nq == 0 || mxv < d) { mxv = d; mxc = c; }
          px[nq] = q.x;
          py[nq] = q.y;
          pz[nq] = q.z;
          ++nq;
        }
        if (nq > 0) {
          depth = fsub(mnv, mxv);
          const float ssum = fadd(mxv, mnv);
          const f3 mid = mk3(fmul(fmul(n.x, ssum), 0.5f), fmul(fmul(n.y, ssum), 0.5f), fmul(fmul(n.z, ssum), 0.5f));
          const float eps = 1.1920928955078125e-06f;  // 10 * FLT_EPSILON
          for (int i = 0; i < nq; ++i) {
            f3 q = mk3(px[i], py[i], pz[i]);
            const float kk = dot3(n, sub3(q, mid));
            q = sub3(q, mk3(fmul(kk, n.x), fmul(kk, n.y), fmul(kk, n.z)));
            px[i] = q.x;
            py[i] = q.y;
            pz[i] = q.z;
            bool u = true;
            for (int j = 0; j < i && u; ++j) {
              float m = smax(smax(fabsf(fsub(px[j], q.x)), fabsf(fsub(py[j], q.y))), fabsf(fsub(pz[j], q.z)));
              if (m < eps) u = false;
            }
            if (u) {
              kept |= 1ull << i;
              ++nu;
            }
          }
          record.y = (mnc & 0xFF) | ((mxc & 0xFF) << 8);
          record.z = nu;
        }
      }
    }
    // rows of the warp: one atomic
    int incl = nu;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned wbase = 0;
    if (lane == 0 && total > 0) wbase = atomicAdd(&a.ctl->n_contacts, (unsigned)total);
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    if (act) {
      if (nu > 0) {
        unsigned r = wbase + (unsigned)(incl - nu);
        record.w = (int)r;
        for (int i = 0; i < nq; ++i) {
          if (!((kept >> i) & 1ull)) continue;
          if (r < a.out_cap) {
            kdop_contact c;
            c.p[0] = px[i]; c.p[1] = py[i]; c.p[2] = pz[i];
            c.n[0] = n.x; c.n[1] = n.y; c.n[2] = n.z;
            c.depth = depth;
            c.cand = ci;
            a.out[r] = c;
          }
          ++r;
        }
      }
      a.rec[ci] = record;
    }
  }
}

// ---- adjoint -------------------------------------------------------------------
// Frozen-decision depth d = q_min . n - q_max . n with n = m / |m|, m the
// cross product of A's chosen face; q a vertex or an edge/plane crossing
// a + (b - a) t, t = |sA| / (|sA| + |sB|), s = m_p . (x - F0) for the face
// plane p of the other tet.  In exact arithmetic the three corner cross
// products of make_unscaled_plane coincide and every corner lies on the
// plane, so the first corner stands for the chosen one.  The inputs and the
// gradient are float; the chain rule runs in double, because near-parallel
// edge/plane crossings (dA + dB small) amplify rounding by orders of
// magnitude.
struct d3 {
  double x, y, z;
};
__device__ __forceinline__ d3 dmk(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 dof(f3 v) { return d3{(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ d3 dsub(d3 a, d3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ d3 dadd(d3 a, d3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ d3 dscl(d3 a, double s) { return dmk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 dcross(d3 l, d3 r) {
  return dmk(l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x);
}
__device__ __forceinline__ void dacc(d3* g, int i, d3 v) { g[i] = dadd(g[i], v); }

__device__ __forceinline__ d3 face_m(const d3* T, int f, d3& F0) {
  F0 = T[c_face[f][0]];
  return dcross(dsub(T[c_face[f][1]], F0), dsub(T[c_face[f][2]], F0));
}

// adjoint of m = (P1 - P0) x (P2 - P0) for face f of T into gT
__device__ void face_m_adj(const d3* T, int f, d3 gm, d3* gT) {
  int i0 = c_face[f][0], i1 = c_face[f][1], i2 = c_face[f][2];
  d3 u = dsub(T[i1], T[i0]), w = dsub(T[i2], T[i0]);
  d3 gu = dcross(w, gm), gw = dcross(gm, u);
  dacc(gT, i1, gu);
  dacc(gT, i2, gw);
  dacc(gT, i0, dscl(dadd(gu, gw), -1.0));
}

__device__ d3 cand_point(int c, const d3* A, const d3* B) {
  if (c < 8) return (c & 1) ? A[c >> 1] : B[c >> 1];
  int e = (c - 8) >> 3, p = ((c - 8) >> 1) & 3;
  const d3* E = (c & 1) ? A : B;
  const d3* T = (c & 1) ? B : A;
  d3 a = E[c_edge[e][0]], b = E[c_edge[e][1]], F0;
  d3 m = face_m(T, p, F0);
  double dA = fabs(ddot(m, dsub(a, F0))), dB = fabs(ddot(m, dsub(b, F0)));
  double t = dA / (dA + dB);
  return dadd(a, dscl(dsub(b, a), t));
}

__device__ void cand_adj(int c, const d3* A, const d3* B, d3 gq, d3* gA, d3* gB) {
  if (c < 8) {
    dacc((c & 1) ? gA : gB, c >> 1, gq);
    return;
  }
  int e = (c - 8) >> 3, p = ((c - 8) >> 1) & 3;
  const d3* E = (c & 1) ? A : B;
  const d3* T = (c & 1) ? B : A;
  d3* gE = (c & 1) ? gA : gB;
  d3* gT = (c & 1) ? gB : gA;
  int ia = c_edge[e][0], ib = c_edge[e][1];
  d3 a = E[ia], b = E[ib], F0;
  d3 m = face_m(T, p, F0);
  double sA = ddot(m, dsub(a, F0)), sB = ddot(m, dsub(b, F0));
  double sgA = sA < 0.0 ? -1.0 : 1.0, sgB = sB < 0.0 ? -1.0 : 1.0;
  double dA = fabs(sA), dB = fabs(sB), S = dA + dB;
  double t = dA / S;
  // q = a + (b - a) t
  dacc(gE, ia, dscl(gq, 1.0 - t));
  dacc(gE, ib, dscl(gq, t));
  double gt = ddot(gq, dsub(b, a));
  double gdA = gt * dB / (S * S), gdB = -gt * dA / (S * S);
  // dA = sgA m.(a - F0), dB = sgB m.(b - F0)
  dacc(gE, ia, dscl(m, sgA * gdA));
  dacc(gE, ib, dscl(m, sgB * gdB));
  dacc(gT, c_face[p][0], dscl(dadd(dscl(m, sgA * gdA), dscl(m, sgB * gdB)), -1.0));
  d3 gm = dadd(dscl(dsub(a, F0), sgA * gdA), dscl(dsub(b, F0), sgB * gdB));
  face_m_adj(T, p, gm, gT);
}

struct AdjointArgs {
  const uint32_t* candA;
  const uint32_t* candB;
  unsigned cand_cap;
  const uint4* __restrict__ tets;
  const int4* __restrict__ rec;
  const float* dd;
  const float* dn;
  unsigned out_cap;
  VertexSource vs;
  float* grad;
  TravCtl* ctl;
};

__global__ void __launch_bounds__(128) adjoint_kernel(AdjointArgs a) {
  unsigned n_cand = min(*(volatile unsigned*)&a.ctl->n_cand, a.cand_cap);
  for (unsigned ci = blockIdx.x * blockDim.x + threadIdx.x; ci < n_cand; ci += gridDim.x * blockDim.x) {
    int4 r = a.rec[ci];
    if (r.z <= 0 || r.x < 0) continue;
    double gd = 0.0;
    d3 gn = dmk(0.0, 0.0, 0.0);
    for (int k = 0; k < r.z; ++k) {
      unsigned row = (unsigned)r.w + (unsigned)k;
      if (row >= a.out_cap) break;
      gd += (double)a.dd[row];
      if (a.dn) gn = dadd(gn, dmk(a.dn[3 * row], a.dn[3 * row + 1], a.dn[3 * row + 2]));
    }
    uint4 qa = __ldg(a.tets + a.candA[ci]), qb = __ldg(a.tets + a.candB[ci]);
    uint32_t va[4] = {qa.x, qa.y, qa.z, qa.w}, vb[4] = {qb.x, qb.y, qb.z, qb.w};
    d3 A[4], B[4], gA[4], gB[4];
    for (int v = 0; v < 4; ++v) {
      A[v] = dof(world_vertex(a.vs, va[v]));
      B[v] = dof(world_vertex(a.vs, vb[v]));
      gA[v] = gB[v] = dmk(0.0, 0.0, 0.0);
    }
    int imin = r.y & 0xFF, imax = (r.y >> 8) & 0xFF;
    d3 F0;
    d3 m = face_m(A, r.x, F0);
    double len = sqrt(ddot(m, m));
    d3 n = dscl(m, 1.0 / len);
    d3 qmin = cand_point(imin, A, B), qmax = cand_point(imax, A, B);
    // depth = qmin . n - qmax . n
    cand_adj(imin, A, B, dscl(n, gd), gA, gB);
    cand_adj(imax, A, B, dscl(n, -gd), gA, gB);
    d3 gnt = dadd(gn, dscl(dsub(qmin, qmax), gd));
    d3 gm = dscl(dsub(gnt, dscl(n, ddot(n, gnt))), 1.0 / len);
    face_m_adj(A, r.x, gm, gA);
    for (int v = 0; v < 4; ++v) {
      atomicAdd(a.grad + 3 * (size_t)va[v], (float)gA[v].x);
      atomicAdd(a.grad + 3 * (size_t)va[v] + 1, (float)gA[v].y);
      atomicAdd(a.grad + 3 * (size_t)va[v] + 2, (float)gA[v].z);
      atomicAdd(a.grad + 3 * (size_t)vb[v], (float)gB[v].x);
      atomicAdd(a.grad + 3 * (size_t)vb[v] + 1, (float)gB[v].y);
      atomicAdd(a.grad + 3 * (size_t)vb[v] + 2, (float)gB[v].z);
    }
  }
}

__global__ void contacts_reset_kernel(TravCtl* c) {
  if (threadIdx.x == 0) {
    c->n_contacts = 0;
    c->n_surv = 0;
    c->n_mid = 0;
  }
}

static VertexSource vsrc(kdop_scene* s) {
  VertexSource vs;
  vs.rest = s->rest;
  vs.world = s->world;
  vs.quat = s->quat;
  vs.pos = s->pos;
  vs.deform.amp = s->amp;
  vs.deform.w = s->w;
  vs.deform.phase = s->phase_dev;
  vs.mode = s->refit_mode < 0 ? 0 : s->refit_mode;
  if (vs.mode != KDOP_REFIT_VERTICES) {
    // the world positions the last pose / deform refit computed (and traversed)
    vs.mode = KDOP_REFIT_VERTICES;
    vs.world = s->posed;
  }
  return vs;
}

cudaError_t launch_contacts(kdop_scene* s) {
  ContactArgs a;
  a.candA = s->cand;
  a.candB = s->cand + s->cand_cap;
  a.candP = s->cand + 2 * s->cand_cap;
  a.surv = s->cand + 3 * s->cand_cap;
  a.mid = s->cand + 4 * s->cand_cap;
  a.cand_cap = (unsigned)s->cand_cap;
  a.tets = s->tets;
  a.surf = s->surf;
  a.vs = vsrc(s);
  a.out = s->contacts;
  a.rec = s->records;
  a.out_cap = (unsigned)s->contact_cap;
  a.ctl = s->ctl;
  contacts_reset_kernel<<<1, 32, 0, s->ctx->stream>>>(s->ctl);
  unsigned grid = (unsigned)s->ctx->sm_count * 8u;
  contacts_filter_kernel<<<grid, 256, 0, s->ctx->stream>>>(a);
  contacts_edge_kernel<<<grid, 256, 0, s->ctx->stream>>>(a);
  contacts_thread_kernel<<<grid * 2, 128, 0, s->ctx->stream>>>(a);
  s->ctx->launches += 4;
  return cudaGetLastError();
}

cudaError_t launch_adjoint(kdop_scene* s, const float* dd, const float* dn, float* grad) {
  AdjointArgs a;
  a.candA = s->cand;
  a.candB = s->cand + s->cand_cap;
  a.cand_cap = (unsigned)s->cand_cap;
  a.tets = s->tets;
  a.rec = s->records;
  a.dd = dd;
  a.dn = dn;
  a.out_cap = (unsigned)s->contact_cap;
  a.vs = vsrc(s);
  a.grad = grad;
  a.ctl = s->ctl;
  unsigned grid = (unsigned)s->ctx->sm_count * 8u;
  adjoint_kernel<<<grid, 128, 0, s->ctx->stream>>>(a);
  s->ctx->launches += 1;
  return cudaGetLastError();
}

}  // namespace kdop
