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
// Two passes.  A thread per candidate tet pair first runs steps 1 and 2 up
// to the first separating axis or the first admissible face pair (almost all
// leaf pairs of a deep overlap stop there: no contact) and lists the pairs
// that go on.  Then one warp handles each listed pair: lanes evaluate the 44
// SAT axes, the 16 face pairs and the 56 contact candidates in parallel;
// ballots keep the reference's candidate order, so the reported rows and
// every value equal the reference's FP32 results.  Both passes evaluate the
// same functions on the same inputs, so their decisions agree.
#include "kdop_device.cuh"

namespace kdop {

// geometry_tetrahedron.h:231-257: face opposite vertex v, outward for a
// positively oriented tet.
__constant__ int8_t c_face[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
// edge table of geometry_contacts_tetrahedron_tetrahedron.h:584-591
__constant__ int8_t c_edge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
// The 36 edge x edge axes of geometry_overlap_tetrahedron_tetrahedron.h:109-287
// in order: A edge, B edge, A vertex left out, B vertex left out of SAT_line.
__constant__ int8_t c_sat[36][4] = {
    {0, 0, 0, 0}, {0, 1, 0, 2}, {0, 2, 0, 3}, {0, 3, 0, 2}, {0, 4, 0, 3}, {0, 5, 0, 3},
    {1, 0, 0, 0}, {1, 1, 0, 0}, {1, 2, 0, 3}, {1, 3, 0, 2}, {1, 4, 0, 3}, {1, 5, 0, 3},
    {2, 0, 0, 0}, {2, 1, 0, 0}, {2, 2, 0, 0}, {2, 3, 0, 2}, {2, 4, 0, 3}, {2, 5, 0, 3},
    {3, 0, 2, 0}, {3, 1, 2, 0}, {3, 2, 2, 0}, {3, 3, 2, 2}, {3, 4, 2, 3}, {3, 5, 2, 3},
    {4, 0, 3, 0}, {4, 1, 3, 0}, {4, 2, 3, 0}, {4, 3, 3, 2}, {4, 4, 3, 3}, {4, 5, 3, 3},
    {5, 0, 3, 0}, {5, 1, 3, 0}, {5, 2, 3, 0}, {5, 3, 3, 2}, {5, 4, 3, 3}, {5, 5, 3, 3}};

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
    f3 p0 = X[c_face[f][0]], p1 = X[c_face[f][1]], p2 = X[c_face[f][2]];
    // make_plane (geometry_plane.h:102-111) and get_signed_distance (:171-175)
    f3 nrm = unit3(cross3(sub3(p1, p0), sub3(p2, p0)));
    float w = dot3(p0, nrm);
    float d0 = fsub(dot3(nrm, Y[0]), w), d1 = fsub(dot3(nrm, Y[1]), w);
    float d2 = fsub(dot3(nrm, Y[2]), w), d3 = fsub(dot3(nrm, Y[3]), w);
    return d0 > 0.f && d1 > 0.f && d2 > 0.f && d3 > 0.f;
  }
  int e = t - 8;
  int ea = c_sat[e][0], eb = c_sat[e][1], xa = c_sat[e][2], xb = c_sat[e][3];
  f3 axis = cross3(sub3(A[c_edge[ea][1]], A[c_edge[ea][0]]), sub3(B[c_edge[eb][1]], B[c_edge[eb][0]]));
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

__device__ __forceinline__ f3 shfl3(f3 v, int src) {
  return mk3(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
             __shfl_sync(0xffffffffu, v.z, src));
}

struct ContactArgs {
  const uint32_t* candA;
  const uint32_t* candB;
  const uint32_t* candP;
  uint32_t* surv;  // candidates past the pre-filter (n_surv of them)
  unsigned cand_cap;
  const uint4* __restrict__ tets;
  const uint8_t* __restrict__ surf;
  VertexSource vs;
  kdop_contact* out;
  int4* rec;
  unsigned out_cap;
  TravCtl* ctl;
};

constexpr int WARPS_PER_BLOCK_C = 8;

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

// Pass 1: thread per candidate.  A pair that fails the SAT test or has no
// admissible face pair gets its empty record here; the others are listed.
__global__ void __launch_bounds__(256) contacts_filter_kernel(ContactArgs a) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const unsigned n_cand = min(*(volatile unsigned*)&a.ctl->n_cand, a.cand_cap);
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_cand; base += stride) {
    const unsigned ci = base + lane;
    bool keep = false;
    if (ci < n_cand) {
      uint32_t ta = a.candA[ci], tb = a.candB[ci];
      uint32_t sa = a.surf[ta], sb = a.surf[tb];
      if (sa != 0u && sb != 0u) {
        uint4 qa = __ldg(a.tets + ta), qb = __ldg(a.tets + tb);
        f3 A[4] = {world_vertex(a.vs, qa.x), world_vertex(a.vs, qa.y), world_vertex(a.vs, qa.z),
                   world_vertex(a.vs, qa.w)};
        f3 B[4] = {world_vertex(a.vs, qb.x), world_vertex(a.vs, qb.y), world_vertex(a.vs, qb.z),
                   world_vertex(a.vs, qb.w)};
        bool sep = false;
        for (int t = 0; t < 44 && !sep; ++t) sep = sat_test(t, A, B);
        if (!sep) {
          UPlane PA[4], PB[4];
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            PA[f] = unscaled_plane(A[c_face[f][0]], A[c_face[f][1]], A[c_face[f][2]]);
            PB[f] = unscaled_plane(B[c_face[f][0]], B[c_face[f][1]], B[c_face[f][2]]);
          }
          float test;
          f3 nA;
          for (int l = 0; l < 16 && !keep; ++l) keep = face_pair_ok(l >> 2, l & 3, sa, sb, PA, PB, A, B, test, nA);
        }
      }
      if (!keep) a.rec[ci] = make_int4(-1, -1, 0, 0);
    }
    unsigned m = __ballot_sync(0xffffffffu, keep);
    if (m) {
      unsigned at = 0;
      if (lane == 0) at = atomicAdd(&a.ctl->n_surv, (unsigned)__popc(m));
      at = __shfl_sync(0xffffffffu, at, 0);
      if (keep) a.surv[at + __popc(m & lt_mask)] = ci;
    }
  }
}

__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK_C) contacts_kernel(ContactArgs a) {
  __shared__ float s_pts[WARPS_PER_BLOCK_C][56][3];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  unsigned n_surv = *(volatile unsigned*)&a.ctl->n_surv;
  unsigned warp = blockIdx.x * WARPS_PER_BLOCK_C + wib;
  unsigned n_warps = gridDim.x * WARPS_PER_BLOCK_C;
  for (unsigned k = warp; k < n_surv; k += n_warps) {
    const unsigned ci = a.surv[k];
    uint32_t ta = a.candA[ci], tb = a.candB[ci];
    int4 record = make_int4(-1, -1, 0, 0);
    uint32_t sa = a.surf[ta], sb = a.surf[tb];
    // vertices: lane l < 8 fetches vertex l (A0..A3, B0..B3)
    uint4 qa = __ldg(a.tets + ta), qb = __ldg(a.tets + tb);
    f3 mine = mk3(0.f, 0.f, 0.f);
    if (lane < 8) {
      uint32_t vid = (lane == 0) ? qa.x : (lane == 1) ? qa.y : (lane == 2) ? qa.z : (lane == 3) ? qa.w
                   : (lane == 4) ? qb.x : (lane == 5) ? qb.y : (lane == 6) ? qb.z : qb.w;
      mine = world_vertex(a.vs, vid);
    }
    f3 A[4], B[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      A[v] = shfl3(mine, v);
      B[v] = shfl3(mine, 4 + v);
    }
    bool ok = (sa != 0u) && (sb != 0u);
    if (ok) {
      // 1. exact overlap
      bool sepr = sat_test(lane, A, B);
      if (lane < 12) sepr = sepr || sat_test(32 + lane, A, B);
      ok = !__any_sync(0xffffffffu, sepr);
    }
    if (ok) {
      // unscaled face planes: lane l < 8 builds plane l (A faces 0-3, B faces 0-3)
      UPlane mp{mk3(0.f, 0.f, 0.f), mk3(0.f, 0.f, 0.f)};
      if (lane < 8) {
        const f3* X = (lane < 4) ? A : B;
        int f = lane & 3;
        mp = unscaled_plane(X[c_face[f][0]], X[c_face[f][1]], X[c_face[f][2]]);
      }
      UPlane PA[4], PB[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        PA[v].n = shfl3(mp.n, v);
        PA[v].p = shfl3(mp.p, v);
        PB[v].n = shfl3(mp.n, 4 + v);
        PB[v].p = shfl3(mp.p, 4 + v);
      }
      // 2. most opposing boundary faces: lane l < 16 -> (a, b) = (l / 4, l % 4)
      float test = 3.0e38f;
      bool good = false;
      f3 nA = mk3(0.f, 0.f, 0.f);
      if (lane < 16) good = face_pair_ok(lane >> 2, lane & 3, sa, sb, PA, PB, A, B, test, nA);
      // first (a, b) in loop order with the smallest value
      float bv = good ? test : 3.0e38f;
      int bl = good ? lane : 64;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        float ov = __shfl_xor_sync(0xffffffffu, bv, o);
        int ol = __shfl_xor_sync(0xffffffffu, bl, o);
        if (ov < bv || (ov == bv && ol < bl)) {
          bv = ov;
          bl = ol;
        }
      }
      if (bl < 64) {
        f3 n = shfl3(nA, bl);
        record.x = bl >> 2;
        record.y = 0;
        // 3. contact candidates, codes lane and lane + 32
        f3 q0, q1;
        bool h0 = candidate(lane, A, B, PA, PB, q0);
        bool h1 = (lane < 24) ? candidate(32 + lane, A, B, PA, PB, q1) : false;
        unsigned m0 = __ballot_sync(0xffffffffu, h0);
        unsigned m1 = __ballot_sync(0xffffffffu, h1);
        int n0 = __popc(m0);
        int nq = n0 + __popc(m1);
        if (nq > 0) {
          int pos0 = __popc(m0 & lt_mask), pos1 = n0 + __popc(m1 & lt_mask);
          float d0 = h0 ? dot3(q0, n) : 0.f, d1 = h1 ? dot3(q1, n) : 0.f;
          // min and max with the position of their first occurrence
          float mnv = 3.0e38f, mxv = -3.0e38f;
          int mnp = 1 << 20, mxp = 1 << 20, mnc = -1, mxc = -1;
          if (h0) {
            mnv = d0; mnp = pos0; mnc = lane;
            mxv = d0; mxp = pos0; mxc = lane;
          }
          if (h1 && (d1 < mnv || !h0)) { mnv = d1; mnp = pos1; mnc = 32 + lane; }
          if (h1 && (mxv < d1 || !h0)) { mxv = d1; mxp = pos1; mxc = 32 + lane; }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            float ov = __shfl_xor_sync(0xffffffffu, mnv, o);
            int op = __shfl_xor_sync(0xffffffffu, mnp, o);
            int oc = __shfl_xor_sync(0xffffffffu, mnc, o);
            if (ov < mnv || (ov == mnv && op < mnp)) { mnv = ov; mnp = op; mnc = oc; }
            ov = __shfl_xor_sync(0xffffffffu, mxv, o);
            op = __shfl_xor_sync(0xffffffffu, mxp, o);
            oc = __shfl_xor_sync(0xffffffffu, mxc, o);
            if (mxv < ov || (ov == mxv && op < mxp)) { mxv = ov; mxp = op; mxc = oc; }
          }
          float depth = fsub(mnv, mxv);
          float ssum = fadd(mxv, mnv);
          f3 mid = mk3(fmul(fmul(n.x, ssum), 0.5f), fmul(fmul(n.y, ssum), 0.5f), fmul(fmul(n.z, ssum), 0.5f));
          if (h0) {
            float k = dot3(n, sub3(q0, mid));
            q0 = sub3(q0, mk3(fmul(k, n.x), fmul(k, n.y), fmul(k, n.z)));
            s_pts[wib][pos0][0] = q0.x; s_pts[wib][pos0][1] = q0.y; s_pts[wib][pos0][2] = q0.z;
          }
          if (h1) {
            float k = dot3(n, sub3(q1, mid));
            q1 = sub3(q1, mk3(fmul(k, n.x), fmul(k, n.y), fmul(k, n.z)));
            s_pts[wib][pos1][0] = q1.x; s_pts[wib][pos1][1] = q1.y; s_pts[wib][pos1][2] = q1.z;
          }
          __syncwarp();
          const float eps = 1.1920928955078125e-06f;  // 10 * FLT_EPSILON
          bool u0 = h0, u1 = h1;
          for (int j = 0; j < nq; ++j) {
            float px = s_pts[wib][j][0], py = s_pts[wib][j][1], pz = s_pts[wib][j][2];
            if (u0 && j < pos0) {
              float m = smax(smax(fabsf(fsub(px, q0.x)), fabsf(fsub(py, q0.y))), fabsf(fsub(pz, q0.z)));
              if (m < eps) u0 = false;
            }
            if (u1 && j < pos1) {
              float m = smax(smax(fabsf(fsub(px, q1.x)), fabsf(fsub(py, q1.y))), fabsf(fsub(pz, q1.z)));
              if (m < eps) u1 = false;
            }
          }
          unsigned um0 = __ballot_sync(0xffffffffu, u0);
          unsigned um1 = __ballot_sync(0xffffffffu, u1);
          int nu0 = __popc(um0), nu = nu0 + __popc(um1);
          unsigned base = 0;
          if (lane == 0) base = atomicAdd(&a.ctl->n_contacts, (unsigned)nu);
          base = __shfl_sync(0xffffffffu, base, 0);
          if (u0) {
            unsigned r = base + __popc(um0 & lt_mask);
            if (r < a.out_cap) {
              kdop_contact c;
              c.p[0] = q0.x; c.p[1] = q0.y; c.p[2] = q0.z;
              c.n[0] = n.x; c.n[1] = n.y; c.n[2] = n.z;
              c.depth = depth;
              c.cand = ci;
              a.out[r] = c;
            }
          }
          if (u1) {
            unsigned r = base + nu0 + __popc(um1 & lt_mask);
            if (r < a.out_cap) {
              kdop_contact c;
              c.p[0] = q1.x; c.p[1] = q1.y; c.p[2] = q1.z;
              c.n[0] = n.x; c.n[1] = n.y; c.n[2] = n.z;
              c.depth = depth;
              c.cand = ci;
              a.out[r] = c;
            }
          }
          record.y = (mnc & 0xFF) | ((mxc & 0xFF) << 8);
          record.z = nu;
          record.w = (int)base;
          __syncwarp();
        }
      }
    }
    if (lane == 0) a.rec[ci] = record;
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
  return vs;
}

cudaError_t launch_contacts(kdop_scene* s) {
  ContactArgs a;
  a.candA = s->cand;
  a.candB = s->cand + s->cand_cap;
  a.candP = s->cand + 2 * s->cand_cap;
  a.surv = s->cand + 3 * s->cand_cap;
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
  contacts_kernel<<<grid, 32 * WARPS_PER_BLOCK_C, 0, s->ctx->stream>>>(a);
  s->ctx->launches += 3;
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
