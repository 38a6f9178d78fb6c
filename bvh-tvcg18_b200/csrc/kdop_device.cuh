// kdop_device.cuh -- device-side building blocks shared by the kernels.
//
// Floating-point rule: every product and sum that decides a kDOP slab, a
// contact decision or a contact value is a separately rounded IEEE operation
// (__fmul_rn / __fadd_rn / __fsub_rn / __fdiv_rn / __fsqrt_rn), in the
// operation order of the reference's TINY vector library
// (tiny_vector_ops_policy.h:33-76), so results match the reference's FP32
// path bit for bit.  The library is also compiled with -fmad=false.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "kdop_internal.h"

namespace kdop {

constexpr uint32_t LEAF_BIT = 0x80000000u;
constexpr uint32_t SURF_BIT = 0x40000000u;   // leaf word: the tet has a boundary face
constexpr uint32_t NODE_MASK = 0x3FFFFFFFu;  // node index bits of a word
constexpr uint32_t NO_NODE = 0xFFFFFFFFu;

// ---- node record ------------------------------------------------------------
// K floats of slabs (lo_s, hi_s interleaved, s = 0..K/2-1, in direction-table
// order), then two topology words, padded to whole float4 chunks.  The words
// carry kdop_tree.h:15-75's (m_start, m_end) in a form the traversal can push
// without decoding:
//   internal node: (c, c + 1), its children c (even) and c + 1;
//   leaf:          (LEAF_BIT | SURF_BIT if the tet has a boundary face | the
//                   leaf's own node index, global tet index).
// So word 0 of a child is exactly the deque entry that stands for it (its
// first child, or itself flagged as a leaf).  Node indices use 30 bits.
//
// Twin records: siblings always sit at node indices 2t, 2t + 1 (the forest
// pads its root level to an even count), and the two records of twin t are
// stored chunk-interleaved: chunk j of node 2t + s is float4 2 NW t + 2 j + s.
// Chunk j of both siblings is therefore one aligned 32-byte word, and a whole
// twin is 2 NW float4 of consecutive memory.
template <int K>
struct NodeLayout {
  static constexpr int NS = K / 2;                 // slabs
  static constexpr int NW = (K + 2 + 3) / 4;       // float4 chunks per record
  static constexpr int TOPO_CHUNK = K / 4;         // chunk holding (start, end)
  static constexpr bool TOPO_ZW = (K % 4) == 2;    // (start,end) in .z,.w (else .x,.y)
  // float4 index of chunk j of node n
  __host__ __device__ static constexpr int64_t at(int64_t n, int j) { return (n >> 1) * (2 * NW) + 2 * j + (n & 1); }
  // topology words of a record's topology chunk
  __device__ static __forceinline__ uint32_t word0(const float4& c) { return __float_as_uint(TOPO_ZW ? c.z : c.x); }
  __device__ static __forceinline__ uint32_t word1(const float4& c) { return __float_as_uint(TOPO_ZW ? c.w : c.y); }
};

// ---- separately rounded float arithmetic --------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }
// std::min / std::max of the reference (first argument kept on ties and NaN)
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 sub3(f3 a, f3 b) { return mk3(fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)); }
__device__ __forceinline__ f3 add3(f3 a, f3 b) { return mk3(fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)); }
__device__ __forceinline__ f3 scl3(f3 a, float s) { return mk3(fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)); }
// ((0 + a0 b0) + a1 b1) + a2 b2
__device__ __forceinline__ float dot3(f3 a, f3 b) {
  float d = fadd(0.0f, fmul(a.x, b.x));
  d = fadd(d, fmul(a.y, b.y));
  return fadd(d, fmul(a.z, b.z));
}
__device__ __forceinline__ f3 cross3(f3 l, f3 r) {
  return mk3(fsub(fmul(l.y, r.z), fmul(l.z, r.y)), fsub(fmul(l.z, r.x), fmul(l.x, r.z)),
             fsub(fmul(l.x, r.y), fmul(l.y, r.x)));
}
// v * (1 / |v|) when |v| > 0
__device__ __forceinline__ f3 unit3(f3 m) {
  float l = fsqrt(dot3(m, m));
  if (l > 0.0f) {
    float inv = fdiv(1.0f, l);
    m = mk3(fmul(m.x, inv), fmul(m.y, inv), fmul(m.z, inv));
  }
  return m;
}

// ---- rigid pose and deformation ------------------------------------------------
// tiny::rotate(q, r) + p = prod(prod(q, r), conj q).imag + p with
// prod(q, r) = (-q.v . r, q.v x r + r q.s) (tiny_quaternion_functions.h:137-152)
// and mul_assign of tiny_quaternion_ops_policy.h:29-38.
__device__ __forceinline__ f3 rotate_translate(float4 q, float4 p, f3 r) {
  f3 v = mk3(q.y, q.z, q.w);
  float s = q.x;
  float a = -dot3(v, r);
  f3 c = cross3(v, r);
  f3 A = mk3(fadd(c.x, fmul(r.x, s)), fadd(c.y, fmul(r.y, s)), fadd(c.z, fmul(r.z, s)));
  f3 B = mk3(-v.x, -v.y, -v.z);
  f3 x = cross3(A, B);
  f3 im = mk3(fadd(fadd(fmul(a, B.x), fmul(A.x, s)), x.x), fadd(fadd(fmul(a, B.y), fmul(A.y, s)), x.y),
              fadd(fadd(fmul(a, B.z), fmul(A.z, s)), x.z));
  return mk3(fadd(im.x, p.x), fadd(im.y, p.y), fadd(im.z, p.z));
}

// The project's own single-precision sine: Cody-Waite reduction by 2 pi
// (6.28125 + remainder), fold into [-pi/2, pi/2], Taylor series to degree 11.
// Identical operation sequence to the CPU oracle's or_sin_f.
__device__ __forceinline__ float own_sin(float x) {
  const float inv2pi = 0.159154936671257019f;
  const float c1 = 6.28125f;
  const float c2 = 0.00193530717f;
  const float pi = 3.14159274101257324f;
  const float hpi = 1.57079637050628662f;
  float k = rintf(fmul(x, inv2pi));
  float r = fsub(x, fmul(k, c1));
  r = fsub(r, fmul(k, c2));
  if (r > hpi) r = fsub(pi, r);
  if (r < -hpi) r = fsub(-pi, r);
  float r2 = fmul(r, r);
  float s = -2.50521083854417188e-8f;
  s = fadd(fmul(s, r2), 2.75573192239858907e-6f);
  s = fadd(fmul(s, r2), -1.98412698412698413e-4f);
  s = fadd(fmul(s, r2), 8.33333333333333333e-3f);
  s = fadd(fmul(s, r2), -1.66666666666666667e-1f);
  s = fmul(s, r2);
  return fadd(r, fmul(r, s));
}

struct Deform {
  float amp, w;
  const float* phase;  // device scalar, advanced per step by the motion kernel
};
__device__ __forceinline__ f3 deform3(f3 r, Deform df) {
  float arg = fadd(fadd(r.x, r.y), r.z);
  arg = fadd(fmul(df.w, arg), *df.phase);
  float d = fmul(df.amp, own_sin(arg));
  return mk3(fadd(r.x, d), fadd(r.y, d), fadd(r.z, d));
}

// Source of world positions for kernels that read vertices.
struct VertexSource {
  const float4* rest;   // .w holds the mesh index (as int bits)
  const float4* world;  // used in mode 0
  const float4* quat;   // per mesh (w, x, y, z)
  const float4* pos;    // per mesh
  Deform deform;
  int mode;             // 0 vertices, 1 pose, 2 deform + pose
};

__device__ __forceinline__ f3 world_vertex(const VertexSource& vs, uint32_t v) {
  if (vs.mode == 0) {
    float4 w = __ldg(vs.world + v);
    return mk3(w.x, w.y, w.z);
  }
  float4 r = __ldg(vs.rest + v);
  int m = __float_as_int(r.w);
  f3 x = mk3(r.x, r.y, r.z);
  if (vs.mode == 2) x = deform3(x, vs.deform);
  return rotate_translate(__ldg(vs.quat + m), __ldg(vs.pos + m), x);
}

}  // namespace kdop
