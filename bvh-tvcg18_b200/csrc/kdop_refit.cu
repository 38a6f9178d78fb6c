// kdop_refit.cu -- bottom-up kDOP refit of every tree of a scene.
//
// Reference: kdop::refit_tree (SIMULATION/KDOP/KDOP/include/kdop_refit_tree.h:
// 24-115 per chunk, 120-162 per tree): a leaf gets make_dop of its tet's four
// vertices (FOUNDATION/GEOMETRY/GEOMETRY/include/types/geometry_dop.h:49-74),
// an internal node make_union of its two children (geometry_make_union.h:
// 10-24).  The OpenCL back-end did one work-group per object with retry loops
// (cl/kernels/kdop_cl_refit_tree.cl:17-168).
//
// Here the forest is stored level by level, so one launch refits one level of
// every tree at once, deepest level first, one thread per node: a leaf poses
// its four vertices once and projects them on all K/2 directions; an internal
// node reads its children's twin record (2 NW consecutive float4, independent
// loads in flight together).  Two sibling threads write the interleaved
// chunks of one twin, so every store instruction fills whole 32-byte sectors.
// In pose or deform mode the refit first poses every vertex once
// (narrow_update_kdop_bvh.h:154-165 on the device, in the same call and the
// same graph) into a scene-owned array the leaves read: posing inside the leaf
// pass would transform each vertex once per tet that uses it (about 24 times
// in a lattice).  The upper levels, too small to fill the GPU, are refitted by
// one block that walks them with block barriers.
#include "kdop_device.cuh"

namespace kdop {

// The record of one node: a leaf projects its tet's four (posed) vertices on
// the K/2 directions (make_dop), an internal node takes the union of its two
// children chunk by chunk (make_union); the topology words are kept.  Chunk
// j of both children is one aligned 32-byte word of their twin record.
template <int K, bool LDG>
__device__ __forceinline__ void refit_node(float4* nodes, int64_t node, const uint4* __restrict__ tets,
                                           const VertexSource& vs, const DirTable& dt) {
  using L = NodeLayout<K>;
  const float4 tc = LDG ? __ldg(nodes + L::at(node, L::TOPO_CHUNK)) : nodes[L::at(node, L::TOPO_CHUNK)];
  const uint32_t w0 = L::word0(tc), w1 = L::word1(tc);
  float w[4 * L::NW];
#pragma unroll
  for (int k = 0; k < 4 * L::NW; ++k) w[k] = 0.f;
  if (w0 & LEAF_BIT) {
    const uint4 t = __ldg(tets + w1);
    const f3 p[4] = {world_vertex(vs, t.x), world_vertex(vs, t.y), world_vertex(vs, t.z), world_vertex(vs, t.w)};
#pragma unroll
    for (int s = 0; s < L::NS; ++s) {
      const f3 d = mk3(dt.d[s][0], dt.d[s][1], dt.d[s][2]);
      float lo = 3.40282346638528859812e+38f, hi = -3.40282346638528859812e+38f;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float pr = dot3(d, p[v]);
        lo = smin(lo, pr);
        hi = smax(hi, pr);
      }
      w[2 * s] = lo;
      w[2 * s + 1] = hi;
    }
  } else {
    const float4* c = nodes + L::at(w0, 0);  // chunk 0 of child w0; child w0 + 1 follows each chunk
#pragma unroll
    for (int j = 0; j < L::NW; ++j) {
      float4 a, b;
      if (LDG) {
        a = __ldg(c + 2 * j);
        b = __ldg(c + 2 * j + 1);
      } else {
        a = c[2 * j];
        b = c[2 * j + 1];
      }
      // lo: min(A.lo, B.lo) = (B < A) ? B : A ; hi: max(A.hi, B.hi) = (A < B) ? B : A
      if (2 * j < L::NS) {
        w[4 * j] = smin(a.x, b.x);
        w[4 * j + 1] = smax(a.y, b.y);
      }
      if (2 * j + 1 < L::NS) {
        w[4 * j + 2] = smin(a.z, b.z);
        w[4 * j + 3] = smax(a.w, b.w);
      }
    }
  }
  w[L::TOPO_ZW ? 4 * L::TOPO_CHUNK + 2 : 4 * L::TOPO_CHUNK] = __uint_as_float(w0);
  w[L::TOPO_ZW ? 4 * L::TOPO_CHUNK + 3 : 4 * L::TOPO_CHUNK + 1] = __uint_as_float(w1);
#pragma unroll
  for (int j = 0; j < L::NW; ++j)
    nodes[L::at(node, j)] = make_float4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
}

// One level of every tree, thread per node.
template <int K>
__global__ void __launch_bounds__(256) refit_level_kernel(float4* nodes, int64_t begin, int64_t count,
                                                          const uint4* __restrict__ tets, VertexSource vs,
                                                          DirTable dt) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  refit_node<K, true>(nodes, begin + t, tets, vs, dt);
}

// Depths [0, top] of every tree: one block per tree.  The block lists its
// tree's nodes of those depths top-down from the root (children from the
// topology words), then refits them bottom-up, a block barrier per depth
// (plain loads: the block reads records it wrote itself; the children of
// depth `top` were refitted by the level launches before it).  One launch
// replaces the per-level launches of the forest's small top levels, each of
// which was bound by launch and load latency.  The padding node that may end
// the root level (a copy of the first root's topology) is refitted by the
// block of the tree rooted at node 0.
constexpr int kTopDepth = 6;
constexpr int kTopNodes = 2 << kTopDepth;  // >= 2^(kTopDepth + 1) - 1 nodes of a tree's top

template <int K>
__global__ void __launch_bounds__(256) refit_top_kernel(float4* nodes, const uint32_t* __restrict__ root, int top,
                                                        uint32_t pad_node, const uint4* __restrict__ tets,
                                                        VertexSource vs, DirTable dt) {
  using L = NodeLayout<K>;
  __shared__ uint32_t ids[kTopNodes];
  __shared__ int lev[kTopDepth + 2];  // nodes of depth d: ids[lev[d] .. lev[d + 1])
  __shared__ int fill;
  const uint32_t r = root[blockIdx.x];
  if (r == NO_NODE) return;  // empty mesh: the whole block leaves
  if (threadIdx.x == 0) {
    ids[0] = r;
    lev[0] = 0;
    lev[1] = 1;
    fill = 1;
  }
  __syncthreads();
  for (int d = 0; d < top; ++d) {
    const int b = lev[d], e = lev[d + 1];
    for (int i = b + (int)threadIdx.x; i < e; i += blockDim.x) {
      const uint32_t w0 = L::word0(__ldg(nodes + L::at(ids[i], L::TOPO_CHUNK)));
      if (!(w0 & LEAF_BIT)) {
        const int at = atomicAdd(&fill, 2);
        ids[at] = w0 & NODE_MASK;
        ids[at + 1] = (w0 & NODE_MASK) + 1u;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) lev[d + 2] = fill;
    __syncthreads();
  }
  for (int d = top; d >= 0; --d) {
    for (int i = lev[d] + (int)threadIdx.x; i < lev[d + 1]; i += blockDim.x)
      refit_node<K, false>(nodes, ids[i], tets, vs, dt);
    if (d == 0 && r == 0u && pad_node != NO_NODE && threadIdx.x == blockDim.x - 1)
      refit_node<K, false>(nodes, pad_node, tets, vs, dt);
    __syncthreads();
  }
}

// Topology words into the node records, slabs zeroed.  topo holds the
// reference's (m_start, m_end) per node (leaf <=> start == end = tet).
template <int K>
__global__ void write_topology_kernel(float4* nodes, int64_t nn, const uint32_t* __restrict__ topo,
                                      const uint8_t* __restrict__ surf) {
  using L = NodeLayout<K>;
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn * L::NW) return;
  int64_t node = 2 * (t / (2 * L::NW)) + (t & 1);
  int j = (int)((t % (2 * L::NW)) >> 1);
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
  if (j == L::TOPO_CHUNK) {
    uint32_t st = topo[2 * node], en = topo[2 * node + 1];
    if (st == en) {
      en = st;
      st = LEAF_BIT | (surf[en] ? SURF_BIT : 0u) | (uint32_t)node;
    }
    float a = __uint_as_float(st), b = __uint_as_float(en);
    if (L::TOPO_ZW) {
      o.z = a;
      o.w = b;
    } else {
      o.x = a;
      o.y = b;
    }
  }
  nodes[t] = o;
}

// World positions of all vertices (pose / deform modes), for read-back.
__global__ void world_kernel(int64_t nv, VertexSource vs, float4* out) {
  int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  f3 x = world_vertex(vs, (uint32_t)v);
  out[v] = make_float4(x.x, x.y, x.z, 0.f);
}

// One step of rigid motion per mesh and of the deformation phase:
// p += v, q = normalise(q + 0.5 (0, w) q).
__global__ void motion_kernel(int n_meshes, float4* quat, float4* pos, const float4* __restrict__ lin,
                              const float4* __restrict__ ang, float* phase, float phase_rate) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) *phase = *phase + phase_rate;
  if (m >= n_meshes) return;
  float4 p = pos[m], v = lin[m], q = quat[m], w = ang[m];
  p.x += v.x;
  p.y += v.y;
  p.z += v.z;
  // dq = 0.5 * (0, w) (x) q
  float dw = -(w.x * q.y + w.y * q.z + w.z * q.w);
  float dx = w.x * q.x + (w.y * q.w - w.z * q.z);
  float dy = w.y * q.x + (w.z * q.y - w.x * q.w);
  float dz = w.z * q.x + (w.x * q.z - w.y * q.y);
  q.x += 0.5f * dw;
  q.y += 0.5f * dx;
  q.z += 0.5f * dy;
  q.w += 0.5f * dz;
  float inv = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q.x *= inv;
  q.y *= inv;
  q.z *= inv;
  q.w *= inv;
  quat[m] = q;
  pos[m] = p;
}

// xyz triples -> float4 (w = mesh index bits when with_mesh_id >= 0, else 0)
__global__ void pack3_kernel(const float* __restrict__ in, float4* out, int64_t n, const float4* __restrict__ keep_w,
                             int keep) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float w = keep ? keep_w[i].w : 0.f;
  out[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], w);
}
__global__ void pack4_kernel(const float* __restrict__ in, float4* out, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_float4(in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]);
}

cudaError_t launch_pack3(kdop_scene* s, const float* in, float4* out, int64_t n, int with_mesh_id) {
  if (n <= 0) return cudaSuccess;
  pack3_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->ctx->stream>>>(in, out, n, s->rest, with_mesh_id >= 0);
  s->ctx->launches++;
  return cudaGetLastError();
}
cudaError_t launch_pack4(kdop_scene* s, const float* in, float4* out, int64_t n) {
  if (n <= 0) return cudaSuccess;
  pack4_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->ctx->stream>>>(in, out, n);
  s->ctx->launches++;
  return cudaGetLastError();
}

static VertexSource vertex_source(kdop_scene* s, int mode) {
  VertexSource vs;
  vs.rest = s->rest;
  vs.world = s->world;
  vs.quat = s->quat;
  vs.pos = s->pos;
  vs.deform.amp = s->amp;
  vs.deform.w = s->w;
  vs.deform.phase = s->phase_dev;
  vs.mode = mode;
  return vs;
}


template <int K>
static cudaError_t refit_impl(kdop_scene* s, int mode) {
  VertexSource vs = vertex_source(s, mode);
  if (mode != KDOP_REFIT_VERTICES && s->nv > 0) {
    // pose (and deform) every vertex once; the leaves then read world
    // positions instead of transforming each vertex once per tet using it
    world_kernel<<<(unsigned)((s->nv + 255) / 256), 256, 0, s->ctx->stream>>>(s->nv, vs, s->posed);
    s->ctx->launches++;
    vs = vertex_source(s, KDOP_REFIT_VERTICES);
    vs.world = s->posed;
  }
  int levels = (int)s->level_off.size() - 1;
  if (levels <= 0) return cudaSuccess;
  // depths [0, top] of every tree in one launch (a block per tree), the
  // deeper levels one launch each, deepest first
  const int top = std::min(kTopDepth, levels - 1);
  for (int d = levels - 1; d > top; --d) {
    int64_t b = s->level_off[d], n = s->level_off[d + 1] - b;
    unsigned grid = (unsigned)((n + 255) / 256);
    refit_level_kernel<K><<<grid, 256, 0, s->ctx->stream>>>(s->nodes, b, n, s->tets, vs, s->dirs);
    s->ctx->launches++;
  }
  // the root level holds one padding node after the real roots when their
  // count is odd
  int64_t n_roots = 0;
  for (int m = 0; m < s->n_meshes; ++m) n_roots += (s->t_off[m + 1] > s->t_off[m]) ? 1 : 0;
  const uint32_t pad = (s->level_off[1] - s->level_off[0] > n_roots) ? (uint32_t)(s->level_off[1] - 1) : NO_NODE;
  refit_top_kernel<K><<<(unsigned)s->n_meshes, 256, 0, s->ctx->stream>>>(s->nodes, s->root_dev, top, pad, s->tets,
                                                                         vs, s->dirs);
  s->ctx->launches++;
  return cudaGetLastError();
}

cudaError_t launch_refit(kdop_scene* s, int mode) {
  switch (s->K) {
    case 6: return refit_impl<6>(s, mode);
    case 8: return refit_impl<8>(s, mode);
    case 12: return refit_impl<12>(s, mode);
    case 14: return refit_impl<14>(s, mode);
    case 18: return refit_impl<18>(s, mode);
    case 20: return refit_impl<20>(s, mode);
    case 26: return refit_impl<26>(s, mode);
  }
  return cudaErrorInvalidValue;
}

template <int K>
static cudaError_t topo_impl(kdop_scene* s, const uint32_t* topo) {
  int64_t items = s->nn * NodeLayout<K>::NW;
  if (items == 0) return cudaSuccess;
  write_topology_kernel<K><<<(unsigned)((items + 255) / 256), 256, 0, s->ctx->stream>>>(s->nodes, s->nn, topo, s->surf);
  s->ctx->launches++;
  return cudaGetLastError();
}

cudaError_t launch_write_topology(kdop_scene* s, const uint32_t* topo) {
  switch (s->K) {
    case 6: return topo_impl<6>(s, topo);
    case 8: return topo_impl<8>(s, topo);
    case 12: return topo_impl<12>(s, topo);
    case 14: return topo_impl<14>(s, topo);
    case 18: return topo_impl<18>(s, topo);
    case 20: return topo_impl<20>(s, topo);
    case 26: return topo_impl<26>(s, topo);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_world(kdop_scene* s, int mode, float4* out) {
  if (s->nv == 0) return cudaSuccess;
  VertexSource vs = vertex_source(s, mode);
  world_kernel<<<(unsigned)((s->nv + 255) / 256), 256, 0, s->ctx->stream>>>(s->nv, vs, out);
  s->ctx->launches++;
  return cudaGetLastError();
}

cudaError_t launch_motion(kdop_scene* s) {
  int n = s->n_meshes > 0 ? s->n_meshes : 1;
  motion_kernel<<<(n + 127) / 128, 128, 0, s->ctx->stream>>>(s->n_meshes, s->quat, s->pos, s->lin_vel, s->ang_vel,
                                                              s->phase_dev, s->phase_rate);
  s->ctx->launches++;
  return cudaGetLastError();
}

}  // namespace kdop
