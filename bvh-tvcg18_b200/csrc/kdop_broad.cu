// kdop_broad.cu -- broad phase: the mesh pairs worth a tandem traversal.
//
// Reference: broad::find_overlaps (SIMULATION/BROAD/BROAD/include/
// broad_find_overlaps.h:44-125 all-pair, :134- grid; both report the same
// set, lexicographically sorted, lower object first).  Each body's box is
// its position +- its bounding radius (prox_rigid_body.h:159-172), the
// radius of a tetramesh the largest |r0| over its rest vertices
// (narrow_shape_types.h:189-206), and two boxes overlap unless one's max is
// strictly below the other's min on some axis.
//
// Here: the radii once per scene (thread per vertex, float max by its bit
// pattern, exact for non-negative values); per query a count pass (thread per
// body i, bodies j > i), an exclusive scan and a write pass that places each
// body's pairs at its offset in j order -- the sorted list without a sort.
#include <algorithm>

#include "kdop_device.cuh"
#include "kdop_sort.h"

namespace kdop {

namespace {

__global__ void radius_kernel(const float4* __restrict__ rest, int64_t nv, unsigned* rbits) {
  int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  float4 r = __ldg(rest + v);
  f3 x = mk3(r.x, r.y, r.z);
  float n = fsqrt(dot3(x, x));  // tiny::norm
  if (n == n) atomicMax(rbits + __float_as_int(r.w), __float_as_uint(n));
}

struct BoxArgs {
  const float4* pos;     // per body: position (x, y, z)
  const unsigned* rbits; // per body: radius bits
  int n;
};

__device__ __forceinline__ void box(const BoxArgs& a, int i, float* lo, float* hi) {
  float4 p = __ldg(a.pos + i);
  float r = __uint_as_float(__ldg(a.rbits + i));
  lo[0] = fsub(p.x, r);
  lo[1] = fsub(p.y, r);
  lo[2] = fsub(p.z, r);
  hi[0] = fadd(p.x, r);
  hi[1] = fadd(p.y, r);
  hi[2] = fadd(p.z, r);
}

__device__ __forceinline__ bool boxes_overlap(const float* la, const float* ha, const float* lb, const float* hb) {
  return !(hb[0] < la[0]) && !(ha[0] < lb[0]) && !(hb[1] < la[1]) && !(ha[1] < lb[1]) && !(hb[2] < la[2]) &&
         !(ha[2] < lb[2]);
}

__global__ void broad_count_kernel(BoxArgs a, unsigned* counts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  float la[3], ha[3];
  box(a, i, la, ha);
  unsigned c = 0;
  for (int j = i + 1; j < a.n; ++j) {
    float lb[3], hb[3];
    box(a, j, lb, hb);
    c += boxes_overlap(la, ha, lb, hb) ? 1u : 0u;
  }
  counts[i] = c;
}

__global__ void broad_write_kernel(BoxArgs a, const unsigned* __restrict__ offsets, uint2* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  float la[3], ha[3];
  box(a, i, la, ha);
  unsigned at = offsets[i];
  for (int j = i + 1; j < a.n; ++j) {
    float lb[3], hb[3];
    box(a, j, lb, hb);
    if (boxes_overlap(la, ha, lb, hb)) out[at++] = make_uint2((unsigned)i, (unsigned)j);
  }
}

__global__ void pack_pos_kernel(const float* __restrict__ pos, int n, float4* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.f);
}

}  // namespace

cudaError_t launch_mesh_radius(kdop_scene* s, unsigned* rbits) {
  cudaError_t e = cudaMemsetAsync(rbits, 0, (size_t)std::max(s->n_meshes, 1) * 4, s->ctx->stream);
  if (e != cudaSuccess || s->nv == 0) return e;
  radius_kernel<<<(unsigned)((s->nv + 255) / 256), 256, 0, s->ctx->stream>>>(s->rest, s->nv, rbits);
  s->ctx->launches++;
  return cudaGetLastError();
}

// Work buffer of a query: counts, offsets, scan scratch, packed positions.
struct BroadWork {
  size_t counts, offsets, scratch, packed, total;
  explicit BroadWork(int n) {
    size_t at = 0;
    auto take = [&](size_t b) {
      size_t o = at;
      at += (b + 255) & ~(size_t)255;
      return o;
    };
    counts = take((size_t)n * 4);
    offsets = take((size_t)n * 4);
    scratch = take(scan_scratch_words(n) * 4);
    packed = take((size_t)n * 16);
    total = at;
  }
};

size_t broad_work_bytes(int n) { return BroadWork(std::max(n, 1)).total; }

// Overlapping body pairs; pos_dev: device n x 3 positions or NULL for the
// scene's poses.  *total = pairs found; they go to `pairs` (device, room for
// cap) when they fit.  Synchronises.
cudaError_t broad_phase(kdop_scene* s, const unsigned* rbits, const float* pos_dev, void* work, uint2* pairs,
                        int64_t cap, int64_t* total) {
  cudaStream_t st = s->ctx->stream;
  const int n = s->n_meshes;
  *total = 0;
  if (n < 2) return cudaSuccess;
  char* w = static_cast<char*>(work);
  BroadWork L(n);
  unsigned* counts = reinterpret_cast<unsigned*>(w + L.counts);
  unsigned* offsets = reinterpret_cast<unsigned*>(w + L.offsets);
  unsigned* scratch = reinterpret_cast<unsigned*>(w + L.scratch);
  float4* packed = reinterpret_cast<float4*>(w + L.packed);
  BoxArgs a;
  a.rbits = rbits;
  a.n = n;
  if (pos_dev) {
    pack_pos_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos_dev, n, packed);
    a.pos = packed;
  } else {
    a.pos = s->pos;
  }
  const unsigned g = (unsigned)((n + 127) / 128);
  broad_count_kernel<<<g, 128, 0, st>>>(a, counts);
  cudaError_t e = exclusive_scan_u32(counts, offsets, n, scratch, st);
  if (e != cudaSuccess) return e;
  unsigned last[2];
  if ((e = cudaMemcpyAsync(&last[0], offsets + n - 1, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(&last[1], counts + n - 1, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  *total = (int64_t)last[0] + last[1];
  s->ctx->launches += pos_dev ? 2 : 1;
  if (*total > cap) return cudaSuccess;
  broad_write_kernel<<<g, 128, 0, st>>>(a, offsets, pairs);
  s->ctx->launches++;
  return cudaGetLastError();
}

}  // namespace kdop
