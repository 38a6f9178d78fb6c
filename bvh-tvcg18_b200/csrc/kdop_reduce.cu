// kdop_reduce.cu -- contact point reduction on the device.
//
// Reference: the fourth phase of prox::collision_detection
// (SIMULATION/PROX/PROX/include/prox_collision_detection.h:341-350):
// std::sort of the contact points by ContactPoint::operator<
// (prox_contact_point.h:135-194: body i, body j, p.y, p.x, p.z, n.y, n.x, n.z,
// depth, each compared by float `<`), then std::unique with
// ContactPoint::operator== (:91-133: same bodies and every component with
// |new - kept| not above working_precision<float>() = 10 FLT_EPSILON,
// FOUNDATION/TINY/TINY/include/tiny_precision.h:21-24), which keeps a row
// only when it differs from the last row kept.
//
// Here: five stable LSD radix sorts of 64-bit keys build the order (the least
// significant field pair first; floats mapped to integers that order like
// float `<`, -0 folded onto +0).  The unique is sequential by definition (a
// row is compared with the last row kept, not with its predecessor, and the
// tolerance is not transitive), but a row whose p.y exceeds its
// predecessor's by more than the tolerance, or whose bodies differ, can equal
// no earlier row (rounded subtraction is monotonic, so every earlier p.y is
// further away), so the sorted rows split into independent segments there;
// one thread walks each segment.  A scan of the keep flags compacts them.
#include <algorithm>

#include "kdop_device.cuh"
#include "kdop_internal.h"
#include "kdop_sort.h"

namespace kdop {

namespace {

// Integer image of a float that orders like float `<` (NaN aside); -0 and +0
// map to the same value.
__device__ __forceinline__ uint32_t ord_key(float f) {
  uint32_t u = __float_as_uint(f);
  if ((u << 1) == 0u) u = 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void red_iota_kernel(uint32_t* perm, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = (uint32_t)i;
}

// Key of one LSD pass for the row at perm[i]; pass 0 is the least significant
// (n.z, depth), pass 4 the most (body i, body j).
__global__ void red_keys_kernel(const kdop_contact* __restrict__ rows, const uint2* __restrict__ bodies,
                                const uint32_t* __restrict__ perm, int64_t n, int pass, uint64_t* keys) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = perm[i];
  const kdop_contact c = rows[r];
  uint64_t hi = 0, lo = 0;
  switch (pass) {
    case 0: hi = ord_key(c.n[2]); lo = ord_key(c.depth); break;
    case 1: hi = ord_key(c.n[1]); lo = ord_key(c.n[0]); break;
    case 2: hi = ord_key(c.p[0]); lo = ord_key(c.p[2]); break;
    case 3: lo = ord_key(c.p[1]); break;
    default: {
      const uint2 b = bodies[r];
      hi = b.x;
      lo = b.y;
    }
  }
  keys[i] = (hi << 32) | lo;
}

// brk[i] = 1 where a segment starts (first row, new bodies, or a p.y gap
// above the tolerance); brk[n] = 0 so a scan over n + 1 ends with the count.
__global__ void red_breaks_kernel(const kdop_contact* __restrict__ rows, const uint2* __restrict__ bodies,
                                  const uint32_t* __restrict__ perm, int64_t n, float eps, uint32_t* brk) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  uint32_t b = 0;
  if (i == 0) {
    b = 1;
  } else if (i < n) {
    const uint32_t r = perm[i], q = perm[i - 1];
    const uint2 br = bodies[r], bq = bodies[q];
    b = (br.x != bq.x || br.y != bq.y || fabsf(fsub(rows[r].p[1], rows[q].p[1])) > eps) ? 1u : 0u;
  }
  brk[i] = b;
}

__global__ void red_starts_kernel(const uint32_t* __restrict__ brk, const uint32_t* __restrict__ seg, int64_t n,
                                  uint32_t* starts) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && brk[i]) starts[seg[i]] = (uint32_t)i;
}

// ContactPoint::operator== between the last kept row and a new one (bodies
// equal within a segment): no component differs by more than eps.  A NaN
// difference is not "more than eps", as in the reference.
__device__ __forceinline__ bool same_point(const kdop_contact& k, const kdop_contact& c, float eps) {
  return !(fabsf(fsub(c.p[1], k.p[1])) > eps) && !(fabsf(fsub(c.p[0], k.p[0])) > eps) &&
         !(fabsf(fsub(c.p[2], k.p[2])) > eps) && !(fabsf(fsub(c.n[1], k.n[1])) > eps) &&
         !(fabsf(fsub(c.n[0], k.n[0])) > eps) && !(fabsf(fsub(c.n[2], k.n[2])) > eps) &&
         !(fabsf(fsub(c.depth, k.depth)) > eps);
}

// Thread per segment: std::unique's walk (keep a row unless it equals the
// last row kept).  keep[n] = 0 for the compaction scan.
__global__ void red_walk_kernel(const kdop_contact* __restrict__ rows, const uint32_t* __restrict__ perm,
                                const uint32_t* __restrict__ starts, int64_t n_seg, int64_t n, float eps,
                                uint32_t* keep) {
  int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) keep[n] = 0u;
  if (s >= n_seg) return;
  const int64_t a = starts[s], e = (s + 1 < n_seg) ? (int64_t)starts[s + 1] : n;
  kdop_contact last = rows[perm[a]];
  keep[a] = 1u;
  for (int64_t j = a + 1; j < e; ++j) {
    const kdop_contact c = rows[perm[j]];
    const bool eq = same_point(last, c, eps);
    keep[j] = eq ? 0u : 1u;
    if (!eq) last = c;
  }
}

__global__ void red_write_kernel(const kdop_contact* __restrict__ rows, const uint2* __restrict__ bodies,
                                 const uint32_t* __restrict__ perm, const uint32_t* __restrict__ keep,
                                 const uint32_t* __restrict__ pos, int64_t n, kdop_contact* out, uint2* out_bodies) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  const uint32_t r = perm[i];
  out[pos[i]] = rows[r];
  if (out_bodies) out_bodies[pos[i]] = bodies[r];
}

// Bodies (mesh of A, mesh of B) of each contact row of a scene: the row's
// candidate, its pair, the pair's meshes.
__global__ void red_scene_bodies_kernel(const kdop_contact* __restrict__ rows, int64_t n,
                                        const uint32_t* __restrict__ cand_pair, const uint2* __restrict__ pairs,
                                        uint2* bodies) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bodies[i] = pairs[cand_pair[rows[i].cand]];
}

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Work buffer of a reduction of n rows (256-byte aligned pieces).
struct ReduceWork {
  size_t keys, keys_tmp, perm, perm_tmp, radix, brk, seg, starts, keep, pos, scan, total;
  explicit ReduceWork(int64_t n) {
    size_t at = 0;
    auto take = [&](size_t b) {
      size_t o = at;
      at += (b + 255) & ~(size_t)255;
      return o;
    };
    const size_t m = (size_t)std::max<int64_t>(n, 1);
    keys = take(m * 8);
    keys_tmp = take(m * 8);
    perm = take(m * 4);
    perm_tmp = take(m * 4);
    radix = take(radix_scratch_words((int64_t)m) * 4);
    brk = take((m + 1) * 4);
    seg = take((m + 1) * 4);
    starts = take(m * 4);
    keep = take((m + 1) * 4);
    pos = take((m + 1) * 4);
    scan = take(scan_scratch_words((int64_t)m + 1) * 4);
    total = at;
  }
};

size_t reduce_work_bytes(int64_t n) { return ReduceWork(n).total; }

cudaError_t scene_contact_bodies(kdop_scene* s, int64_t n, uint2* bodies) {
  if (n <= 0) return cudaSuccess;
  red_scene_bodies_kernel<<<blocks_for(n, 256), 256, 0, s->ctx->stream>>>(s->contacts, n, s->cand + 2 * s->cand_cap,
                                                                           s->pairs, bodies);
  s->ctx->launches++;
  return cudaGetLastError();
}

// Reduces n rows (device) with their bodies (device); the kept rows go to out
// (and their bodies to out_bodies, may be NULL) in the reduced order; *n_out
// = rows kept.  Synchronises (the radix sort reads its key bits back).
cudaError_t reduce_contact_rows(kdop_ctx* ctx, const kdop_contact* rows, const uint2* bodies, int64_t n, void* work,
                                kdop_contact* out, uint2* out_bodies, int64_t* n_out) {
  cudaStream_t st = ctx->stream;
  *n_out = 0;
  if (n <= 0) return cudaSuccess;
  if (n >= ((int64_t)1 << 32) - 1) return cudaErrorInvalidValue;
  ReduceWork L(n);
  char* w = static_cast<char*>(work);
  uint64_t* keys = reinterpret_cast<uint64_t*>(w + L.keys);
  uint64_t* keys_tmp = reinterpret_cast<uint64_t*>(w + L.keys_tmp);
  uint32_t* perm = reinterpret_cast<uint32_t*>(w + L.perm);
  uint32_t* perm_tmp = reinterpret_cast<uint32_t*>(w + L.perm_tmp);
  uint32_t* radix = reinterpret_cast<uint32_t*>(w + L.radix);
  uint32_t* brk = reinterpret_cast<uint32_t*>(w + L.brk);
  uint32_t* seg = reinterpret_cast<uint32_t*>(w + L.seg);
  uint32_t* starts = reinterpret_cast<uint32_t*>(w + L.starts);
  uint32_t* keep = reinterpret_cast<uint32_t*>(w + L.keep);
  uint32_t* pos = reinterpret_cast<uint32_t*>(w + L.pos);
  uint32_t* scan = reinterpret_cast<uint32_t*>(w + L.scan);
  const float eps = 1.19209290e-07f * 10.0f;  // working_precision<float>()
  const unsigned g = blocks_for(n, 256), g1 = blocks_for(n + 1, 256);
  red_iota_kernel<<<g, 256, 0, st>>>(perm, n);
  ctx->launches++;
  cudaError_t e;
  for (int pass = 0; pass < 5; ++pass) {
    red_keys_kernel<<<g, 256, 0, st>>>(rows, bodies, perm, n, pass, keys);
    ctx->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = radix_sort_pairs(keys, perm, keys_tmp, perm_tmp, n, radix, st)) != cudaSuccess) return e;
  }
  red_breaks_kernel<<<g1, 256, 0, st>>>(rows, bodies, perm, n, eps, brk);
  ctx->launches++;
  if ((e = exclusive_scan_u32(brk, seg, n + 1, scan, st)) != cudaSuccess) return e;
  red_starts_kernel<<<g, 256, 0, st>>>(brk, seg, n, starts);
  ctx->launches++;
  uint32_t n_seg = 0;
  if ((e = cudaMemcpyAsync(&n_seg, seg + n, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  red_walk_kernel<<<blocks_for(std::max<int64_t>(n_seg, 1), 128), 128, 0, st>>>(rows, perm, starts, n_seg, n, eps,
                                                                                   keep);
  ctx->launches++;
  if ((e = exclusive_scan_u32(keep, pos, n + 1, scan, st)) != cudaSuccess) return e;
  red_write_kernel<<<g, 256, 0, st>>>(rows, bodies, perm, keep, pos, n, out, out_bodies);
  ctx->launches++;
  uint32_t kept = 0;
  if ((e = cudaMemcpyAsync(&kept, pos + n, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  *n_out = kept;
  return cudaGetLastError();
}

}  // namespace kdop
