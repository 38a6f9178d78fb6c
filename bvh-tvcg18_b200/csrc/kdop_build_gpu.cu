// kdop_build_gpu.cu -- the scene's trees built on the GPU.
//
// Same trees as the host build (kdop_build.cpp) and the reference's
// mesh_reorder + make_tree (kdop_mesh_reorder.h:173-353, kdop_make_tree.h:
// 191-288):
//   * leaf order: Morton codes of the tets' rest centroids with the
//     reference's arithmetic (float sums scaled by the double 0.25, 21-bit
//     quantisation with an integer scale, the initial maximum FLT_MIN),
//     sorted per mesh by the device radix sort.  A stable sort breaks equal
//     codes by tet index, std::sort in its own way, so a mesh with equal
//     codes (or a degenerate scale) takes the host's std::sort order instead;
//   * topology: a function of the tet counts alone.  The index-median split
//     makes every tree complete down to depth L = floor(log2 n), plus the
//     children of the size-2 nodes of depth L; a node's tet range follows
//     from its heap index (one halving per level), its place in the level
//     from the ranges to its left, so one thread per node writes its
//     (m_start, m_end) directly.
#include <algorithm>
#include <cfloat>
#include <cstring>

#include "kdop_device.cuh"
#include "kdop_sort.h"

namespace kdop {

namespace {

// float <-> unsigned key with the order of the float values
__device__ __forceinline__ uint32_t ordered(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ int mesh_of(const float4* __restrict__ rest, uint32_t v) {
  return __float_as_int(__ldg(rest + v).w);
}

// centroid of kdop_mesh_reorder.h: ((x0 + x1) + x2) + x3 in float, times the double 0.25
__device__ __forceinline__ f3 centroid(const float4* __restrict__ rest, uint4 t) {
  float4 a = __ldg(rest + t.x), b = __ldg(rest + t.y), c = __ldg(rest + t.z), d = __ldg(rest + t.w);
  float sx = fadd(fadd(fadd(a.x, b.x), c.x), d.x);
  float sy = fadd(fadd(fadd(a.y, b.y), c.y), d.y);
  float sz = fadd(fadd(fadd(a.z, b.z), c.z), d.z);
  return mk3((float)(0.25 * (double)sx), (float)(0.25 * (double)sy), (float)(0.25 * (double)sz));
}

// per mesh: ordered min of the centroids (3 words), ordered max (3 words)
__global__ void bounds_kernel(const uint4* __restrict__ tets, const float4* __restrict__ rest, int64_t nt,
                              uint32_t* mm) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool ok = t < nt;
  int m = -1;
  f3 c = mk3(0.f, 0.f, 0.f);
  if (ok) {
    uint4 q = __ldg(tets + t);
    m = mesh_of(rest, q.x);
    c = centroid(rest, q);
  }
  const int lane = threadIdx.x & 31;
  int m0 = __shfl_sync(0xffffffffu, m, 0);
  bool uniform = __all_sync(0xffffffffu, ok && m == m0);
  // NaN centroids are skipped, as the reference's std::min / std::max skip them
  uint32_t k[6];
  const float cv[3] = {c.x, c.y, c.z};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const bool nan = !(cv[j] == cv[j]);
    k[j] = nan || !ok ? 0xFFFFFFFFu : ordered(cv[j]);
    k[j + 3] = nan || !ok ? 0u : ordered(cv[j]);
  }
  if (uniform) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        uint32_t y = __shfl_xor_sync(0xffffffffu, k[j], o);
        k[j] = j < 3 ? min(k[j], y) : max(k[j], y);
      }
    if (lane == 0)
#pragma unroll
      for (int j = 0; j < 6; ++j) j < 3 ? atomicMin(&mm[6 * m0 + j], k[j]) : atomicMax(&mm[6 * m0 + j], k[j]);
  } else if (ok) {
#pragma unroll
    for (int j = 0; j < 6; ++j) j < 3 ? atomicMin(&mm[6 * m + j], k[j]) : atomicMax(&mm[6 * m + j], k[j]);
  }
}

__global__ void bounds_init_kernel(uint32_t* mm, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 6 * n) mm[i] = (i % 6) < 3 ? 0xFFFFFFFFu : 0u;
}

struct MortonParam {
  float mn[3];
  float scale;  // (float) of the integer scale
};

__device__ __forceinline__ uint64_t spread3(uint64_t x) {
  // bit k of x to bit 3k (21 bits)
  x &= 0x1FFFFFull;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// code = interleave(x, y, z) with x on bit 3k, y on 3k + 1, z on 3k + 2
__global__ void codes_kernel(const uint4* __restrict__ tets, const float4* __restrict__ rest, int64_t nt,
                             const MortonParam* __restrict__ prm, uint64_t* codes, uint64_t* keys, uint32_t* vals) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  uint4 q = __ldg(tets + t);
  MortonParam p = prm[mesh_of(rest, q.x)];
  f3 c = centroid(rest, q);
  uint64_t x = (uint64_t)(float)__float2int_rz(fmul(fsub(c.x, p.mn[0]), p.scale));
  uint64_t y = (uint64_t)(float)__float2int_rz(fmul(fsub(c.y, p.mn[1]), p.scale));
  uint64_t z = (uint64_t)(float)__float2int_rz(fmul(fsub(c.z, p.mn[2]), p.scale));
  uint64_t code = spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
  codes[t] = code;
  keys[t] = code;
  vals[t] = (uint32_t)t;
}

__global__ void mesh_keys_kernel(const uint4* __restrict__ tets, const float4* __restrict__ rest,
                                 const uint32_t* __restrict__ vals, int64_t nt, uint64_t* keys) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nt) keys[i] = (uint64_t)(uint32_t)mesh_of(rest, __ldg(tets + vals[i]).x);
}

// equal neighbouring codes within a mesh
__global__ void ties_kernel(const uint4* __restrict__ tets, const float4* __restrict__ rest,
                            const uint32_t* __restrict__ vals, const uint64_t* __restrict__ codes, int64_t nt,
                            uint32_t* tied) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 1 || i >= nt) return;
  uint32_t a = vals[i - 1], b = vals[i];
  int ma = mesh_of(rest, __ldg(tets + a).x), mb = mesh_of(rest, __ldg(tets + b).x);
  if (ma == mb && codes[a] == codes[b]) tied[ma] = 1u;
}

// range (first, size) of heap node h at depth d of a tree over n leaves
__device__ __forceinline__ void heap_range(uint32_t n, int d, uint64_t h, uint32_t& f, uint32_t& s) {
  f = 0;
  s = n;
  for (int k = d - 1; k >= 0; --k) {
    uint32_t left = s - (s >> 1);
    if ((h >> k) & 1ull) {
      f += left;
      s >>= 1;
    } else {
      s = left;
    }
  }
}

// size-2 nodes before heap node p at depth L (where sizes are 1 or 2)
__device__ __forceinline__ uint32_t twos_before(uint32_t n, int L, uint64_t p) {
  uint32_t f, s;
  heap_range(n, L, p, f, s);
  return f - (uint32_t)(p - (1ull << L));
}

struct TopoArgs {
  int64_t nn;
  int levels;
  int nm;
  int64_t n_roots;                  // real roots (the root level may hold one padding node)
  const int64_t* __restrict__ level_off;
  const int64_t* __restrict__ pre;  // levels x (nm + 1)
  const int64_t* __restrict__ ntet;
  const int32_t* __restrict__ lg;
  const int64_t* __restrict__ t_off;
  int first_tree;                   // the tree whose root the padding node repeats
  const uint32_t* __restrict__ perm;
  uint32_t* topo;
};

__global__ void topology_kernel(TopoArgs a) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.nn) return;
  int d = 0;
  while (d + 1 < a.levels && a.level_off[d + 1] <= g) ++d;
  int64_t li = g - a.level_off[d];
  const int64_t* P = a.pre + (int64_t)d * (a.nm + 1);
  int m;
  if (d == 0 && li >= a.n_roots) {
    m = a.first_tree;  // padding node: a copy of the first root
    li = P[m];
  } else {
    int lo = 0, hi = a.nm - 1;  // largest m with P[m] <= li
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (P[mid] <= li) lo = mid;
      else hi = mid - 1;
    }
    m = lo;
  }
  const int64_t i = li - P[m];
  const uint32_t n = (uint32_t)a.ntet[m];
  const int L = a.lg[m];
  uint64_t h;
  if (d <= L) {
    h = (1ull << d) + (uint64_t)i;
  } else {
    // depth L + 1: child (i & 1) of the (i >> 1)-th size-2 node of depth L
    const uint32_t j = (uint32_t)(i >> 1);
    uint64_t lo = 1ull << L, hi = (2ull << L) - 1;  // smallest p with twos_before(p) + (size(p) == 2) > j
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      uint32_t f, s;
      heap_range(n, L, mid, f, s);
      uint32_t c = f - (uint32_t)(mid - (1ull << L)) + (s == 2u ? 1u : 0u);
      if (c > j) hi = mid;
      else lo = mid + 1;
    }
    h = 2 * lo + (uint64_t)(i & 1);
  }
  uint32_t f, s;
  heap_range(n, d, h, f, s);
  uint32_t w0, w1;
  if (s <= 1u) {
    w0 = w1 = a.perm[a.t_off[m] + f];
  } else {
    int64_t ic = (d + 1 <= L) ? 2 * i : 2 * (int64_t)twos_before(n, L, h);
    int64_t c = a.level_off[d + 1] + a.pre[(int64_t)(d + 1) * (a.nm + 1) + m] + ic;
    w0 = (uint32_t)c;
    w1 = (uint32_t)(c + 1);
  }
  a.topo[2 * g] = w0;
  a.topo[2 * g + 1] = w1;
}

float ordered_to_float(uint32_t k) {
  uint32_t b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

}  // namespace

cudaError_t device_morton_perm(kdop_scene* s, uint32_t* perm, std::vector<char>& need_host) {
  cudaStream_t st = s->ctx->stream;
  const int64_t nt = s->nt;
  const int nm = s->n_meshes;
  need_host.assign((size_t)nm, 0);
  if (nt <= 0) return cudaSuccess;
  // scratch: mm (6 nm words) | tied (nm) | params (nm) | codes, keys, keys_tmp (nt u64) | vals_tmp (nt) | radix
  const size_t radix_words = radix_scratch_words(nt);
  size_t bytes = 0;
  auto take = [&](size_t b) {
    size_t o = bytes;
    bytes += (b + 255) & ~(size_t)255;
    return o;
  };
  const size_t o_mm = take((size_t)6 * nm * 4), o_tied = take((size_t)nm * 4),
               o_prm = take((size_t)nm * sizeof(MortonParam)), o_codes = take((size_t)nt * 8),
               o_keys = take((size_t)nt * 8), o_ktmp = take((size_t)nt * 8), o_vtmp = take((size_t)nt * 4),
               o_rad = take(radix_words * 4);
  char* w = nullptr;
  cudaError_t e = cudaMalloc((void**)&w, bytes);
  if (e != cudaSuccess) return e;
  uint32_t* mm = reinterpret_cast<uint32_t*>(w + o_mm);
  uint32_t* tied = reinterpret_cast<uint32_t*>(w + o_tied);
  MortonParam* prm = reinterpret_cast<MortonParam*>(w + o_prm);
  uint64_t* codes = reinterpret_cast<uint64_t*>(w + o_codes);
  uint64_t* keys = reinterpret_cast<uint64_t*>(w + o_keys);
  uint64_t* ktmp = reinterpret_cast<uint64_t*>(w + o_ktmp);
  uint32_t* vtmp = reinterpret_cast<uint32_t*>(w + o_vtmp);
  uint32_t* rad = reinterpret_cast<uint32_t*>(w + o_rad);
  const unsigned g = (unsigned)((nt + 255) / 256);
  do {
    bounds_init_kernel<<<(6 * nm + 255) / 256, 256, 0, st>>>(mm, nm);
    bounds_kernel<<<g, 256, 0, st>>>(s->tets, s->rest, nt, mm);
    std::vector<uint32_t> hmm((size_t)6 * nm);
    if ((e = cudaMemcpyAsync(hmm.data(), mm, hmm.size() * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) break;
    std::vector<MortonParam> hp((size_t)nm);
    for (int m = 0; m < nm; ++m) {
      if (s->t_off[m + 1] == s->t_off[m]) continue;
      // the reference's running min from FLT_MAX and max from FLT_MIN
      float mn[3], mx[3];
      for (int d = 0; d < 3; ++d) {
        float lo = ordered_to_float(hmm[6 * m + d]), hi = ordered_to_float(hmm[6 * m + 3 + d]);
        mn[d] = std::min(std::numeric_limits<float>::max(), lo);
        mx[d] = std::max(std::numeric_limits<float>::min(), hi);
      }
      int scale = 0;
      if (!morton_scale(mn, mx, scale)) need_host[m] = 1;
      for (int d = 0; d < 3; ++d) hp[m].mn[d] = mn[d];
      hp[m].scale = (float)scale;
    }
    if ((e = cudaMemcpyAsync(prm, hp.data(), (size_t)nm * sizeof(MortonParam), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
      break;
    codes_kernel<<<g, 256, 0, st>>>(s->tets, s->rest, nt, prm, codes, keys, perm);
    if ((e = radix_sort_pairs(keys, perm, ktmp, vtmp, nt, rad, st)) != cudaSuccess) break;
    mesh_keys_kernel<<<g, 256, 0, st>>>(s->tets, s->rest, perm, nt, keys);
    if ((e = radix_sort_pairs(keys, perm, ktmp, vtmp, nt, rad, st)) != cudaSuccess) break;
    if ((e = cudaMemsetAsync(tied, 0, (size_t)nm * 4, st)) != cudaSuccess) break;
    ties_kernel<<<g, 256, 0, st>>>(s->tets, s->rest, perm, codes, nt, tied);
    std::vector<uint32_t> ht((size_t)nm);
    if ((e = cudaMemcpyAsync(ht.data(), tied, (size_t)nm * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) break;
    for (int m = 0; m < nm; ++m)
      if (ht[m]) need_host[m] = 1;
    s->ctx->launches += 7;
    e = cudaGetLastError();
  } while (0);
  cudaStreamSynchronize(st);
  cudaFree(w);
  return e;
}

cudaError_t device_topology(kdop_scene* s, const ForestBuild& fb, const std::vector<int64_t>& pre,
                            const std::vector<int32_t>& lg, const uint32_t* perm, uint32_t* topo) {
  cudaStream_t st = s->ctx->stream;
  const int nm = s->n_meshes;
  const int levels = (int)fb.level_off.size() - 1;
  const int64_t nn = levels > 0 ? fb.level_off[levels] : 0;
  if (nn <= 0) return cudaSuccess;
  // device copies: level_off | pre | ntet | lg | t_off
  std::vector<int64_t> ntet((size_t)nm);
  for (int m = 0; m < nm; ++m) ntet[m] = s->t_off[m + 1] - s->t_off[m];
  size_t n64 = fb.level_off.size() + pre.size() + ntet.size() + s->t_off.size();
  std::vector<int64_t> buf;
  buf.reserve(n64);
  buf.insert(buf.end(), fb.level_off.begin(), fb.level_off.end());
  buf.insert(buf.end(), pre.begin(), pre.end());
  buf.insert(buf.end(), ntet.begin(), ntet.end());
  buf.insert(buf.end(), s->t_off.begin(), s->t_off.end());
  char* w = nullptr;
  size_t bytes = n64 * 8 + (size_t)nm * 4 + 16;
  cudaError_t e = cudaMalloc((void**)&w, bytes);
  if (e != cudaSuccess) return e;
  int64_t* d64 = reinterpret_cast<int64_t*>(w);
  int32_t* dlg = reinterpret_cast<int32_t*>(w + n64 * 8);
  e = cudaMemcpyAsync(d64, buf.data(), n64 * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nm) e = cudaMemcpyAsync(dlg, lg.data(), (size_t)nm * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    TopoArgs a;
    a.nn = nn;
    a.levels = levels;
    a.nm = nm;
    a.n_roots = pre[nm];
    a.level_off = d64;
    a.pre = d64 + fb.level_off.size();
    a.ntet = a.pre + pre.size();
    a.lg = dlg;
    a.t_off = a.ntet + ntet.size();
    a.first_tree = 0;
    while (a.first_tree < nm && lg[a.first_tree] < 0) ++a.first_tree;
    a.perm = perm;
    a.topo = topo;
    topology_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(a);
    s->ctx->launches += 1;
    e = cudaGetLastError();
  }
  cudaStreamSynchronize(st);
  cudaFree(w);
  return e;
}

}  // namespace kdop
