// kdop_sort.cu -- stable device radix sort and exclusive scan used to put the
// traversal's results in a reproducible order (the role of the OpenCL
// back-end's qsort, cl/kdop_cl_tandem_traversal.h:1773-1788) and to order
// tets by Morton code on the device (kdop_mesh_reorder.h:173-353).
//
// Radix sort: least-significant digit first, 8-bit digits, 64-bit keys with
// 32-bit values.  A pass is a per-tile digit histogram, an exclusive scan of
// the (digit, tile) counts in digit-major order, and a scatter in which every
// warp ranks its keys with __match_any_sync; warps, rounds and lanes follow
// the input order, so every pass (and the sort) is stable.  Digits in which
// all keys agree are skipped (one reduction and one read-back per sort).
#include <algorithm>

#include "kdop_device.cuh"
#include "kdop_sort.h"

namespace kdop {

namespace {

constexpr int RS_WARPS = 8;
constexpr int RS_THREADS = 32 * RS_WARPS;
constexpr int RS_ROUNDS = 8;                           // keys per lane per tile
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;        // 2048 keys
constexpr int SC_THREADS = 1024, SC_ITEMS = 4;
constexpr int SC_BLOCK = SC_THREADS * SC_ITEMS;        // 4096 counts per scan block

__global__ void key_bits_kernel(const uint64_t* __restrict__ keys, int64_t n, unsigned long long* and_or) {
  unsigned long long a = ~0ull, o = 0ull;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long k = keys[i];
    a &= k;
    o |= k;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    a &= __shfl_xor_sync(0xffffffffu, a, s);
    o |= __shfl_xor_sync(0xffffffffu, o, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAnd(&and_or[0], a);
    atomicOr(&and_or[1], o);
  }
}

__global__ void key_bits_init(unsigned long long* and_or) {
  and_or[0] = ~0ull;
  and_or[1] = 0ull;
}

// counts[d * n_tiles + tile] = keys of the tile with digit d
__global__ void __launch_bounds__(RS_THREADS) hist_kernel(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                         uint32_t* counts, int64_t n_tiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    int64_t i = base + r * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[(int64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS) scatter_kernel(const uint64_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin, uint64_t* kout,
                                                            uint32_t* vout, int64_t n, int shift,
                                                            const uint32_t* __restrict__ offsets, int64_t n_tiles) {
  __shared__ uint32_t wc[RS_WARPS][256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (int d = threadIdx.x; d < RS_WARPS * 256; d += RS_THREADS) (&wc[0][0])[d] = 0;
  __syncthreads();
  // warp w owns keys [base + w * 32 * ROUNDS, ...) in ROUNDS rounds of 32
  const int64_t base = (int64_t)blockIdx.x * RS_TILE + (int64_t)w * 32 * RS_ROUNDS;
  uint64_t k[RS_ROUNDS];
  uint32_t v[RS_ROUNDS];
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    int64_t i = base + r * 32 + lane;
    bool ok = i < n;
    k[r] = ok ? kin[i] : 0ull;
    v[r] = ok ? vin[i] : 0u;
    unsigned active = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      unsigned d = (unsigned)(k[r] >> shift) & 255u;
      unsigned peers = __match_any_sync(active, d);
      if ((peers & lt) == 0u) wc[w][d] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // per digit: tile offset, then the warps in order
  {
    const int d = threadIdx.x;
    uint32_t run = offsets[(int64_t)d * n_tiles + blockIdx.x];
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      uint32_t c = wc[ww][d];
      wc[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    int64_t i = base + r * 32 + lane;
    bool ok = i < n;
    unsigned active = __ballot_sync(0xffffffffu, ok);
    unsigned d = 0, peers = 0, pos = 0;
    if (ok) {
      d = (unsigned)(k[r] >> shift) & 255u;
      peers = __match_any_sync(active, d);
      pos = wc[w][d] + __popc(peers & lt);
      kout[pos] = k[r];
      vout[pos] = v[r];
    }
    __syncwarp();
    if (ok && (peers & lt) == 0u) wc[w][d] += __popc(peers);
    __syncwarp();
  }
}

// Exclusive scan of one block of SC_BLOCK counts; block total to sums.
__global__ void __launch_bounds__(SC_THREADS) scan_block_kernel(const uint32_t* in, uint32_t* out,
                                                               int64_t n, uint32_t* sums) {
  __shared__ uint32_t ws[SC_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * SC_BLOCK + (int64_t)threadIdx.x * SC_ITEMS;
  uint32_t x[SC_ITEMS], t = 0;
#pragma unroll
  for (int j = 0; j < SC_ITEMS; ++j) {
    x[j] = (base + j < n) ? in[base + j] : 0u;
    t += x[j];
  }
  uint32_t incl = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) ws[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t s = ws[lane];
    uint32_t si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    ws[lane] = si - s;
    if (lane == 31 && sums) sums[blockIdx.x] = si;
  }
  __syncthreads();
  uint32_t run = ws[w] + incl - t;
#pragma unroll
  for (int j = 0; j < SC_ITEMS; ++j) {
    if (base + j < n) out[base + j] = run;
    run += x[j];
  }
}

__global__ void scan_add_kernel(uint32_t* out, int64_t n, const uint32_t* __restrict__ block_off) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += block_off[i / SC_BLOCK];
}

}  // namespace

size_t scan_scratch_words(int64_t n) {
  size_t w = 0;
  while (n > SC_BLOCK) {
    n = (n + SC_BLOCK - 1) / SC_BLOCK;
    w += (size_t)n;
  }
  return w + 1;
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* scratch, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int64_t blocks = (n + SC_BLOCK - 1) / SC_BLOCK;
  if (blocks == 1) {
    scan_block_kernel<<<1, SC_THREADS, 0, st>>>(in, out, n, nullptr);
    return cudaGetLastError();
  }
  uint32_t* sums = scratch;
  scan_block_kernel<<<(unsigned)blocks, SC_THREADS, 0, st>>>(in, out, n, sums);
  cudaError_t e = exclusive_scan_u32(sums, sums, blocks, scratch + blocks, st);
  if (e != cudaSuccess) return e;
  scan_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, sums);
  return cudaGetLastError();
}

size_t radix_scratch_words(int64_t n) {
  int64_t tiles = (n + RS_TILE - 1) / RS_TILE;
  int64_t counts = 256 * std::max<int64_t>(tiles, 1);
  return (size_t)(2 * counts) + scan_scratch_words(counts) + 4;
}

cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, int64_t n,
                             uint32_t* scratch, cudaStream_t st) {
  if (n <= 1) return cudaSuccess;
  const int64_t tiles = (n + RS_TILE - 1) / RS_TILE;
  const int64_t nc = 256 * tiles;
  unsigned long long* bits = reinterpret_cast<unsigned long long*>(scratch);  // 4 words, 8-byte aligned
  uint32_t* counts = scratch + 4;
  uint32_t* offsets = counts + nc;
  uint32_t* scan_tmp = offsets + nc;
  key_bits_init<<<1, 1, 0, st>>>(bits);
  key_bits_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 1184), 256, 0, st>>>(keys, n, bits);
  unsigned long long hb[2];
  cudaError_t e = cudaMemcpyAsync(hb, bits, sizeof(hb), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  const unsigned long long diff = hb[0] ^ hb[1];  // bits in which keys differ
  uint64_t *ka = keys, *kb = keys_tmp;
  uint32_t *va = vals, *vb = vals_tmp;
  for (int shift = 0; shift < 64; shift += 8) {
    if (((diff >> shift) & 255ull) == 0ull) continue;
    hist_kernel<<<(unsigned)tiles, RS_THREADS, 0, st>>>(ka, n, shift, counts, tiles);
    e = exclusive_scan_u32(counts, offsets, nc, scan_tmp, st);
    if (e != cudaSuccess) return e;
    scatter_kernel<<<(unsigned)tiles, RS_THREADS, 0, st>>>(ka, va, kb, vb, n, shift, offsets, tiles);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    e = cudaMemcpyAsync(keys, ka, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vals, va, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

}  // namespace kdop

// ---- reproducible order of a traversal's results ------------------------------
namespace kdop {
namespace {

// key = (tet A, tet B); the pair follows in a second, stable sort
__global__ void cand_keys_kernel(const uint32_t* __restrict__ cA, const uint32_t* __restrict__ cB, int64_t n,
                                 uint64_t* keys, uint32_t* vals) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = ((uint64_t)cA[i] << 32) | (uint64_t)cB[i];
  vals[i] = (uint32_t)i;
}

__global__ void pair_keys_kernel(const uint32_t* __restrict__ cP, const uint32_t* __restrict__ perm, int64_t n,
                                 uint64_t* keys) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = cP[perm[i]];
}

// rows and records in sorted order; per-candidate contact counts
__global__ void cand_gather_kernel(const uint32_t* __restrict__ perm, int64_t n, const uint32_t* __restrict__ cand,
                                   int64_t cap, uint32_t* cand_out, const int4* __restrict__ rec, int4* rec_out,
                                   uint32_t* counts) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t o = perm[k];
  cand_out[k] = cand[o];
  cand_out[n + k] = cand[cap + o];
  cand_out[2 * n + k] = cand[2 * cap + o];
  if (rec) {
    int4 r = rec[o];
    rec_out[k] = r;
    counts[k] = (uint32_t)max(r.z, 0);
  }
}

// contact rows of sorted candidate k to rows first[k] ..; records follow
__global__ void contact_gather_kernel(int64_t n, int4* rec, const uint32_t* __restrict__ first,
                                      const kdop_contact* __restrict__ rows, kdop_contact* rows_out) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int4 r = rec[k];
  uint32_t f = first[k];
  for (int c = 0; c < r.z; ++c) {
    kdop_contact x = rows[r.w + c];
    x.cand = (uint32_t)k;
    rows_out[f + c] = x;
  }
  if (r.z > 0) r.w = (int)f;
  rec[k] = r;
}

}  // namespace

// Work buffer of sort_results, every region 256-byte aligned.
struct SortWork {
  size_t keys, keys_tmp, vals, vals_tmp, cand_out, first, rec_out, rows_out, scratch, total;
  SortWork(int64_t n, int64_t n_contacts) {
    size_t at = 0;
    auto take = [&](size_t bytes) {
      size_t o = at;
      at += (bytes + 255) & ~(size_t)255;
      return o;
    };
    keys = take((size_t)n * 8);
    keys_tmp = take((size_t)n * 8);
    vals = take((size_t)n * 4);
    vals_tmp = take((size_t)n * 4);
    cand_out = take((size_t)n * 12);
    first = take((size_t)n * 4);
    rec_out = take((size_t)n * 16);
    rows_out = take((size_t)std::max<int64_t>(n_contacts, 1) * sizeof(kdop_contact));
    scratch = take(std::max(radix_scratch_words(n), scan_scratch_words(n)) * 4);
    total = at;
  }
};

cudaError_t sort_results(kdop_scene* s, int64_t n, int64_t n_contacts, void* work, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  char* w = static_cast<char*>(work);
  SortWork L(n, n_contacts);
  uint64_t* keys = reinterpret_cast<uint64_t*>(w + L.keys);
  uint64_t* keys_tmp = reinterpret_cast<uint64_t*>(w + L.keys_tmp);
  uint32_t* vals = reinterpret_cast<uint32_t*>(w + L.vals);
  uint32_t* vals_tmp = reinterpret_cast<uint32_t*>(w + L.vals_tmp);
  uint32_t* cand_out = reinterpret_cast<uint32_t*>(w + L.cand_out);
  uint32_t* first = reinterpret_cast<uint32_t*>(w + L.first);
  int4* rec_out = reinterpret_cast<int4*>(w + L.rec_out);
  kdop_contact* rows_out = reinterpret_cast<kdop_contact*>(w + L.rows_out);
  uint32_t* scratch = reinterpret_cast<uint32_t*>(w + L.scratch);
  const unsigned g = (unsigned)((n + 255) / 256);
  const uint32_t* cA = s->cand;
  const uint32_t* cB = s->cand + s->cand_cap;
  const uint32_t* cP = s->cand + 2 * s->cand_cap;
  cand_keys_kernel<<<g, 256, 0, st>>>(cA, cB, n, keys, vals);
  cudaError_t e = radix_sort_pairs(keys, vals, keys_tmp, vals_tmp, n, scratch, st);
  if (e != cudaSuccess) return e;
  pair_keys_kernel<<<g, 256, 0, st>>>(cP, vals, n, keys);
  e = radix_sort_pairs(keys, vals, keys_tmp, vals_tmp, n, scratch, st);
  if (e != cudaSuccess) return e;
  const bool with_contacts = s->contacted;
  cand_gather_kernel<<<g, 256, 0, st>>>(vals, n, s->cand, s->cand_cap, cand_out, with_contacts ? s->records : nullptr,
                                        rec_out, first);
  for (int k = 0; k < 3; ++k) {
    e = cudaMemcpyAsync(s->cand + k * s->cand_cap, cand_out + k * n, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  if (with_contacts) {
    e = exclusive_scan_u32(first, first, n, scratch, st);
    if (e != cudaSuccess) return e;
    contact_gather_kernel<<<g, 256, 0, st>>>(n, rec_out, first, s->contacts, rows_out);
    e = cudaMemcpyAsync(s->records, rec_out, (size_t)n * sizeof(int4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && n_contacts > 0)
      e = cudaMemcpyAsync(s->contacts, rows_out, (size_t)n_contacts * sizeof(kdop_contact), cudaMemcpyDeviceToDevice,
                          st);
    if (e != cudaSuccess) return e;
  }
  s->ctx->launches += with_contacts ? 4 : 3;
  return cudaGetLastError();
}

size_t sort_results_bytes(int64_t n, int64_t n_contacts) { return SortWork(n, n_contacts).total; }

}  // namespace kdop
