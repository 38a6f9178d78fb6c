// kdop_traverse.cu -- tandem (BVTT) traversal of mesh-pair trees.
//
// Reference semantics: kdop::details::traversal and kdop::tandem_traversal
// (SIMULATION/KDOP/KDOP/include/kdop_tandem_traversal.h:19-196): test the two
// root kDOPs (:164), then descend simultaneously; an overlapping pair of
// internal nodes expands into its 2 x 2 child pairs, an internal/leaf pair into
// 1 x 2 (:122-155); an overlapping leaf pair whose tets both have a boundary
// face (:56-88) goes to contact generation.  Overlap is the strict slab test
// of geometry_overlap_dop_dop.h:13-25 / geometry_overlap_interval_interval.h:
// 12-20.  The set of emitted tet pairs and the number of kDOP tests equal the
// reference's; only the emission order differs (sort for a canonical order).
//
// B200 design (replacing the OpenCL backlog kernel, cl/kernels/
// kdop_cl_tandem_traversal.cl:19-233, and the gProximity queues,
// cl/kernels/gproximity/*.cl):
//   * one persistent launch sized to the resident-block count; each warp owns
//     a node-pair deque in shared memory and pops up to 32 pairs per step, one
//     per lane;
//   * "test on expand": a popped entry is a pair already known to overlap; the
//     lane loads the children records (the two children of a node are adjacent,
//     so a 2-child side is one contiguous 2-record read, float4 by float4,
//     stopping as soon as every child pair is separated), tests all child pairs
//     and keeps the overlapping ones;
//   * ballot/shuffle compaction: one warp-wide prefix sum packs the kept pairs
//     into the deque and the leaf pairs into the output with one atomic per warp;
//   * load balance: root pairs are claimed from the pair list, and a warp whose
//     deque holds many pairs while other warps wait gives its oldest (largest)
//     entries to a global queue; a deque overflow spills there too;
//   * termination: a global count of outstanding work units reaches zero;
//     every wait is bounded by a time limit after which the kernel records
//     DEV_ERR_TIMEOUT and returns (no unbounded spin).
#include <algorithm>
#include <mutex>

#include "kdop_device.cuh"

namespace kdop {

struct TravArgs {
  const float4* __restrict__ nodes;
  const uint8_t* __restrict__ surf;
  const uint32_t* __restrict__ root;
  const uint2* __restrict__ pairs;
  uint32_t* candA;
  uint32_t* candB;
  uint32_t* candP;
  unsigned cand_cap;
  uint4* q_items;
  uint32_t* q_tags;
  unsigned q_cap;
  TravCtl* ctl;
  int stack_cap;  // power of two
  int init_chunk;
  int donate_min;
  int surface_filter;
  long long timeout_ns;
  unsigned n_meshes;
  const uint32_t* __restrict__ order;  // root pair i -> pair index (NULL: identity)
};

// Device buffers one traversal works in: pairs (input), candidates (output),
// work queue and control block (scratch).
struct TravBuffers {
  const uint2* pairs;
  const uint32_t* order;  // processing order of the pairs, or NULL
  uint32_t* cand;  // 3 * cand_cap: A tets | B tets | pair ids
  int64_t cand_cap;
  uint4* q_items;
  uint32_t* q_tags;
  int64_t q_cap;
  TravCtl* ctl;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// 256-bit read-only load of two consecutive float4 chunks (p 32-byte aligned).
__device__ __forceinline__ void ldg256(const float4* p, float4& x, float4& y) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(y.x), "=f"(y.y), "=f"(y.z), "=f"(y.w)
               : "l"(p));
}
__device__ __forceinline__ unsigned ld_volatile(const unsigned* p) { return *(const volatile unsigned*)p; }
__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

// Overlap of the child pairs of one deque entry.  Side X is either a leaf
// node (1 candidate: the node itself) or an internal node given by its first
// child c (2 candidates: c, c + 1).  The records are fetched G float4 chunks
// per round (all loads of a round in flight together); the next round is only
// fetched while some child pair is still undecided.
template <int K, int G>
struct Expand {
  using L = NodeLayout<K>;
  uint32_t idxA[2], idxB[2];  // node indices of the candidates
  uint32_t stA[2], enA[2], stB[2], enB[2];
  int na, nb;
  unsigned sep;  // bit (2 i + k): child pair (i, k) separated (or absent)

  __device__ __forceinline__ void chunk(int j, const float4& A0, const float4& A1, const float4& B0,
                                        const float4& B1) {
    if (2 * j < L::NS) {
      // separated iff A.hi < B.lo || B.hi < A.lo
      sep |= ((A0.y < B0.x) || (B0.y < A0.x)) ? 1u : 0u;
      sep |= ((A0.y < B1.x) || (B1.y < A0.x)) ? 2u : 0u;
      sep |= ((A1.y < B0.x) || (B0.y < A1.x)) ? 4u : 0u;
      sep |= ((A1.y < B1.x) || (B1.y < A1.x)) ? 8u : 0u;
    }
    if (2 * j + 1 < L::NS) {
      sep |= ((A0.w < B0.z) || (B0.w < A0.z)) ? 1u : 0u;
      sep |= ((A0.w < B1.z) || (B1.w < A0.z)) ? 2u : 0u;
      sep |= ((A1.w < B0.z) || (B0.w < A1.z)) ? 4u : 0u;
      sep |= ((A1.w < B1.z) || (B1.w < A1.z)) ? 8u : 0u;
    }
    if (j == L::TOPO_CHUNK) {
      stA[0] = __float_as_uint(L::TOPO_ZW ? A0.z : A0.x);
      enA[0] = __float_as_uint(L::TOPO_ZW ? A0.w : A0.y);
      stA[1] = __float_as_uint(L::TOPO_ZW ? A1.z : A1.x);
      enA[1] = __float_as_uint(L::TOPO_ZW ? A1.w : A1.y);
      stB[0] = __float_as_uint(L::TOPO_ZW ? B0.z : B0.x);
      enB[0] = __float_as_uint(L::TOPO_ZW ? B0.w : B0.y);
      stB[1] = __float_as_uint(L::TOPO_ZW ? B1.z : B1.x);
      enB[1] = __float_as_uint(L::TOPO_ZW ? B1.w : B1.y);
    }
  }

  __device__ __forceinline__ void run(const float4* __restrict__ nodes, uint32_t ea, uint32_t eb) {
    na = (ea & LEAF_BIT) ? 1 : 2;
    nb = (eb & LEAF_BIT) ? 1 : 2;
    uint32_t a0 = ea & ~LEAF_BIT, b0 = eb & ~LEAF_BIT;
    idxA[0] = a0;
    idxA[1] = a0 + 1;
    idxB[0] = b0;
    idxB[1] = b0 + 1;
    sep = 0;
    if (na == 1) sep |= 0xC;  // pairs (1,0), (1,1)
    if (nb == 1) sep |= 0xA;  // pairs (0,1), (1,1)
    const float4* pa = nodes + (int64_t)a0 * L::NW;
    const float4* pb = nodes + (int64_t)b0 * L::NW;
    stA[0] = stA[1] = enA[0] = enA[1] = stB[0] = stB[1] = enB[0] = enB[1] = 0;
    // Records of an even number of chunks start on 32-byte boundaries, so
    // two chunks come in one 256-bit load (half the L1 wavefronts).
    constexpr bool kWide = (L::NW % 2 == 0) && (G % 2 == 0);
#pragma unroll
    for (int j0 = 0; j0 < L::NW; j0 += G) {
      if (sep == 0xF) break;
      float4 A0[G], A1[G], B0[G], B1[G];
      if (kWide) {
#pragma unroll
        for (int g = 0; g < G; g += 2) {
          if (j0 + g < L::NW) {
            ldg256(pa + j0 + g, A0[g], A0[g + 1]);
            ldg256(pb + j0 + g, B0[g], B0[g + 1]);
            A1[g] = A0[g];
            A1[g + 1] = A0[g + 1];
            B1[g] = B0[g];
            B1[g + 1] = B0[g + 1];
            if (na == 2) ldg256(pa + L::NW + j0 + g, A1[g], A1[g + 1]);
            if (nb == 2) ldg256(pb + L::NW + j0 + g, B1[g], B1[g + 1]);
          }
        }
      } else {
#pragma unroll
        for (int g = 0; g < G; ++g) {
          if (j0 + g < L::NW) {
            A0[g] = __ldg(pa + j0 + g);
            B0[g] = __ldg(pb + j0 + g);
            A1[g] = A0[g];
            B1[g] = B0[g];
            if (na == 2) A1[g] = __ldg(pa + L::NW + j0 + g);
            if (nb == 2) B1[g] = __ldg(pb + L::NW + j0 + g);
          }
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g)
        if (j0 + g < L::NW) chunk(j0 + g, A0[g], A1[g], B0[g], B1[g]);
    }
  }
};

template <int K, int G>
__global__ void __launch_bounds__(512, 2) traverse_kernel(TravArgs a) {
  extern __shared__ uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int CAP = a.stack_cap;
  const int MASK = CAP - 1;
  uint32_t* sA = smem + (size_t)wib * 3 * CAP;
  uint32_t* sB = sA + CAP;
  uint32_t* sP = sB + CAP;
  TravCtl* ctl = a.ctl;
  const unsigned n_init = ctl->n_init;
  const unsigned pair_base = ctl->pair_base;

  int top = 0, bot = 0;  // deque [bot, top) in virtual positions
  int release = 0;       // work units taken and not yet released
  bool init_done = false;
  unsigned claim = 0xFFFFFFFFu;
  unsigned long long my_tests = 0, my_lo = 0;
  unsigned max_depth = 0;
  bool failed = false;

  for (;;) {
    // per-lane results of this step
    unsigned push_mask = 0, emit_mask = 0;
    uint32_t pushA[4], pushB[4], emitA[4], emitB[4];
    uint32_t pid = 0;

    // queue counters for the donation check, read early so that their
    // latency overlaps the node loads of this step
    unsigned q_h = 0, q_t = 0;
    if (lane == 0 && top - bot >= a.donate_min) {
      q_h = ld_volatile(&ctl->q_head);
      q_t = ld_volatile(&ctl->q_tail);
    }

    if (top == bot) {
      // Work handed to the queue was counted before it was published, so the
      // release needs no fence.
      if (release) {
        if (lane == 0) atomicSub(&ctl->work, release);
        release = 0;
      }
      bool have = false;
      if (!init_done) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&ctl->init_head, (unsigned)a.init_chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base < n_init) {
          int n = (int)min((unsigned)a.init_chunk, n_init - base);
          release += n;
          have = true;
          if (lane < n) {
            // root test (kdop_tandem_traversal.h:164), then the traversal's own
            // test of the root pair (:42), both counted as the reference does.
            pid = pair_base + base + lane;
            if (a.order) pid = a.order[pid];
            uint2 mp = a.pairs[pid];
            uint32_t ra = NO_NODE, rb = NO_NODE;
            if (mp.x < a.n_meshes && mp.y < a.n_meshes) {
              ra = a.root[mp.x];
              rb = a.root[mp.y];
            } else {
              atomicOr(&ctl->error, DEV_ERR_BAD_INDEX);
            }
            if (ra != NO_NODE && rb != NO_NODE) {
              Expand<K, G> ex;
              ex.run(a.nodes, ra | LEAF_BIT, rb | LEAF_BIT);
              my_tests += 1;
              if (!(ex.sep & 1u)) {
                my_tests += 1;
                bool la = ex.stA[0] == ex.enA[0], lb = ex.stB[0] == ex.enB[0];
                if (la && lb) {
                  my_lo += 1;
                  if (!a.surface_filter || (a.surf[ex.stA[0]] && a.surf[ex.stB[0]])) {
                    emit_mask = 1;
                    emitA[0] = ex.stA[0];
                    emitB[0] = ex.stB[0];
                  }
                } else {
                  push_mask = 1;
                  pushA[0] = la ? (ra | LEAF_BIT) : ex.stA[0];
                  pushB[0] = lb ? (rb | LEAF_BIT) : ex.stB[0];
                }
              }
            }
          }
        } else {
          init_done = true;
        }
      }
      if (!have) {
        // wait for a queue item or the end of all work
        if (claim == 0xFFFFFFFFu) {
          unsigned c = 0;
          if (lane == 0) c = atomicAdd(&ctl->q_head, 1u);
          claim = __shfl_sync(0xffffffffu, c, 0);
        }
        unsigned long long t0 = global_ns();
        unsigned backoff = 64;
        int got = 0;
        for (;;) {
          if (claim < a.q_cap && ld_volatile(&a.q_tags[claim]) != 0u) {
            got = 1;
            break;
          }
          if (ld_volatile(&ctl->work) == 0) break;
          if ((long long)(global_ns() - t0) > a.timeout_ns) {
            failed = true;
            break;
          }
          __nanosleep(backoff);
          backoff = min(backoff * 2u, 2048u);
        }
        got = __shfl_sync(0xffffffffu, got, 0);
        if (__shfl_sync(0xffffffffu, (int)failed, 0)) {
          failed = true;
          break;
        }
        if (!got) break;
        __threadfence();
        uint4 it = __ldcg(a.q_items + claim);
        if (lane == 0) {
          a.q_tags[claim] = 0u;
          sA[top & MASK] = it.x;
          sB[top & MASK] = it.y;
          sP[top & MASK] = it.z;
        }
        top += 1;
        release += 1;
        claim = 0xFFFFFFFFu;
        __syncwarp();
        continue;
      }
    } else {
      int n = min(32, top - bot);
      top -= n;
      if (lane < n) {
        int at = (top + lane) & MASK;
        uint32_t ea = sA[at], eb = sB[at];
        pid = sP[at];
        Expand<K, G> ex;
        ex.run(a.nodes, ea, eb);
        my_tests += (unsigned long long)(ex.na * ex.nb);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          int i = c >> 1, k = c & 1;
          if (ex.sep & (1u << c)) continue;
          bool la = ex.stA[i] == ex.enA[i], lb = ex.stB[k] == ex.enB[k];
          if (la && lb) {
            my_lo += 1;
            if (!a.surface_filter || (a.surf[ex.stA[i]] && a.surf[ex.stB[k]])) {
              emit_mask |= 1u << c;
              emitA[c] = ex.stA[i];
              emitB[c] = ex.stB[k];
            }
          } else {
            push_mask |= 1u << c;
            pushA[c] = la ? (ex.idxA[i] | LEAF_BIT) : ex.stA[i];
            pushB[c] = lb ? (ex.idxB[k] | LEAF_BIT) : ex.stB[k];
          }
        }
      }
      __syncwarp();
    }

    // ---- compaction: one warp prefix sum of (pushes, emits) ----
    int np = __popc(push_mask), ne = __popc(emit_mask);
    int v = np | (ne << 16);
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    int tot = __shfl_sync(0xffffffffu, incl, 31);
    int excl = incl - v;
    int tot_p = tot & 0xFFFF, tot_e = tot >> 16;
    int off_p = excl & 0xFFFF, off_e = excl >> 16;

    if (tot_e) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&ctl->n_cand, (unsigned)tot_e);
      base = __shfl_sync(0xffffffffu, base, 0) + (unsigned)off_e;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (emit_mask & (1u << c)) {
          if (base < a.cand_cap) {
            a.candA[base] = emitA[c];
            a.candB[base] = emitB[c];
            a.candP[base] = pid;
          }
          ++base;
        }
      }
    }
    if (tot_p) {
      if (top - bot + tot_p <= CAP) {
        int at = top + off_p;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (push_mask & (1u << c)) {
            sA[at & MASK] = pushA[c];
            sB[at & MASK] = pushB[c];
            sP[at & MASK] = pid;
            ++at;
          }
        }
        top += tot_p;
      } else {
        // deque full: the new entries go to the global queue
        unsigned t0 = 0;
        if (lane == 0) t0 = atomicAdd(&ctl->q_tail, (unsigned)tot_p);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        int room = (int)min((unsigned long long)tot_p,
                            (t0 < a.q_cap) ? (unsigned long long)(a.q_cap - t0) : 0ull);
        if (room < tot_p && lane == 0) atomicOr(&ctl->error, DEV_ERR_QUEUE_FULL);
        if (room > 0 && lane == 0) atomicAdd(&ctl->work, room);
        __syncwarp();
        unsigned slot = t0 + (unsigned)off_p;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (push_mask & (1u << c)) {
            if (slot < t0 + (unsigned)room) a.q_items[slot] = make_uint4(pushA[c], pushB[c], pid, 0u);
            ++slot;
          }
        }
        __threadfence();
        __syncwarp();
        slot = t0 + (unsigned)off_p;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (push_mask & (1u << c)) {
            if (slot < t0 + (unsigned)room) atomicExch(&a.q_tags[slot], 1u);
            ++slot;
          }
        }
      }
    }
    int depth = top - bot;
    if ((unsigned)depth > max_depth) max_depth = (unsigned)depth;

    // ---- donation: give the oldest entries to waiting warps ----
    if (depth >= a.donate_min) {
      int waiting = 0;
      if (lane == 0) waiting = (q_h > q_t) ? (int)min(q_h - q_t, 32u) : 0;
      waiting = __shfl_sync(0xffffffffu, waiting, 0);
      int d = min(waiting, depth / 2);
      if (d > 0) {
        unsigned t0 = 0;
        if (lane == 0) t0 = atomicAdd(&ctl->q_tail, (unsigned)d);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        int room = (int)min((unsigned long long)d, (t0 < a.q_cap) ? (unsigned long long)(a.q_cap - t0) : 0ull);
        if (room < d && lane == 0) atomicOr(&ctl->error, DEV_ERR_QUEUE_FULL);
        if (room > 0 && lane == 0) atomicAdd(&ctl->work, room);
        __syncwarp();
        if (lane < room) {
          int at = (bot + lane) & MASK;
          a.q_items[t0 + lane] = make_uint4(sA[at], sB[at], sP[at], 0u);
        }
        __threadfence();
        __syncwarp();
        if (lane < room) atomicExch(&a.q_tags[t0 + lane], 1u);
        // entries that found no room stay lost only with DEV_ERR_QUEUE_FULL set
        bot += d;
      }
    }
    __syncwarp();
  }

  // ---- totals ----
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    my_tests += __shfl_down_sync(0xffffffffu, my_tests, o);
    my_lo += __shfl_down_sync(0xffffffffu, my_lo, o);
  }
  if (lane == 0) {
    atomicAdd(&ctl->tests, my_tests);
    atomicAdd(&ctl->leaf_overlaps, my_lo);
    atomicMax(&ctl->max_stack, max_depth);
    if (failed) atomicOr(&ctl->error, DEV_ERR_TIMEOUT);
  }
}

__global__ void trav_init_kernel(TravCtl* c, unsigned n_init, unsigned pair_base, int reset_totals) {
  if (threadIdx.x != 0) return;
  if (reset_totals) {
    c->tests = 0;
    c->leaf_overlaps = 0;
    c->n_cand = 0;
    c->error = 0;
    c->max_stack = 0;
    c->n_contacts = 0;
  }
  c->init_head = 0;
  c->q_head = 0;
  c->q_tail = 0;
  c->work = (int)n_init;
  c->n_init = n_init;
  c->pair_base = pair_base;
}

int traverse_block_threads(int block_warps) { return 32 * block_warps; }
size_t traverse_smem_bytes(int block_warps, int stack_cap) {
  return (size_t)block_warps * 3 * (size_t)stack_cap * sizeof(uint32_t);
}

template <int K>
static cudaError_t prepare_k(size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(traverse_kernel<K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(traverse_kernel<K, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(traverse_kernel<K, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return e;
}

cudaError_t traverse_prepare(int K, size_t smem) {
  switch (K) {
    case 6: return prepare_k<6>(smem);
    case 8: return prepare_k<8>(smem);
    case 12: return prepare_k<12>(smem);
    case 14: return prepare_k<14>(smem);
    case 18: return prepare_k<18>(smem);
    case 20: return prepare_k<20>(smem);
    case 26: return prepare_k<26>(smem);
  }
  return cudaErrorInvalidValue;
}

template <int K, int G>
static cudaError_t traverse_impl(kdop_scene* s, int64_t n_pairs, const TravBuffers& b, const TravParams& p,
                                 int plain) {
  cudaStream_t st = s->ctx->stream;
  int threads = traverse_block_threads(p.block_warps);
  size_t smem = traverse_smem_bytes(p.block_warps, p.stack_cap);
  cudaError_t e = prepare_k<K>(smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(traverse_kernel<K, G>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           p.smem_carveout > 0 ? p.smem_carveout : -1);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, traverse_kernel<K, G>, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  unsigned grid = (unsigned)(per_sm * s->ctx->sm_count);
  TravArgs a;
  a.nodes = s->nodes;
  a.surf = s->surf;
  a.root = s->root_dev;
  a.pairs = b.pairs;
  a.order = b.order;
  a.candA = b.cand;
  a.candB = b.cand + b.cand_cap;
  a.candP = b.cand + 2 * b.cand_cap;
  a.cand_cap = (unsigned)b.cand_cap;
  a.q_items = b.q_items;
  a.q_tags = b.q_tags;
  a.q_cap = (unsigned)b.q_cap;
  a.ctl = b.ctl;
  a.n_meshes = (unsigned)s->n_meshes;
  a.stack_cap = p.stack_cap;
  a.init_chunk = p.init_chunk;
  a.donate_min = p.donate_min;
  a.surface_filter = p.surface_filter;
  a.timeout_ns = p.timeout_ns;
  if (!plain) {
    // waves of wave_pairs root pairs (largest first), or all at once
    int64_t wave = p.wave_pairs > 0 ? p.wave_pairs : n_pairs;
    if (wave < 1) wave = 1;
    for (int64_t off = 0; off < n_pairs || off == 0; off += wave) {
      int64_t n = std::min<int64_t>(wave, n_pairs - off);
      trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, (unsigned)std::max<int64_t>(n, 0), (unsigned)off, off == 0);
      traverse_kernel<K, G><<<grid, threads, smem, st>>>(a);
      s->ctx->launches += 2;
      if (n_pairs == 0) break;
    }
  } else {
    for (int64_t i = 0; i < n_pairs; ++i) {
      trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, 1u, (unsigned)i, i == 0 ? 1 : 0);
      traverse_kernel<K, G><<<grid, threads, smem, st>>>(a);
      s->ctx->launches += 2;
    }
    if (n_pairs == 0) {
      trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, 0u, 0u, 1);
      s->ctx->launches += 1;
    }
  }
  return cudaGetLastError();
}

template <int K>
static cudaError_t traverse_group(kdop_scene* s, int64_t n_pairs, const TravBuffers& b, const TravParams& p,
                                  int plain) {
  switch (p.load_group) {
    case 1: return traverse_impl<K, 1>(s, n_pairs, b, p, plain);
    case 4: return traverse_impl<K, 4>(s, n_pairs, b, p, plain);
    default: return traverse_impl<K, 2>(s, n_pairs, b, p, plain);
  }
}

static cudaError_t traverse_buffers(kdop_scene* s, int64_t n_pairs, const TravBuffers& b, const TravParams& p,
                                    int plain) {
  switch (s->K) {
    case 6: return traverse_group<6>(s, n_pairs, b, p, plain);
    case 8: return traverse_group<8>(s, n_pairs, b, p, plain);
    case 12: return traverse_group<12>(s, n_pairs, b, p, plain);
    case 14: return traverse_group<14>(s, n_pairs, b, p, plain);
    case 18: return traverse_group<18>(s, n_pairs, b, p, plain);
    case 20: return traverse_group<20>(s, n_pairs, b, p, plain);
    case 26: return traverse_group<26>(s, n_pairs, b, p, plain);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_traverse(kdop_scene* s, int64_t n_pairs, const uint2* pairs, const TravParams& p, int plain) {
  TravBuffers b;
  b.pairs = pairs;
  b.order = s->pair_order;
  b.cand = s->cand;
  b.cand_cap = s->cand_cap;
  b.q_items = s->q_items;
  b.q_tags = s->q_tags;
  b.q_cap = s->queue_cap;
  b.ctl = s->ctl;
  return traverse_buffers(s, n_pairs, b, p, plain);
}

}  // namespace kdop

// ---- traversal that allocates no device memory -------------------------------
// Its scratch -- the traversal's control block and work queue -- lives in this
// file-scope device array instead of the scene's allocated buffers.  Every GPU
// that loads the library holds the array until the process exits.
namespace kdop {
namespace {

constexpr int64_t kStaticQueueEntries = 65536;
constexpr size_t kStaticCtlBytes = 256;
constexpr size_t kStaticTagBytes = (size_t)kStaticQueueEntries * sizeof(uint32_t);
constexpr size_t kStaticScratchBytes = kStaticCtlBytes + kStaticTagBytes + (size_t)kStaticQueueEntries * sizeof(uint4);
static_assert(sizeof(TravCtl) <= kStaticCtlBytes, "control block does not fit");

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch per device, found once per device with
// that device current.  In host code the array's name only stands in for the
// symbol; it is not a device address.
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void* g_static_addr[kMaxDevices] = {nullptr};

cudaError_t static_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_static_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_static_addr[device]);
  return cudaSuccess;
}

__global__ void static_counters_kernel(const TravCtl* c, unsigned long long* out) {
  if (threadIdx.x != 0) return;
  out[0] = c->n_cand;
  out[1] = c->tests;
  out[2] = c->leaf_overlaps;
  out[3] = c->error;
}

}  // namespace
}  // namespace kdop

extern "C" int kdop_traverse_noalloc(kdop_scene* s, int64_t n_pairs, const uint32_t* pairs, uint32_t* candidates,
                                     int64_t cap, unsigned long long* counters, const kdop_traverse_opts* opts) {
  using namespace kdop;
  if (!s || n_pairs < 0 || (n_pairs > 0 && !pairs) || !candidates || cap <= 0 || !counters) return KDOP_ERR_INVALID;
  if (cap > (int64_t)0xFFFFFFF0ll || n_pairs >= (int64_t)0x7FFFFFFF) return KDOP_ERR_CAPACITY;
  TravParams p;
  int mode = 0;
  if (kdop_resolve_traverse_opts(s, opts, p, mode) != KDOP_OK) return KDOP_ERR_INVALID;
  if (cudaSetDevice(s->ctx->device) != cudaSuccess) return KDOP_ERR_CUDA;
  unsigned char* base = nullptr;
  if (static_scratch(s->ctx->device, &base) != cudaSuccess) {
    cudaGetLastError();
    return KDOP_ERR_CUDA;
  }
  TravBuffers b;
  b.pairs = reinterpret_cast<const uint2*>(pairs);
  b.order = nullptr;
  b.cand = candidates;
  b.cand_cap = cap;
  b.ctl = reinterpret_cast<TravCtl*>(base);
  b.q_tags = reinterpret_cast<uint32_t*>(base + kStaticCtlBytes);
  b.q_items = reinterpret_cast<uint4*>(base + kStaticCtlBytes + kStaticTagBytes);
  b.q_cap = kStaticQueueEntries;
  cudaStream_t st = s->ctx->stream;
  // the array keeps the previous call's contents: the control block and the
  // queue tags must start at zero
  if (cudaMemsetAsync(base, 0, kStaticCtlBytes + kStaticTagBytes, st) != cudaSuccess) {
    cudaGetLastError();
    return KDOP_ERR_CUDA;
  }
  cudaError_t e = traverse_buffers(s, n_pairs, b, p, mode == KDOP_TRAVERSE_PLAIN);
  if (e == cudaSuccess) {
    static_counters_kernel<<<1, 32, 0, st>>>(b.ctl, counters);
    s->ctx->launches += 1;
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return KDOP_ERR_CUDA;
  }
  return KDOP_OK;
}
