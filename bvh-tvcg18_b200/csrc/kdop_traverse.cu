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
//     a node-pair deque in shared memory;
//   * "test on expand": a popped entry is a pair already known to overlap;
//     a few lanes take one entry together and read the children of both sides
//     as whole twin records (siblings' chunks interleaved, so one 256-bit load
//     per lane and chunk pair), test the four child pairs slab by slab, and
//     keep the overlapping ones (see traverse_kernel);
//   * ballot compaction: prefix sums over per-lane push counts pack the kept
//     pairs into the deque, and emitted leaf pairs reserve rows with one
//     atomic per warp;
//   * load balance: root pairs are claimed from the pair list (largest first),
//     and a warp whose deque is deep while other warps wait gives its oldest
//     (largest) entries to a global queue -- any deque with work gives half
//     while many warps wait; a deque overflow spills there too;
//   * termination: a global count of outstanding work units reaches zero;
//     every wait is bounded by a time limit after which the kernel records
//     DEV_ERR_TIMEOUT and returns (no unbounded spin).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "kdop_device.cuh"
#include "kdop_sort.h"

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
  const uint4* __restrict__ entries;   // when set: initial work = these deque entries (A, B, pair)
  unsigned poll_mask;  // queue counters polled on steps with (step & poll_mask) == 0
};

// Device buffers one traversal works in: pairs (input), candidates (output),
// work queue and control block (scratch).
struct TravBuffers {
  const uint2* pairs;
  const uint32_t* order;  // processing order of the pairs, or NULL
  const uint4* entries = nullptr;  // initial deque entries instead of root pairs (n_init of them)
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

// Overlap of two single nodes by one lane (the root test of a mesh pair): both
// records chunk by chunk; wa, wb get the records' word 0.
template <int K>
__device__ __forceinline__ bool node_overlap(const float4* __restrict__ nodes, uint32_t na, uint32_t nb,
                                             uint32_t& wa, uint32_t& wb) {
  using L = NodeLayout<K>;
  bool sep = false;
  wa = wb = 0;
#pragma unroll
  for (int j = 0; j < L::NW; ++j) {
    float4 A = __ldg(nodes + L::at(na, j)), B = __ldg(nodes + L::at(nb, j));
    if (2 * j < L::NS) sep |= (A.y < B.x) || (B.y < A.x);
    if (2 * j + 1 < L::NS) sep |= (A.w < B.z) || (B.w < A.z);
    if (j == L::TOPO_CHUNK) {
      wa = L::word0(A);
      wb = L::word0(B);
    }
  }
  return !sep;
}

// Waiting warps from which on every deque with work donates (tail mode).
constexpr int kTailWaiting = 512;

// Warp total and exclusive prefix of per-lane counts below 2^BITS, one
// ballot per bit.
template <int BITS>
__device__ __forceinline__ void warp_prefix(int v, unsigned lt_mask, int& total, int& excl) {
  total = excl = 0;
#pragma unroll
  for (int k = 0; k < BITS; ++k) {
    unsigned m = __ballot_sync(0xffffffffu, (v >> k) & 1);
    total += __popc(m) << k;
    excl += __popc(m & lt_mask) << k;
  }
}

// Tet of a leaf node (word 1 of its record).
template <int K>
__device__ __forceinline__ uint32_t leaf_tet(const float4* __restrict__ nodes, uint32_t w) {
  using L = NodeLayout<K>;
  return L::word1(__ldg(nodes + L::at(w & NODE_MASK, L::TOPO_CHUNK)));
}

// Lanes per deque entry: chunk pairs of a record over C chunks per lane,
// rounded up to a power of two so that entries sit on aligned lane groups.
template <int K, int C>
struct Coop {
  static constexpr int NW = NodeLayout<K>::NW;
  static constexpr int Q0 = (NW + C - 1) / C;
  static constexpr int Q = Q0 <= 1 ? 1 : Q0 <= 2 ? 2 : Q0 <= 4 ? 4 : 8;
  static constexpr int E = 32 / Q;             // entries per sub-batch
  static constexpr int PM = (4 + Q - 1) / Q;   // child pairs per lane
};

// Deque entries (X, Y, pair): X and Y overlap and their children are to be
// tested.  A side with LEAF_BIT is the single node X & NODE_MASK (a leaf);
// otherwise X is the first child of an internal node, whose children X, X + 1
// form one twin record.  Word 0 of a child's record is its entry value.
//
// Cooperative expansion: Q lanes take one entry (E = 32 / Q entries per
// sub-batch).  Lane q reads chunks j = q, q + Q, ... (C of them) of both
// children of each side, one 256-bit load per chunk and side (twin records
// interleave the siblings' chunks), so the lanes of an entry read whole
// 128-byte lines (k = 14) and a warp-wide load touches E lines instead of 32.
// The lane tests its slabs for the four child pairs; a butterfly OR over the
// entry's lanes combines the verdicts; the lane holding the topology chunk
// broadcasts the children's word 0; lane q then handles child pairs q, q + Q.
// S sub-batches are loaded together per step, and one compaction per step
// packs the pushes of all of them.
template <int K, int C, int S>
__global__ void __launch_bounds__(512, (C * S >= 4) ? 1 : 2) traverse_kernel(TravArgs a) {
  using L = NodeLayout<K>;
  using CP = Coop<K, C>;
  constexpr int NW = L::NW;
  constexpr int Q = CP::Q, E = CP::E, PM = CP::PM;
  constexpr int SLOTS = PM * S;                     // pushes per lane per step
  constexpr int TQ = L::TOPO_CHUNK % Q, TR = L::TOPO_CHUNK / Q;  // lane and round holding topology
  constexpr int CBITS = SLOTS <= 1 ? 1 : SLOTS <= 3 ? 2 : 3;  // bits of a lane's push count
  extern __shared__ uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int ge = lane / Q, gq = lane % Q;  // entry and chunk lane of this lane
  const float4* __restrict__ nodes_q = a.nodes + 2 * gq;  // chunk gq of twin 0
  const unsigned lt_mask = (1u << lane) - 1u;
  const int CAP = a.stack_cap;
  const int MASK = CAP - 1;
  // this warp's deque: CAP entries of (A, B) words, then CAP pair indices
  // (written and read only while the deque mixes pairs, see curP below)
  uint32_t* wbase = smem + (size_t)wib * 3 * CAP;
  uint2* sAB = reinterpret_cast<uint2*>(wbase);
  uint32_t* sP = wbase + 2 * CAP;
  TravCtl* ctl = a.ctl;
  const unsigned n_init = ctl->n_init;
  const unsigned pair_base = ctl->pair_base;

  int top = 0, bot = 0;  // deque [bot, top) in virtual positions
  int release = 0;       // work units taken and not yet released
  bool init_done = false;
  unsigned claim = 0xFFFFFFFFu;
  // per-lane counts, added to the control block's 64-bit totals every 1024
  // steps and at the end (at most 4 per lane and step: no overflow)
  unsigned tests32 = 0, lo32 = 0;
  auto fold_counts = [&]() {
    unsigned t = tests32, l = lo32;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      t += __shfl_down_sync(0xffffffffu, t, o);
      l += __shfl_down_sync(0xffffffffu, l, o);
    }
    if (lane == 0) {
      if (t) atomicAdd(&ctl->tests, (unsigned long long)t);
      if (l) atomicAdd(&ctl->leaf_overlaps, (unsigned long long)l);
    }
    tests32 = lo32 = 0;
  };
  unsigned max_depth = 0;
  bool failed = false;
  // Pair index of the deque's entries.  A deque filled from one root pair or
  // one queue item holds a single pair (entries inherit their parent's pair),
  // kept in curP; only a claim of several root pairs or frontier entries at
  // once mixes pairs, and then each entry's pair is kept in sP (warp-uniform).
  uint32_t curP = 0;
  bool mixed = false;

  unsigned step = 0;
  for (;;) {
    // Queue counters for the donation check, read early so that their
    // latency overlaps the node loads of this step.
    unsigned q_h = 0, q_t = 0;
    ++step;
    if ((step & 1023u) == 0u) fold_counts();
    // warp-uniform: poll the queue counters on every (poll_mask + 1)-th step
    // with work
    const bool polled = top - bot >= 2 && (step & a.poll_mask) == 0u;
    if (lane == 0 && polled) {
      q_h = ld_volatile(&ctl->q_head);
      q_t = ld_volatile(&ctl->q_tail);
    }
    // this step's pushes (entry words) and emitted leaf pairs (node words)
    unsigned push_mask = 0, emit_mask = 0;
    uint32_t pushA[SLOTS], pushB[SLOTS], slotP[SLOTS];

    if (top == bot) {
      // Work handed to the queue was counted before it was published, so the
      // release needs no fence.
      if (release) {
        if (lane == 0) atomicSub(&ctl->work, release);
        release = 0;
      }
      bool have = false;
      mixed = false;  // the deque is empty
      if (!init_done) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&ctl->init_head, (unsigned)a.init_chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base < n_init) {
          int n = (int)min((unsigned)a.init_chunk, n_init - base);
          release += n;
          have = true;
          uint32_t p0 = 0;
          if (lane < n && a.entries) {
            // a pending node pair of a frontier (its tests are counted already)
            const uint4 e = a.entries[base + lane];
            pushA[0] = e.x;
            pushB[0] = e.y;
            slotP[0] = e.z;
            p0 = e.z;
            push_mask = 1;
          } else if (lane < n) {
            // root test (kdop_tandem_traversal.h:164), then the traversal's own
            // test of the root pair (:42), both counted as the reference does.
            uint32_t pid = pair_base + base + lane;
            if (a.order) pid = a.order[pid];
            p0 = pid;
            uint2 mp = a.pairs[pid];
            uint32_t ra = NO_NODE, rb = NO_NODE;
            if (mp.x < a.n_meshes && mp.y < a.n_meshes) {
              ra = a.root[mp.x];
              rb = a.root[mp.y];
            } else {
              atomicOr(&ctl->error, DEV_ERR_BAD_INDEX);
            }
            if (ra != NO_NODE && rb != NO_NODE) {
              uint32_t wa, wb;
              bool ov = node_overlap<K>(a.nodes, ra, rb, wa, wb);
              tests32 += 1u;
              if (ov) {
                tests32 += 1u;
                pushA[0] = wa;
                pushB[0] = wb;
                slotP[0] = pid;
                if (wa & wb & LEAF_BIT) {
                  lo32 += 1u;
                  if (!a.surface_filter || (wa & wb & SURF_BIT)) emit_mask = 1;
                } else {
                  push_mask = 1;
                }
              }
            }
          }
          if (n > 1)
            mixed = true;  // entries of several pairs
          else
            curP = __shfl_sync(0xffffffffu, p0, 0);
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
        for (unsigned it = 0;; ++it) {
          if (claim < a.q_cap && ld_volatile(&a.q_tags[claim]) != 0u) {
            got = 1;
            break;
          }
          // the end-of-work counter is polled by every waiting warp: every
          // 4th round only, to keep its line free for the workers' atomics
          if ((it & 3u) == 0u && ld_volatile(&ctl->work) == 0) break;
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
          sAB[top & MASK] = make_uint2(it.x, it.y);
        }
        curP = it.z;  // the deque was empty: one pair
        top += 1;
        release += 1;
        claim = 0xFFFFFFFFu;
        __syncwarp();
        continue;
      }
    } else {
      const int n = min(E * S, top - bot);
      top -= n;
      uint2 eab[S];
      uint32_t ep[S];
      float4 A0[S][C], A1[S][C], B0[S][C], B1[S][C];
#pragma unroll
      for (int b = 0; b < S; ++b) {
        const int i = b * E + ge;
        eab[b] = make_uint2(0u, 0u);
        ep[b] = 0;
        if (i < n) {
          const int at = (top + i) & MASK;
          eab[b] = sAB[at];
          ep[b] = mixed ? sP[at] : curP;
        }
        const float4* pa = nodes_q + (size_t)((eab[b].x & NODE_MASK) >> 1) * (2 * NW);
        const float4* pb = nodes_q + (size_t)((eab[b].y & NODE_MASK) >> 1) * (2 * NW);
#pragma unroll
        for (int r = 0; r < C; ++r) {
          const int j = gq + Q * r;
          // a lane without an entry (i >= n) loads the record of node 0's
          // twin and its verdicts are never used: no zero fill
          if (j < NW) {
            ldg256(pa + 2 * Q * r, A0[b][r], A1[b][r]);
            ldg256(pb + 2 * Q * r, B0[b][r], B1[b][r]);
          }
        }
      }
      __syncwarp();  // entries read before this step's pushes overwrite them
#pragma unroll
      for (int b = 0; b < S; ++b) {
        const bool valid = b * E + ge < n;
        const uint32_t xa = eab[b].x, xb = eab[b].y;
        const bool singleA = (xa & LEAF_BIT) != 0, singleB = (xb & LEAF_BIT) != 0;
        // Separation of child pairs (0,0), (0,1), (1,0), (1,1).  A single
        // side is the node itself, which is side (x & 1) of the twin just
        // loaded: the pairs with the other side of that twin are absent and
        // count as separated.
        const bool noA0 = singleA && (xa & 1u), noA1 = singleA && !(xa & 1u);
        const bool noB0 = singleB && (xb & 1u), noB1 = singleB && !(xb & 1u);
        bool s0 = noA0 || noB0, s1 = noA0 || noB1, s2 = noA1 || noB0, s3 = noA1 || noB1;
        uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
#pragma unroll
        for (int r = 0; r < C; ++r) {
          const int j = gq + Q * r;
          const float4 a0 = A0[b][r], a1 = A1[b][r], b0 = B0[b][r], b1 = B1[b][r];
          if (2 * j < L::NS) {
            s0 = s0 || (a0.y < b0.x) || (b0.y < a0.x);
            s1 = s1 || (a0.y < b1.x) || (b1.y < a0.x);
            s2 = s2 || (a1.y < b0.x) || (b0.y < a1.x);
            s3 = s3 || (a1.y < b1.x) || (b1.y < a1.x);
          }
          if (2 * j + 1 < L::NS) {
            s0 = s0 || (a0.w < b0.z) || (b0.w < a0.z);
            s1 = s1 || (a0.w < b1.z) || (b1.w < a0.z);
            s2 = s2 || (a1.w < b0.z) || (b0.w < a1.z);
            s3 = s3 || (a1.w < b1.z) || (b1.w < a1.z);
          }
          if (r == TR) {
            t0 = L::word0(a0);
            t1 = L::word0(a1);
            t2 = L::word0(b0);
            t3 = L::word0(b1);
          }
        }
        unsigned sep = (s0 ? 1u : 0u) | (s1 ? 2u : 0u) | (s2 ? 4u : 0u) | (s3 ? 8u : 0u);
#pragma unroll
        for (int o = 1; o < Q; o <<= 1) sep |= __shfl_xor_sync(0xffffffffu, sep, o);
        // word 0 of the four children, from the lane holding the topology chunk
        const int src = ge * Q + TQ;
        const uint32_t wA0 = __shfl_sync(0xffffffffu, t0, src);
        const uint32_t wA1 = __shfl_sync(0xffffffffu, t1, src);
        uint32_t wB0, wB1;
        if (Q == 2) {
          // lane gq only handles child gq of B (see below): the topology lane
          // keeps its own word, the other lane gets the other child's
          const uint32_t wo = __shfl_sync(0xffffffffu, TQ ? t2 : t3, src);
          wB0 = wB1 = (gq == TQ) ? (TQ ? t3 : t2) : wo;
        } else {
          wB0 = __shfl_sync(0xffffffffu, t2, src);
          wB1 = __shfl_sync(0xffffffffu, t3, src);
        }
        if (valid) {
          if (gq == 0) tests32 += (singleA ? 1u : 2u) * (singleB ? 1u : 2u);
          // the lane's child pairs c = gq + Q r (c = 2 i + k: child i of A,
          // child k of B) as bit masks: overlapping, both leaves, both on
          // the surface
          unsigned alive = 0, leaf = 0, surf = 0;
#pragma unroll
          for (int r = 0; r < PM; ++r) {
            const int c = gq + Q * r;
            const int ci = (Q == 2) ? r : (c >> 1), ck = (Q == 2) ? gq : (c & 1);
            const uint32_t wa = ci ? wA1 : wA0, wb = ck ? wB1 : wB0;
            const uint32_t both = wa & wb;
            const int k = b * PM + r;
            pushA[k] = wa;
            pushB[k] = wb;
            slotP[k] = ep[b];
            const bool ok = (Q * r + Q - 1 < 4 || c < 4) && !((sep >> c) & 1u);
            alive |= (ok ? 1u : 0u) << r;
            leaf |= (both >> 31) << r;
            surf |= ((both >> 30) & 1u) << r;
          }
          if (!a.surface_filter) surf = ~0u;
          lo32 += __popc(alive & leaf);  // both leaves
          emit_mask |= (alive & leaf & surf) << (b * PM);
          push_mask |= (alive & ~leaf & ((1u << PM) - 1u)) << (b * PM);
        }
      }
    }

    // ---- emits (rare): leaf pairs to candidate rows, one atomic per warp ----
    if (__any_sync(0xffffffffu, emit_mask != 0u)) {
      int tot_e = 0, off_e = 0;
      warp_prefix<CBITS>(__popc(emit_mask), lt_mask, tot_e, off_e);
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&ctl->n_cand, (unsigned)tot_e);
      base = __shfl_sync(0xffffffffu, base, 0) + (unsigned)off_e;
#pragma unroll
      for (int k = 0; k < SLOTS; ++k) {
        if (emit_mask & (1u << k)) {
          if (base < a.cand_cap) {
            a.candA[base] = leaf_tet<K>(a.nodes, pushA[k]);
            a.candB[base] = leaf_tet<K>(a.nodes, pushB[k]);
            a.candP[base] = slotP[k];
          }
          ++base;
        }
      }
    }
    // ---- pushes: deque (or the global queue), slot-major: every lane's
    // slot-0 push, then every slot-1 push, ..., so that the lanes of one store
    // instruction write consecutive positions (one ballot per slot) ----
    {
      unsigned pm[SLOTS];
      int pbase[SLOTS];
      int tot_p = 0;
#pragma unroll
      for (int k = 0; k < SLOTS; ++k) {
        pm[k] = __ballot_sync(0xffffffffu, (push_mask >> k) & 1u);
        pbase[k] = tot_p;
        tot_p += __popc(pm[k]);
      }
      if (tot_p) {
        if (top - bot + tot_p <= CAP) {
#pragma unroll
          for (int k = 0; k < SLOTS; ++k) {
            if (push_mask & (1u << k)) {
              const int at = (top + pbase[k] + __popc(pm[k] & lt_mask)) & MASK;
              sAB[at] = make_uint2(pushA[k], pushB[k]);
              if (mixed) sP[at] = slotP[k];
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
#pragma unroll
          for (int k = 0; k < SLOTS; ++k) {
            const unsigned slot = t0 + (unsigned)(pbase[k] + __popc(pm[k] & lt_mask));
            if ((push_mask & (1u << k)) && slot < t0 + (unsigned)room)
              a.q_items[slot] = make_uint4(pushA[k], pushB[k], slotP[k], 0u);
          }
          __threadfence();
          __syncwarp();
#pragma unroll
          for (int k = 0; k < SLOTS; ++k) {
            const unsigned slot = t0 + (unsigned)(pbase[k] + __popc(pm[k] & lt_mask));
            if ((push_mask & (1u << k)) && slot < t0 + (unsigned)room) atomicExch(&a.q_tags[slot], 1u);
          }
        }
      }
    }
    int depth = top - bot;
    if (polled && (unsigned)depth > max_depth) max_depth = (unsigned)depth;

    // ---- donation: give the oldest entries to waiting warps ----
    // A deep deque gives to any waiting warp; while many warps wait (the
    // tail of the traversal) any deque with two or more entries gives half.
    if (polled && depth >= 2) {
      int waiting = 0;
      if (lane == 0) waiting = (q_h > q_t) ? (int)min(q_h - q_t, 1024u) : 0;
      waiting = __shfl_sync(0xffffffffu, waiting, 0);
      int d = (depth >= a.donate_min || waiting >= kTailWaiting) ? min(min(waiting, 32), depth / 2) : 0;
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
          uint2 ab = sAB[at];
          a.q_items[t0 + lane] = make_uint4(ab.x, ab.y, mixed ? sP[at] : curP, 0u);
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
  fold_counts();
  if (lane == 0) {
    atomicMax(&ctl->max_stack, max_depth);
    if (failed) atomicOr(&ctl->error, DEV_ERR_TIMEOUT);
  }
}

__global__ void trav_init_kernel(TravCtl* c, unsigned n_init, unsigned pair_base, int reset_totals, int stuck) {
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
  c->work = (int)n_init + stuck;
  c->n_init = n_init;
  c->pair_base = pair_base;
}

int traverse_block_threads(int block_warps) { return 32 * block_warps; }
size_t traverse_smem_bytes(int block_warps, int stack_cap) {
  return (size_t)block_warps * 3 * (size_t)stack_cap * sizeof(uint32_t);
}

template <int K>
static cudaError_t prepare_k(size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(traverse_kernel<K, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(traverse_kernel<K, 1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(traverse_kernel<K, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(traverse_kernel<K, 2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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

template <int K, int C, int S>
static cudaError_t traverse_impl(kdop_scene* s, int64_t n_pairs, const TravBuffers& b, const TravParams& p,
                                 int plain) {
  cudaStream_t st = s->ctx->stream;
  int threads = traverse_block_threads(p.block_warps);
  size_t smem = traverse_smem_bytes(p.block_warps, p.stack_cap);
  cudaError_t e = prepare_k<K>(smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(traverse_kernel<K, C, S>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           p.smem_carveout > 0 ? p.smem_carveout : -1);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, traverse_kernel<K, C, S>, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  unsigned grid = (unsigned)(per_sm * s->ctx->sm_count);
  TravArgs a;
  a.nodes = s->nodes;
  a.surf = s->surf;
  a.root = s->root_dev;
  a.pairs = b.pairs;
  a.order = b.order;
  a.entries = b.entries;
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
  // Donations reach waiting warps only through polls.  A batched launch keeps
  // most warps busy with root pairs and polls every 16th step (config 3: 10.49
  // ms vs 10.65 ms every 4th step); a one-pair launch leaves most warps
  // waiting for donations and polls every 4th step (config 3, one launch per
  // pair: 88 ms vs 103 ms every 16th).
  a.poll_mask = plain ? 3u : 15u;
  if (b.entries) {
    // seeded by a frontier: its tests and leaf pairs are in the totals already
    trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, (unsigned)n_pairs, 0u, 0, p.stuck_work);
    traverse_kernel<K, C, S><<<grid, threads, smem, st>>>(a);
    s->ctx->launches += 2;
  } else if (!plain) {
    // waves of wave_pairs root pairs (largest first), or all at once
    int64_t wave = p.wave_pairs > 0 ? p.wave_pairs : n_pairs;
    if (wave < 1) wave = 1;
    for (int64_t off = 0; off < n_pairs || off == 0; off += wave) {
      int64_t n = std::min<int64_t>(wave, n_pairs - off);
      trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, (unsigned)std::max<int64_t>(n, 0), (unsigned)off, off == 0,
                                         p.stuck_work);
      traverse_kernel<K, C, S><<<grid, threads, smem, st>>>(a);
      s->ctx->launches += 2;
      if (n_pairs == 0) break;
    }
  } else {
    for (int64_t i = 0; i < n_pairs; ++i) {
      trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, 1u, (unsigned)i, i == 0 ? 1 : 0, p.stuck_work);
      traverse_kernel<K, C, S><<<grid, threads, smem, st>>>(a);
      s->ctx->launches += 2;
    }
    if (n_pairs == 0) {
      trav_init_kernel<<<1, 32, 0, st>>>(b.ctl, 0u, 0u, 1, 0);
      s->ctx->launches += 1;
    }
  }
  return cudaGetLastError();
}

template <int K>
static cudaError_t traverse_group(kdop_scene* s, int64_t n_pairs, const TravBuffers& b, const TravParams& p,
                                  int plain) {
  // load_group: 1 = one chunk pair per lane, one sub-batch per step;
  // 2 = two sub-batches per step; 4 = two chunk pairs per lane (half the
  // lanes per entry, twice the entries per sub-batch); 8 = two chunk pairs
  // per lane and two sub-batches per step (twice the registers, one block
  // per SM)
  switch (p.load_group) {
    case 1: return traverse_impl<K, 1, 1>(s, n_pairs, b, p, plain);
    case 4: return traverse_impl<K, 2, 1>(s, n_pairs, b, p, plain);
    case 8: return traverse_impl<K, 2, 2>(s, n_pairs, b, p, plain);
    default: return traverse_impl<K, 1, 2>(s, n_pairs, b, p, plain);
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

// ---- frontier-seeded and sharded traversal ----------------------------------
// The node-pair tree is expanded breadth first, one launch per level, until
// enough pairs are pending; every test and leaf pair of that expansion is the
// reference's own (the same rule, in breadth-first order).  The pending pairs
// are sorted (a deterministic list on every rank) and dealt round-robin to the
// shards; each shard's persistent traversal starts from its share.
namespace {

template <int K>
__device__ void frontier_emit(const TravArgs& a, uint32_t wa, uint32_t wb, uint32_t pid) {
  unsigned at = atomicAdd(&a.ctl->n_cand, 1u);
  if (at < a.cand_cap) {
    a.candA[at] = leaf_tet<K>(a.nodes, wa);
    a.candB[at] = leaf_tet<K>(a.nodes, wb);
    a.candP[at] = pid;
  }
}

__device__ void frontier_push(uint4* out, unsigned* count, unsigned cap, uint32_t wa, uint32_t wb, uint32_t pid,
                              unsigned* error) {
  unsigned at = atomicAdd(count, 1u);
  if (at < cap)
    out[at] = make_uint4(wa, wb, pid, 0u);
  else
    atomicOr(error, DEV_ERR_QUEUE_FULL);
}

// root test of each mesh pair (kdop_tandem_traversal.h:164, then :42)
template <int K>
__global__ void frontier_root_kernel(TravArgs a, unsigned n_pairs, uint4* out, unsigned* count, unsigned cap) {
  // count: level 0's count (the frontier state's first word)
  unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_pairs) return;
  uint2 mp = a.pairs[p];
  if (mp.x >= a.n_meshes || mp.y >= a.n_meshes) {
    atomicOr(&a.ctl->error, DEV_ERR_BAD_INDEX);
    return;
  }
  uint32_t ra = a.root[mp.x], rb = a.root[mp.y];
  if (ra == NO_NODE || rb == NO_NODE) return;
  uint32_t wa, wb;
  bool ov = node_overlap<K>(a.nodes, ra, rb, wa, wb);
  atomicAdd(&a.ctl->tests, ov ? 2ull : 1ull);
  if (!ov) return;
  if (wa & wb & LEAF_BIT) {
    atomicAdd(&a.ctl->leaf_overlaps, 1ull);
    if (!a.surface_filter || (wa & wb & SURF_BIT)) frontier_emit<K>(a, wa, wb, p);
  } else {
    frontier_push(out, count, cap, wa, wb, p, &a.ctl->error);
  }
}

// Frontier state: level counts fs[0 .. kMaxLevels], then the frozen flag,
// the final level and the final count.
constexpr int kMaxLevels = 20;
constexpr int FS_FROZEN = kMaxLevels + 1, FS_LEVEL = kMaxLevels + 2, FS_COUNT = kMaxLevels + 3, FS_WORDS = 32;

// one level: every pending pair's child pairs.  The level stops the expansion
// (freezes) when its input is empty, large enough, or could overflow the
// next buffer; all later levels then do nothing.  Every thread reads the
// same counts, so they all take the same decision.
template <int K>
__global__ void frontier_level_kernel(TravArgs a, int level, const uint4* __restrict__ in, uint4* out, unsigned* fs,
                                      unsigned cap, unsigned fmin) {
  if (fs[FS_FROZEN]) return;
  const unsigned n_in = min(fs[level], cap);
  if (n_in == 0 || n_in >= fmin || 4ull * n_in > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      fs[FS_FROZEN] = 1u;
      fs[FS_LEVEL] = (unsigned)level;
      fs[FS_COUNT] = n_in;
    }
    return;
  }
  unsigned* count = fs + level + 1;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n_in; i += gridDim.x * blockDim.x) {
  uint4 e = in[i];
  uint32_t A[2], B[2];
  int na = 2, nb = 2;
  if (e.x & LEAF_BIT) {
    A[0] = e.x & NODE_MASK;
    na = 1;
  } else {
    A[0] = e.x;
    A[1] = e.x + 1;
  }
  if (e.y & LEAF_BIT) {
    B[0] = e.y & NODE_MASK;
    nb = 1;
  } else {
    B[0] = e.y;
    B[1] = e.y + 1;
  }
  unsigned long long lo = 0;
  for (int x = 0; x < na; ++x)
    for (int y = 0; y < nb; ++y) {
      uint32_t wa, wb;
      if (!node_overlap<K>(a.nodes, A[x], B[y], wa, wb)) continue;
      if (wa & wb & LEAF_BIT) {
        ++lo;
        if (!a.surface_filter || (wa & wb & SURF_BIT)) frontier_emit<K>(a, wa, wb, e.z);
      } else {
        frontier_push(out, count, cap, wa, wb, e.z, &a.ctl->error);
      }
    }
  atomicAdd(&a.ctl->tests, (unsigned long long)(na * nb));
  if (lo) atomicAdd(&a.ctl->leaf_overlaps, lo);
  }
}

__global__ void frontier_final_kernel(unsigned* fs, unsigned cap) {
  if (threadIdx.x == 0 && !fs[FS_FROZEN]) {
    fs[FS_FROZEN] = 1u;
    fs[FS_LEVEL] = kMaxLevels;
    fs[FS_COUNT] = min(fs[kMaxLevels], cap);
  }
}

__global__ void entry_keys_kernel(const uint4* __restrict__ f, unsigned n, uint64_t* keys, uint32_t* vals,
                                  int by_pair) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (by_pair) {
    keys[i] = f[vals[i]].z;
  } else {
    uint4 e = f[i];
    keys[i] = ((uint64_t)e.x << 32) | e.y;
    vals[i] = i;
  }
}

// this shard's entries: sorted positions rank, rank + n_ranks, ...
__global__ void deal_kernel(const uint4* __restrict__ f, const uint32_t* __restrict__ order, unsigned n, int rank,
                            int n_ranks, uint4* mine) {
  unsigned j = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned src = (unsigned)rank + j * (unsigned)n_ranks;
  if (src < n) mine[j] = f[order[src]];
}

__global__ void clear_totals_kernel(TravCtl* c) {
  if (threadIdx.x == 0) {
    c->tests = 0;
    c->leaf_overlaps = 0;
    c->n_cand = 0;
  }
}

template <int K>
TravArgs frontier_args(kdop_scene* s, const uint2* pairs, const TravParams& p) {
  TravArgs a;
  std::memset(&a, 0, sizeof(a));
  a.nodes = s->nodes;
  a.surf = s->surf;
  a.root = s->root_dev;
  a.pairs = pairs;
  a.candA = s->cand;
  a.candB = s->cand + s->cand_cap;
  a.candP = s->cand + 2 * s->cand_cap;
  a.cand_cap = (unsigned)s->cand_cap;
  a.ctl = s->ctl;
  a.n_meshes = (unsigned)s->n_meshes;
  a.surface_filter = p.surface_filter;
  return a;
}

// Work buffer of a sharded traversal: frontier state, two frontiers, the
// sort (keys, values, scratch), this shard's entries; 256-byte regions.
struct ShardWork {
  size_t fs, f0, f1, k, kt, v, vt, sc, mine, total;
  explicit ShardWork(int64_t cap) {
    size_t at = 0;
    auto take = [&](size_t b) {
      size_t o = at;
      at += (b + 255) & ~(size_t)255;
      return o;
    };
    fs = take(FS_WORDS * 4);
    f0 = take((size_t)cap * 16);
    f1 = take((size_t)cap * 16);
    k = take((size_t)cap * 8);
    kt = take((size_t)cap * 8);
    v = take((size_t)cap * 4);
    vt = take((size_t)cap * 4);
    sc = take(radix_scratch_words(cap) * 4);
    mine = take((size_t)cap * 16);
    total = at;
  }
};

template <int K>
cudaError_t shard_impl(kdop_scene* s, int64_t n_pairs, const uint2* pairs, const TravParams& p, int rank,
                       int n_ranks, int64_t frontier_min, char* w, int64_t cap, int64_t* n_entries) {
  cudaStream_t st = s->ctx->stream;
  ShardWork L(cap);
  unsigned* fs = reinterpret_cast<unsigned*>(w + L.fs);
  uint4* F[2] = {reinterpret_cast<uint4*>(w + L.f0), reinterpret_cast<uint4*>(w + L.f1)};
  uint64_t* keys = reinterpret_cast<uint64_t*>(w + L.k);
  uint64_t* ktmp = reinterpret_cast<uint64_t*>(w + L.kt);
  uint32_t* vals = reinterpret_cast<uint32_t*>(w + L.v);
  uint32_t* vtmp = reinterpret_cast<uint32_t*>(w + L.vt);
  uint32_t* scratch = reinterpret_cast<uint32_t*>(w + L.sc);
  uint4* mine = reinterpret_cast<uint4*>(w + L.mine);
  TravArgs a = frontier_args<K>(s, pairs, p);
  cudaError_t e;
  trav_init_kernel<<<1, 32, 0, st>>>(s->ctl, 0u, 0u, 1, 0);  // totals and queue state to zero
  if ((e = cudaMemsetAsync(fs, 0, FS_WORDS * 4, st)) != cudaSuccess) return e;
  if (n_pairs > 0)
    frontier_root_kernel<K><<<(unsigned)((n_pairs + 255) / 256), 256, 0, st>>>(a, (unsigned)n_pairs, F[0], fs,
                                                                                (unsigned)cap);
  const unsigned g = (unsigned)std::min<int64_t>((cap / 4 + 255) / 256, 4 * (int64_t)s->ctx->sm_count);
  for (int level = 0; level < kMaxLevels; ++level)
    frontier_level_kernel<K><<<g, 256, 0, st>>>(a, level, F[level & 1], F[(level + 1) & 1], fs, (unsigned)cap,
                                               (unsigned)frontier_min);
  frontier_final_kernel<<<1, 32, 0, st>>>(fs, (unsigned)cap);
  s->ctx->launches += 3 + kMaxLevels;
  unsigned hfs[FS_WORDS];
  if ((e = cudaMemcpyAsync(hfs, fs, sizeof(hfs), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  const unsigned n = hfs[FS_COUNT];
  const uint4* fin = F[hfs[FS_LEVEL] & 1];
  // deterministic order: by (A, B), then by pair
  if (n > 0) {
    const unsigned gn = (n + 255) / 256;
    entry_keys_kernel<<<gn, 256, 0, st>>>(fin, n, keys, vals, 0);
    if ((e = radix_sort_pairs(keys, vals, ktmp, vtmp, n, scratch, st)) != cudaSuccess) return e;
    entry_keys_kernel<<<gn, 256, 0, st>>>(fin, n, keys, vals, 1);
    if ((e = radix_sort_pairs(keys, vals, ktmp, vtmp, n, scratch, st)) != cudaSuccess) return e;
    deal_kernel<<<gn, 256, 0, st>>>(fin, vals, n, rank, n_ranks, mine);
    s->ctx->launches += 3;
  }
  // the expansion's tests and leaf pairs belong to shard 0
  if (rank != 0) {
    clear_totals_kernel<<<1, 32, 0, st>>>(s->ctl);
    s->ctx->launches++;
  }
  const int64_t m = n > (unsigned)rank ? ((int64_t)n - rank + n_ranks - 1) / n_ranks : 0;
  *n_entries = m;
  TravBuffers b;
  b.pairs = pairs;
  b.order = nullptr;
  b.entries = mine;
  b.cand = s->cand;
  b.cand_cap = s->cand_cap;
  b.q_items = s->q_items;
  b.q_tags = s->q_tags;
  b.q_cap = s->queue_cap;
  b.ctl = s->ctl;
  return traverse_group<K>(s, m, b, p, 0);
}

}  // namespace

cudaError_t launch_traverse_shard(kdop_scene* s, int64_t n_pairs, const uint2* pairs, const TravParams& p, int rank,
                                  int n_ranks, int64_t frontier_min, void** work, size_t* work_bytes,
                                  int64_t* n_entries) {
  const int64_t cap = std::max<int64_t>(8 * std::max<int64_t>(frontier_min, 1), n_pairs) + 1024;
  const size_t need = ShardWork(cap).total;
  if (*work_bytes < need) {
    if (*work) cudaFree(*work);
    *work = nullptr;
    *work_bytes = 0;
    cudaError_t e = cudaMalloc(work, need);
    if (e != cudaSuccess) return e;
    *work_bytes = need;
  }
  char* w = static_cast<char*>(*work);
  switch (s->K) {
    case 6: return shard_impl<6>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
    case 8: return shard_impl<8>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
    case 12: return shard_impl<12>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
    case 14: return shard_impl<14>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
    case 18: return shard_impl<18>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
    case 20: return shard_impl<20>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
    case 26: return shard_impl<26>(s, n_pairs, pairs, p, rank, n_ranks, frontier_min, w, cap, n_entries);
  }
  return cudaErrorInvalidValue;
}

}  // namespace kdop

// ---- traversal that allocates no device memory -------------------------------
// Its scratch -- the traversal's control block and work queue -- lives in this
// file-scope device array instead of the scene's allocated buffers.  Every GPU
// that loads the library holds the array until the process exits.
namespace kdop {
namespace {

constexpr int64_t kStaticQueueEntries = 65536;
constexpr size_t kStaticCtlBytes = 1024;
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
