// kdop_internal.h -- host-side structures shared by the C ABI and the kernels.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <thread>
#include <limits>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/kdop_cuda.h"

namespace kdop {

constexpr uint32_t LEAF_BIT_HOST = 0x80000000u;

// Unit directions of the K/2 slabs (geometry_direction_table.h:54-176).
struct DirTable {
  float d[13][3];
};

// Columns of a scene's candidate buffer (each cand_cap uint32).
constexpr int kCandCols = 5;

// Device-side control block of one traversal (+ contact generation).  The counters that every warp updates or polls
// while the traversal runs sit on 128-byte lines of their own, so that atomics
// and polls on one do not queue behind traffic on another in the same L2 slice.
struct TravCtl {
  unsigned long long tests;          // node-pair tests
  unsigned long long leaf_overlaps;  // overlapping leaf pairs before the surface filter
  unsigned int error;                // DEV_ERR_* bits
  unsigned int n_contacts;           // contacts emitted (may exceed capacity)
  unsigned int n_init;               // root pairs in this launch
  unsigned int pair_base;            // pair index of the first root pair
  unsigned int max_stack;            // deepest warp stack seen
  unsigned int n_surv;               // candidates past the contact pre-filter
  unsigned int n_mid;                // candidates past the face axes of the SAT test
  unsigned int pad0[21];
  unsigned int n_cand;               // candidates emitted (may exceed capacity)
  unsigned int pad1[31];
  unsigned int init_head;            // root pairs claimed
  unsigned int pad2[31];
  unsigned int q_head;               // queue slots claimed by idle warps
  unsigned int pad3[31];
  unsigned int q_tail;               // queue slots reserved by producers
  unsigned int pad4[31];
  int work;                          // outstanding work units; 0 = traversal finished
  unsigned int pad5[31];
};
static_assert(sizeof(TravCtl) == 768, "one 128-byte line per hot counter");

enum : unsigned int {
  DEV_ERR_TIMEOUT = 1u,
  DEV_ERR_QUEUE_FULL = 2u,
  DEV_ERR_BAD_INDEX = 4u,
};

struct TravParams {
  int block_warps;
  int stack_cap;
  int init_chunk;
  int donate_min;
  long long timeout_ns;
  int surface_filter;
  int load_group;
  int wave_pairs;
  int smem_carveout;
  int stuck_work;  // test hook: outstanding work units nobody completes
};

}  // namespace kdop

struct kdop_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  size_t smem_optin = 0;
  std::string err;
  long long launches = 0;
  // scenes alive on this context; a destroyed context is freed with its last scene
  int n_scenes = 0;
  bool destroy_pending = false;
  // autotuned traversal options keyed by (K, size class)
  std::map<std::pair<int, int>, kdop_traverse_opts> tuned;
  // grow-only device scratch of the contact reduction, freed with the context
  char* scratch = nullptr;
  size_t scratch_bytes = 0;
};

struct kdop_scene {
  kdop_ctx* ctx = nullptr;
  int K = 0;
  int NW = 0;  // float4 chunks per node record
  int n_meshes = 0;
  int64_t nv = 0, nt = 0, nn = 0;
  int depth = 0;
  std::vector<int64_t> v_off, t_off, level_off;
  std::vector<uint32_t> root;  // per mesh root node, 0xFFFFFFFF for an empty mesh
  kdop::DirTable dirs;

  // device arrays
  float4* rest = nullptr;
  float4* world = nullptr;
  float4* posed = nullptr;  // world positions a pose / deform refit computes before its leaf pass
  bool posed_valid = false;  // posed holds the positions of an executed pose / deform refit
  uint4* tets = nullptr;  // global vertex indices
  uint8_t* surf = nullptr;
  float4* nodes = nullptr;
  uint32_t* root_dev = nullptr;
  float4* quat = nullptr;
  float4* pos = nullptr;
  float4* lin_vel = nullptr;
  float4* ang_vel = nullptr;
  float* phase_dev = nullptr;  // deformation phase, advanced by the motion kernel
  float amp = 0.f, w = 0.f, phase = 0.f, phase_rate = 0.f;
  bool have_world = false;

  // traversal / contacts buffers
  uint2* pairs = nullptr;
  uint32_t* pair_order = nullptr;  // pair indices by decreasing size (tets of A + tets of B)
  int64_t pairs_cap = 0;
  uint32_t* cand = nullptr;  // kCandCols * cand_cap: A tets | B tets | pair ids | pre-filter survivors |
                             // candidates past the face axes of the SAT test
  int64_t cand_cap = 0;
  kdop_contact* contacts = nullptr;
  int4* records = nullptr;  // per candidate: faces, candidate codes, count, first contact
  int64_t contact_cap = 0;
  uint4* q_items = nullptr;
  uint32_t* q_tags = nullptr;
  int64_t queue_cap = 0;
  kdop::TravCtl* ctl = nullptr;
  kdop::TravCtl* ctl_host = nullptr;  // pinned

  int host_orders = 0;  // meshes whose leaf order came from the host (device build)
  int refit_mode = -1;
  bool traversed = false;
  bool contacted = false;
  int64_t last_pairs = 0;
  int last_mode = 0;
  kdop::TravParams last_params{};

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int64_t device_bytes = 0;
  int build = 0;  // KDOP_BUILD_DEVICE or KDOP_BUILD_HOST
};

namespace kdop {

// fn(0 .. n-1) on up to 64 host threads
template <typename F>
inline void parallel_for(int n, F fn) {
  int th = (int)std::thread::hardware_concurrency();
  if (th < 1) th = 1;
  if (th > 64) th = 64;
  if (th > n) th = n;
  if (th <= 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> pool;
  std::atomic<int> next(0);
  for (int t = 0; t < th; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        int i = next.fetch_add(1);
        if (i >= n) break;
        fn(i);
      }
    });
  for (auto& t : pool) t.join();
}

// host tree construction (kdop_build.cpp)
int direction_table(int K, float* out);
struct ForestBuild {
  std::vector<int64_t> level_off;          // per level start, size depth+2
  std::vector<uint32_t> topo;              // 2 per node: start, end (global ids)
  std::vector<uint32_t> root;              // per mesh
  int depth = 0;
};
// meshes: tet counts and concatenated (global-vertex) tets; t_off per mesh.
int build_forest(const std::vector<const float*>& xyz, const std::vector<int64_t>& n_verts,
                 const std::vector<const uint32_t*>& tets, const std::vector<int64_t>& n_tets,
                 const std::vector<const uint32_t*>& orders, const std::vector<int64_t>& t_off, ForestBuild& out);
void morton_order(const float* xyz, int64_t n_tets, const uint32_t* tets, std::vector<uint32_t>& perm);
// Level offsets, roots and per-level tree offsets (pre: levels x (meshes + 1))
// of the forest from the tet counts; lg[m] = floor(log2 n_tets[m]) or -1.
int forest_layout(const std::vector<int64_t>& n_tets, ForestBuild& out, std::vector<int64_t>& pre,
                  std::vector<int32_t>& lg);
// Morton scale of kdop_mesh_reorder.h from a mesh's centroid bounds; false
// when the reference's integer conversion would overflow.
bool morton_scale(const float* mn, const float* mx, int& scale);
// Device build of the leaf order: Morton codes of the rest centroids sorted
// per mesh on the GPU (ties by tet index); meshes whose codes tie, or whose
// scale degenerates, are flagged for the host order (std::sort's).
// perm (nt): global tet ids, mesh by mesh in leaf order.
cudaError_t device_morton_perm(kdop_scene* s, uint32_t* perm, std::vector<char>& need_host);
// Topology (m_start, m_end per node, global ids) of the forest from its
// layout and the leaf order perm; topo: 2 nn words.
cudaError_t device_topology(kdop_scene* s, const ForestBuild& fb, const std::vector<int64_t>& pre,
                            const std::vector<int32_t>& lg, const uint32_t* perm, uint32_t* topo);
void surface_map(int64_t n_tets, const uint32_t* tets, uint8_t* surf);

// kernel launchers (return cudaGetLastError of the launches)
cudaError_t launch_write_topology(kdop_scene* s, const uint32_t* topo_dev);
cudaError_t launch_refit(kdop_scene* s, int mode);
cudaError_t launch_traverse(kdop_scene* s, int64_t n_pairs, const uint2* pairs, const TravParams& p, int plain);
// broad phase (kdop_broad.cu)
cudaError_t launch_mesh_radius(kdop_scene* s, unsigned* rbits);
size_t broad_work_bytes(int n);
cudaError_t broad_phase(kdop_scene* s, const unsigned* rbits, const float* pos_dev, void* work, uint2* pairs,
                        int64_t cap, int64_t* total);
// Frontier-seeded traversal of shard `rank` of `n_ranks` (synchronises once,
// for the frontier's size); *work / *work_bytes: the scene's scratch for it,
// grown here; *n_entries = frontier pairs this shard started from.
cudaError_t launch_traverse_shard(kdop_scene* s, int64_t n_pairs, const uint2* pairs, const TravParams& p, int rank,
                                  int n_ranks, int64_t frontier_min, void** work, size_t* work_bytes,
                                  int64_t* n_entries);
cudaError_t launch_contacts(kdop_scene* s);
// contact reduction (kdop_reduce.cu)
size_t reduce_work_bytes(int64_t n);
cudaError_t reduce_contact_rows(kdop_ctx* ctx, const kdop_contact* rows, const uint2* bodies, int64_t n, void* work,
                                kdop_contact* out, uint2* out_bodies, int64_t* n_out);
cudaError_t scene_contact_bodies(kdop_scene* s, int64_t n, uint2* bodies);
cudaError_t launch_adjoint(kdop_scene* s, const float* dd, const float* dn, float* grad);
cudaError_t launch_motion(kdop_scene* s);
cudaError_t launch_world(kdop_scene* s, int mode, float4* out);
int traverse_block_threads(int block_warps);

}  // namespace kdop

// Defaults + validation of traversal options (kdop_capi.cpp).
int kdop_resolve_traverse_opts(const kdop_scene* s, const kdop_traverse_opts* o, kdop::TravParams& p, int& mode);

namespace kdop {
size_t traverse_smem_bytes(int block_warps, int stack_cap);
cudaError_t traverse_prepare(int K, size_t smem);

}  // namespace kdop
