// kdop_capi.cpp -- the C ABI of include/kdop_cuda.h: contexts, scenes,
// device-buffer management, statistics, CUDA-graph capture and the autotuner.
// Kernels live in kdop_refit.cu, kdop_traverse.cu and kdop_contacts.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "kdop_internal.h"
#include "kdop_sort.h"

using kdop::TravCtl;

namespace {

const int64_t kDefaultCand = 1 << 20;
const int64_t kDefaultContacts = 1 << 20;
const int64_t kDefaultQueue = 1 << 20;

int fail(kdop_ctx* ctx, int status, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return status;
}

int cuda_fail(kdop_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return fail(ctx, KDOP_ERR_CUDA, m);
}

#define KDOP_CUDA(ctx, call)                                   \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
  } while (0)

bool valid_K(int K) { return K == 6 || K == 8 || K == 12 || K == 14 || K == 18 || K == 20 || K == 26; }

template <typename T>
cudaError_t dalloc(kdop_scene* s, T** p, int64_t n) {
  *p = nullptr;
  if (n <= 0) n = 1;
  size_t bytes = (size_t)n * sizeof(T);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e == cudaSuccess) s->device_bytes += (int64_t)bytes;
  return e;
}

template <typename T>
void dfree(kdop_scene* s, T** p, int64_t n) {
  if (*p) {
    cudaFree(*p);
    s->device_bytes -= (int64_t)((n <= 0 ? 1 : n) * sizeof(T));
  }
  *p = nullptr;
}

}  // namespace

namespace kdop {
cudaError_t launch_pack3(kdop_scene* s, const float* in, float4* out, int64_t n, int with_mesh_id);
cudaError_t launch_pack4(kdop_scene* s, const float* in, float4* out, int64_t n);
}  // namespace kdop

struct kdop_scene_ext {
  float* stage = nullptr;
  int64_t stage_n = 0;
  void* sort_work = nullptr;  // kdop_sort_results scratch
  size_t sort_work_bytes = 0;
  void* shard_work = nullptr;  // kdop_traverse_shard scratch
  size_t shard_work_bytes = 0;
  unsigned* radius_bits = nullptr;  // broad phase: bounding radius per mesh (float bits)
  void* broad_work = nullptr;
  size_t broad_work_bytes = 0;
  uint2* broad_pairs = nullptr;
  int64_t broad_cap = 0;
  float* broad_pos = nullptr;
  std::vector<uint32_t> pairs_host;  // last traversed mesh pairs
  std::vector<uint32_t> order_host;  // their order of processing
  int64_t graph_kernels = 0;
  int graph_refit_mode = 0;  // refit mode of the captured step
  kdop_traverse_opts tuned{};
  bool has_tuned = false;
};

static kdop_scene_ext* ext(kdop_scene* s);

// The extension block lives right after the scene object (allocated together).
struct SceneBox {
  kdop_scene s;
  kdop_scene_ext x;
};
static kdop_scene_ext* ext(kdop_scene* s) { return &reinterpret_cast<SceneBox*>(s)->x; }

static float* stage(kdop_scene* s, int64_t nfloats, cudaError_t* err) {
  kdop_scene_ext* x = ext(s);
  *err = cudaSuccess;
  if (x->stage_n < nfloats) {
    if (x->stage) {
      cudaFree(x->stage);
      s->device_bytes -= x->stage_n * 4;
    }
    x->stage = nullptr;
    x->stage_n = 0;
    *err = cudaMalloc((void**)&x->stage, (size_t)std::max<int64_t>(nfloats, 1) * 4);
    if (*err != cudaSuccess) return nullptr;
    x->stage_n = std::max<int64_t>(nfloats, 1);
    s->device_bytes += x->stage_n * 4;
  }
  return x->stage;
}

extern "C" {

int kdop_api_version(void) { return KDOP_API_VERSION; }

const char* kdop_status_string(int status) {
  switch (status) {
    case KDOP_OK: return "ok";
    case KDOP_ERR_INVALID: return "invalid argument";
    case KDOP_ERR_CAPACITY: return "capacity exceeded";
    case KDOP_ERR_CUDA: return "CUDA error";
    case KDOP_ERR_TIMEOUT: return "device wait timed out";
    case KDOP_ERR_NOMEM: return "out of memory";
    case KDOP_ERR_STATE: return "call out of order";
  }
  return "unknown status";
}

const char* kdop_last_error(const kdop_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int kdop_ctx_create(int device, kdop_ctx** out) {
  if (!out) return KDOP_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return KDOP_ERR_CUDA;
  }
  if (device < 0 || device >= n) return KDOP_ERR_INVALID;
  kdop_ctx* c = new (std::nothrow) kdop_ctx();
  if (!c) return KDOP_ERR_NOMEM;
  c->device = device;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  int optin = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  c->smem_optin = (size_t)optin;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return KDOP_ERR_CUDA;
  }
  c->own_stream = true;
  *out = c;
  return KDOP_OK;
}

static void ctx_free(kdop_ctx* ctx) {
  cudaSetDevice(ctx->device);
  if (ctx->scratch) cudaFree(ctx->scratch);  // waits for the device
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int kdop_ctx_destroy(kdop_ctx* ctx) {
  if (!ctx || ctx->destroy_pending) return KDOP_ERR_INVALID;
  // scenes keep using the context's stream: free it with the last scene
  if (ctx->n_scenes > 0) {
    ctx->destroy_pending = true;
    return KDOP_OK;
  }
  ctx_free(ctx);
  return KDOP_OK;
}

int kdop_ctx_set_stream(kdop_ctx* ctx, void* stream) {
  if (!ctx) return KDOP_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->own_stream = false;
  ctx->stream = (cudaStream_t)stream;
  if (!stream) {
    KDOP_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return KDOP_OK;
}

void* kdop_ctx_stream(const kdop_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int kdop_ctx_synchronize(kdop_ctx* ctx) {
  if (!ctx) return KDOP_ERR_INVALID;
  cudaSetDevice(ctx->device);
  KDOP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return KDOP_OK;
}

int64_t kdop_ctx_launch_count(const kdop_ctx* ctx) { return ctx ? ctx->launches : 0; }

static void scene_free(kdop_scene* s) {
  kdop_scene_ext* x = ext(s);
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->graph_exec = nullptr;
  s->graph = nullptr;
  dfree(s, &s->rest, s->nv);
  dfree(s, &s->world, s->nv);
  dfree(s, &s->posed, s->nv);
  dfree(s, &s->tets, s->nt);
  dfree(s, &s->surf, s->nt);
  dfree(s, &s->nodes, s->nn * s->NW);
  if (s->root_dev) cudaFree(s->root_dev);
  s->root_dev = nullptr;
  dfree(s, &s->quat, s->n_meshes);
  dfree(s, &s->pos, s->n_meshes);
  dfree(s, &s->lin_vel, s->n_meshes);
  dfree(s, &s->ang_vel, s->n_meshes);
  dfree(s, &s->phase_dev, 1);
  dfree(s, &s->pairs, s->pairs_cap);
  dfree(s, &s->pair_order, s->pairs_cap);
  dfree(s, &s->cand, kdop::kCandCols * s->cand_cap);
  dfree(s, &s->contacts, s->contact_cap);
  dfree(s, &s->records, s->cand_cap);
  dfree(s, &s->q_items, s->queue_cap);
  dfree(s, &s->q_tags, s->queue_cap);
  dfree(s, &s->ctl, 1);
  if (s->ctl_host) cudaFreeHost(s->ctl_host);
  s->ctl_host = nullptr;
  if (x->stage) cudaFree(x->stage);
  x->stage = nullptr;
  if (x->sort_work) cudaFree(x->sort_work);
  x->sort_work = nullptr;
  x->sort_work_bytes = 0;
  if (x->shard_work) cudaFree(x->shard_work);
  x->shard_work = nullptr;
  x->shard_work_bytes = 0;
  if (x->radius_bits) cudaFree(x->radius_bits);
  if (x->broad_work) cudaFree(x->broad_work);
  if (x->broad_pairs) cudaFree(x->broad_pairs);
  if (x->broad_pos) cudaFree(x->broad_pos);
  x->radius_bits = nullptr;
  x->broad_work = nullptr;
  x->broad_pairs = nullptr;
  x->broad_pos = nullptr;
  x->broad_work_bytes = 0;
  x->broad_cap = 0;
}

// A captured graph holds the buffer addresses of its capture: any
// reallocation drops the graph (kdop_graph_launch then reports
// KDOP_ERR_STATE until the step is captured again).
static void drop_graph(kdop_scene* s) {
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->graph_exec = nullptr;
  s->graph = nullptr;
}

static int grow_candidates(kdop_scene* s, int64_t n) {
  if (n <= s->cand_cap) return KDOP_OK;
  drop_graph(s);
  dfree(s, &s->cand, kdop::kCandCols * s->cand_cap);
  dfree(s, &s->records, s->cand_cap);
  s->cand_cap = 0;
  if (n >= (int64_t)0xFFFFFFF0ll) return fail(s->ctx, KDOP_ERR_CAPACITY, "candidate capacity above 2^32");
  KDOP_CUDA(s->ctx, dalloc(s, &s->cand, kdop::kCandCols * n));
  KDOP_CUDA(s->ctx, dalloc(s, &s->records, n));
  s->cand_cap = n;
  return KDOP_OK;
}

static int grow_contacts(kdop_scene* s, int64_t n) {
  if (n <= s->contact_cap) return KDOP_OK;
  drop_graph(s);
  dfree(s, &s->contacts, s->contact_cap);
  s->contact_cap = 0;
  if (n >= (int64_t)0xFFFFFFF0ll) return fail(s->ctx, KDOP_ERR_CAPACITY, "contact capacity above 2^32");
  KDOP_CUDA(s->ctx, dalloc(s, &s->contacts, n));
  s->contact_cap = n;
  return KDOP_OK;
}

static int grow_queue(kdop_scene* s, int64_t n) {
  if (n <= s->queue_cap) return KDOP_OK;
  drop_graph(s);
  dfree(s, &s->q_items, s->queue_cap);
  dfree(s, &s->q_tags, s->queue_cap);
  s->queue_cap = 0;
  if (n >= (int64_t)0x7FFFFFF0ll) return fail(s->ctx, KDOP_ERR_CAPACITY, "queue capacity above 2^31");
  KDOP_CUDA(s->ctx, dalloc(s, &s->q_items, n));
  KDOP_CUDA(s->ctx, dalloc(s, &s->q_tags, n));
  KDOP_CUDA(s->ctx, cudaMemsetAsync(s->q_tags, 0, (size_t)n * 4, s->ctx->stream));
  s->queue_cap = n;
  return KDOP_OK;
}

static int grow_pairs(kdop_scene* s, int64_t n) {
  if (n <= s->pairs_cap) return KDOP_OK;
  drop_graph(s);
  dfree(s, &s->pairs, s->pairs_cap);
  dfree(s, &s->pair_order, s->pairs_cap);
  s->pairs_cap = 0;
  KDOP_CUDA(s->ctx, dalloc(s, &s->pair_order, n));
  KDOP_CUDA(s->ctx, dalloc(s, &s->pairs, n));
  s->pairs_cap = n;
  return KDOP_OK;
}

int kdop_scene_create(kdop_ctx* ctx, int K, int n_meshes, const kdop_mesh_desc* meshes, kdop_scene** out) {
  return kdop_scene_create_ex(ctx, K, n_meshes, meshes, KDOP_BUILD_DEVICE, out);
}

int kdop_scene_create_ex(kdop_ctx* ctx, int K, int n_meshes, const kdop_mesh_desc* meshes, int build,
                         kdop_scene** out) {
  if (!ctx || !out) return KDOP_ERR_INVALID;
  if (build != KDOP_BUILD_DEVICE && build != KDOP_BUILD_HOST) return fail(ctx, KDOP_ERR_INVALID, "unknown build mode");
  *out = nullptr;
  if (!valid_K(K)) return fail(ctx, KDOP_ERR_INVALID, "K must be one of 6, 8, 12, 14, 18, 20, 26");
  if (n_meshes < 0 || (n_meshes > 0 && !meshes)) return fail(ctx, KDOP_ERR_INVALID, "bad mesh list");
  int64_t nv = 0, nt = 0;
  for (int m = 0; m < n_meshes; ++m) {
    const kdop_mesh_desc& d = meshes[m];
    if (d.n_verts < 0 || d.n_tets < 0) return fail(ctx, KDOP_ERR_INVALID, "negative mesh size");
    if ((d.n_verts > 0 && !d.xyz) || (d.n_tets > 0 && !d.tets))
      return fail(ctx, KDOP_ERR_INVALID, "null mesh array");
    for (int64_t i = 0; i < 4 * d.n_tets; ++i)
      if ((int64_t)d.tets[i] >= d.n_verts)
        return fail(ctx, KDOP_ERR_INVALID, "tet vertex index out of range in mesh " + std::to_string(m));
    if (d.leaf_order) {
      std::vector<char> seen((size_t)d.n_tets, 0);
      for (int64_t i = 0; i < d.n_tets; ++i) {
        uint32_t t = d.leaf_order[i];
        if ((int64_t)t >= d.n_tets || seen[t])
          return fail(ctx, KDOP_ERR_INVALID, "leaf_order is not a permutation in mesh " + std::to_string(m));
        seen[t] = 1;
      }
    }
    nv += d.n_verts;
    nt += d.n_tets;
  }
  if (nv >= (int64_t)0x7FFFFFFF || nt >= (int64_t)0x3FFFFFFF)
    return fail(ctx, KDOP_ERR_INVALID, "scene too large for 32-bit indices");
  KDOP_CUDA(ctx, cudaSetDevice(ctx->device));
  SceneBox* box = new (std::nothrow) SceneBox();
  if (!box) return KDOP_ERR_NOMEM;
  kdop_scene* s = &box->s;
  s->ctx = ctx;
  s->K = K;
  s->NW = (K + 2 + 3) / 4;
  s->n_meshes = n_meshes;
  s->nv = nv;
  s->nt = nt;
  s->v_off.assign((size_t)n_meshes + 1, 0);
  s->t_off.assign((size_t)n_meshes + 1, 0);
  for (int m = 0; m < n_meshes; ++m) {
    s->v_off[m + 1] = s->v_off[m] + meshes[m].n_verts;
    s->t_off[m + 1] = s->t_off[m] + meshes[m].n_tets;
  }
  std::memset(&s->dirs, 0, sizeof(s->dirs));
  kdop::direction_table(K, &s->dirs.d[0][0]);

  // host tree build
  std::vector<const float*> xyz((size_t)n_meshes);
  std::vector<const uint32_t*> tets((size_t)n_meshes);
  std::vector<int64_t> nvs((size_t)n_meshes), nts((size_t)n_meshes);
  std::vector<const uint32_t*> orders((size_t)n_meshes);
  for (int m = 0; m < n_meshes; ++m) {
    xyz[m] = meshes[m].xyz;
    tets[m] = meshes[m].tets;
    orders[m] = meshes[m].leaf_order;
    nvs[m] = meshes[m].n_verts;
    nts[m] = meshes[m].n_tets;
  }
  kdop::ForestBuild fb;
  std::vector<int64_t> pre;
  std::vector<int32_t> lg;
  int brc = build == KDOP_BUILD_HOST ? kdop::build_forest(xyz, nvs, tets, nts, orders, s->t_off, fb)
                                     : kdop::forest_layout(nts, fb, pre, lg);
  if (brc != 0) {
    delete box;
    return fail(ctx, KDOP_ERR_INVALID, "scene too large for 30-bit node indices");
  }
  s->build = build;
  s->level_off = fb.level_off;
  s->root = fb.root;
  s->nn = fb.level_off.empty() ? 0 : fb.level_off.back();
  s->depth = fb.depth;

  // host staging of meshes
  std::vector<float4> rest((size_t)std::max<int64_t>(nv, 1));
  std::vector<uint4> gt((size_t)std::max<int64_t>(nt, 1));
  std::vector<uint8_t> surf((size_t)std::max<int64_t>(nt, 1));
  kdop::parallel_for(n_meshes, [&](int m) {
    const kdop_mesh_desc& d = meshes[m];
    int mid = m;
    float midf;
    std::memcpy(&midf, &mid, 4);
    for (int64_t i = 0; i < d.n_verts; ++i)
      rest[s->v_off[m] + i] = make_float4(d.xyz[3 * i], d.xyz[3 * i + 1], d.xyz[3 * i + 2], midf);
    uint32_t vo = (uint32_t)s->v_off[m];
    for (int64_t t = 0; t < d.n_tets; ++t)
      gt[s->t_off[m] + t] = make_uint4(d.tets[4 * t] + vo, d.tets[4 * t + 1] + vo, d.tets[4 * t + 2] + vo,
                                       d.tets[4 * t + 3] + vo);
    if (d.surface)
      std::memcpy(&surf[s->t_off[m]], d.surface, (size_t)d.n_tets);
    else if (d.n_tets)
      kdop::surface_map(d.n_tets, d.tets, &surf[s->t_off[m]]);
  });

  int rc = KDOP_OK;
  cudaStream_t st = ctx->stream;
  uint32_t* topo_dev = nullptr;
  uint32_t* perm_dev = nullptr;
  do {
    cudaError_t e;
#define SC_TRY(call)                                 \
  if ((e = (call)) != cudaSuccess) {                 \
    rc = cuda_fail(ctx, e, #call);                   \
    break;                                           \
  }
    SC_TRY(dalloc(s, &s->rest, nv));
    SC_TRY(dalloc(s, &s->world, nv));
    SC_TRY(dalloc(s, &s->posed, nv));
    SC_TRY(dalloc(s, &s->tets, nt));
    SC_TRY(dalloc(s, &s->surf, nt));
    SC_TRY(dalloc(s, &s->nodes, s->nn * s->NW));
    size_t root_bytes = (size_t)n_meshes * 4;
    SC_TRY(cudaMalloc((void**)&s->root_dev, std::max<size_t>(root_bytes, 8)));
    s->device_bytes += (int64_t)root_bytes;
    SC_TRY(dalloc(s, &s->quat, n_meshes));
    SC_TRY(dalloc(s, &s->pos, n_meshes));
    SC_TRY(dalloc(s, &s->lin_vel, n_meshes));
    SC_TRY(dalloc(s, &s->ang_vel, n_meshes));
    SC_TRY(dalloc(s, &s->phase_dev, 1));
    SC_TRY(dalloc(s, &s->ctl, 1));
    SC_TRY(cudaMallocHost((void**)&s->ctl_host, sizeof(TravCtl)));
    std::memset(s->ctl_host, 0, sizeof(TravCtl));
    SC_TRY(cudaMemcpyAsync(s->rest, rest.data(), (size_t)nv * sizeof(float4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemcpyAsync(s->world, rest.data(), (size_t)nv * sizeof(float4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemcpyAsync(s->tets, gt.data(), (size_t)nt * sizeof(uint4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemcpyAsync(s->surf, surf.data(), (size_t)nt, cudaMemcpyHostToDevice, st));
    std::vector<uint8_t> rbuf(std::max<size_t>(root_bytes, 8), 0);
    if (n_meshes) std::memcpy(rbuf.data(), s->root.data(), (size_t)n_meshes * 4);
    SC_TRY(cudaMemcpyAsync(s->root_dev, rbuf.data(), root_bytes, cudaMemcpyHostToDevice, st));
    std::vector<float4> q((size_t)std::max(n_meshes, 1), make_float4(1.f, 0.f, 0.f, 0.f));
    std::vector<float4> z((size_t)std::max(n_meshes, 1), make_float4(0.f, 0.f, 0.f, 0.f));
    SC_TRY(cudaMemcpyAsync(s->quat, q.data(), (size_t)n_meshes * sizeof(float4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemcpyAsync(s->pos, z.data(), (size_t)n_meshes * sizeof(float4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemcpyAsync(s->lin_vel, z.data(), (size_t)n_meshes * sizeof(float4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemcpyAsync(s->ang_vel, z.data(), (size_t)n_meshes * sizeof(float4), cudaMemcpyHostToDevice, st));
    SC_TRY(cudaMemsetAsync(s->phase_dev, 0, sizeof(float), st));
    SC_TRY(cudaMemsetAsync(s->ctl, 0, sizeof(TravCtl), st));
    SC_TRY(cudaMalloc((void**)&topo_dev, (size_t)std::max<int64_t>(2 * s->nn, 1) * 4));
    if (build == KDOP_BUILD_HOST) {
      SC_TRY(cudaMemcpyAsync(topo_dev, fb.topo.data(), fb.topo.size() * 4, cudaMemcpyHostToDevice, st));
    } else {
      // leaf order on the device; caller-given orders and meshes whose Morton
      // codes tie take the host's order
      SC_TRY(cudaMalloc((void**)&perm_dev, (size_t)std::max<int64_t>(nt, 1) * 4));
      std::vector<char> need_host;
      SC_TRY(kdop::device_morton_perm(s, perm_dev, need_host));
      std::vector<int> hm;
      for (int m = 0; m < n_meshes; ++m)
        if (meshes[m].n_tets > 0 && (meshes[m].leaf_order || need_host[m])) hm.push_back(m);
      std::vector<std::vector<uint32_t> > hperm(hm.size());
      kdop::parallel_for((int)hm.size(), [&](int k) {
        int m = hm[k];
        if (meshes[m].leaf_order)
          hperm[k].assign(meshes[m].leaf_order, meshes[m].leaf_order + meshes[m].n_tets);
        else
          kdop::morton_order(meshes[m].xyz, meshes[m].n_tets, meshes[m].tets, hperm[k]);
        for (auto& t : hperm[k]) t += (uint32_t)s->t_off[m];
      });
      for (size_t k = 0; k < hm.size(); ++k)
        SC_TRY(cudaMemcpyAsync(perm_dev + s->t_off[hm[k]], hperm[k].data(), hperm[k].size() * 4,
                               cudaMemcpyHostToDevice, st));
      if (rc != KDOP_OK) break;
      SC_TRY(kdop::device_topology(s, fb, pre, lg, perm_dev, topo_dev));
      s->host_orders = (int)hm.size();
    }
    SC_TRY(kdop::launch_write_topology(s, topo_dev));
    // make_tree ends with a refit (kdop_make_tree.h:285)
    SC_TRY(kdop::launch_refit(s, KDOP_REFIT_VERTICES));
    s->refit_mode = KDOP_REFIT_VERTICES;
    s->have_world = true;
    SC_TRY(cudaStreamSynchronize(st));
#undef SC_TRY
  } while (0);
  if (topo_dev) cudaFree(topo_dev);
  if (perm_dev) cudaFree(perm_dev);
  if (rc == KDOP_OK) rc = grow_candidates(s, kDefaultCand);
  if (rc == KDOP_OK) rc = grow_contacts(s, kDefaultContacts);
  if (rc == KDOP_OK) rc = grow_queue(s, kDefaultQueue);
  if (rc == KDOP_OK) rc = grow_pairs(s, std::max(n_meshes, 1));
  if (rc != KDOP_OK) {
    scene_free(s);
    delete box;
    return rc;
  }
  ctx->n_scenes++;
  *out = s;
  return KDOP_OK;
}

int kdop_scene_destroy(kdop_scene* s) {
  if (!s) return KDOP_ERR_INVALID;
  kdop_ctx* ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  scene_free(s);
  delete reinterpret_cast<SceneBox*>(s);
  if (--ctx->n_scenes == 0 && ctx->destroy_pending) ctx_free(ctx);
  return KDOP_OK;
}

int kdop_scene_get_info(const kdop_scene* s, kdop_scene_info* info) {
  if (!s || !info) return KDOP_ERR_INVALID;
  info->K = s->K;
  info->n_meshes = s->n_meshes;
  info->n_verts = s->nv;
  info->n_tets = s->nt;
  info->n_nodes = s->nn;
  info->depth = s->depth;
  info->node_bytes = s->NW * 16;
  info->build = s->build;
  info->host_orders = s->host_orders;
  info->device_bytes = s->device_bytes;
  return KDOP_OK;
}

int kdop_read_tree(kdop_scene* s, int mesh, int64_t cap, float* vol, int64_t* tet, int64_t* n_nodes) {
  if (!s || mesh < 0 || mesh >= s->n_meshes || !n_nodes) return KDOP_ERR_INVALID;
  int64_t ntm = s->t_off[mesh + 1] - s->t_off[mesh];
  *n_nodes = ntm > 0 ? 2 * ntm - 1 : 0;
  if (*n_nodes == 0) return KDOP_OK;
  if (cap < *n_nodes) return fail(s->ctx, KDOP_ERR_CAPACITY, "tree read buffer too small");
  if (!vol || !tet) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  std::vector<float> rec((size_t)(s->nn * s->NW * 4));
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(rec.data(), s->nodes, rec.size() * 4, cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  const int tw = s->K;  // word index of `start`
  std::vector<uint32_t> stack(1, s->root[mesh]);
  int64_t k = 0;
  while (!stack.empty()) {
    uint32_t n = stack.back();
    stack.pop_back();
    // chunk j of node n sits at float4 2 NW (n / 2) + 2 j + n % 2 (twin records)
    float r[32];  // NW <= 7 chunks
    for (int j = 0; j < s->NW; ++j)
      std::memcpy(r + 4 * j, &rec[4 * (size_t)((int64_t)(n >> 1) * 2 * s->NW + 2 * j + (n & 1))], 16);
    // topology words: leaf (LEAF_BIT | flags | own index, tet), internal (c, c + 1)
    uint32_t w0, w1;
    std::memcpy(&w0, r + tw, 4);
    std::memcpy(&w1, r + tw + 1, 4);
    if (k >= *n_nodes) return fail(s->ctx, KDOP_ERR_STATE, "tree walk overran the node count");
    std::memcpy(vol + k * s->K, r, (size_t)s->K * 4);
    if (w0 & kdop::LEAF_BIT_HOST) {
      tet[k] = (int64_t)w1 - s->t_off[mesh];
    } else {
      tet[k] = -1;
      stack.push_back(w1);
      stack.push_back(w0);
    }
    ++k;
  }
  return KDOP_OK;
}

int kdop_set_vertices(kdop_scene* s, const float* xyz, int64_t n, int memory) {
  if (!s || (n > 0 && !xyz) || n != s->nv) return s ? fail(s->ctx, KDOP_ERR_INVALID, "vertex count mismatch") : KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  if (n == 0) return KDOP_OK;
  const float* src = xyz;
  if (memory == KDOP_HOST) {
    cudaError_t e;
    float* d = stage(s, 3 * n, &e);
    if (!d) return cuda_fail(s->ctx, e, "staging alloc");
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(d, xyz, (size_t)n * 12, cudaMemcpyHostToDevice, s->ctx->stream));
    src = d;
  }
  KDOP_CUDA(s->ctx, kdop::launch_pack3(s, src, s->world, n, 0));
  s->have_world = true;
  return KDOP_OK;
}

int kdop_set_poses(kdop_scene* s, const float* quat, const float* pos, int memory) {
  if (!s || (s->n_meshes > 0 && (!quat || !pos))) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  int64_t n = s->n_meshes;
  if (n == 0) return KDOP_OK;
  const float* q = quat;
  const float* p = pos;
  if (memory == KDOP_HOST) {
    cudaError_t e;
    float* d = stage(s, 7 * n, &e);
    if (!d) return cuda_fail(s->ctx, e, "staging alloc");
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(d, quat, (size_t)n * 16, cudaMemcpyHostToDevice, s->ctx->stream));
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(d + 4 * n, pos, (size_t)n * 12, cudaMemcpyHostToDevice, s->ctx->stream));
    q = d;
    p = d + 4 * n;
  }
  KDOP_CUDA(s->ctx, kdop::launch_pack4(s, q, s->quat, n));
  KDOP_CUDA(s->ctx, kdop::launch_pack3(s, p, s->pos, n, -1));
  return KDOP_OK;
}

int kdop_set_deformation(kdop_scene* s, float amp, float w, float phase) {
  if (!s) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  s->amp = amp;
  s->w = w;
  s->phase = phase;
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->phase_dev, &s->phase, 4, cudaMemcpyHostToDevice, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  return KDOP_OK;
}

int kdop_set_motion(kdop_scene* s, const float* lin, const float* ang, float phase_rate, int memory) {
  if (!s || (s->n_meshes > 0 && (!lin || !ang))) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  int64_t n = s->n_meshes;
  s->phase_rate = phase_rate;
  if (n == 0) return KDOP_OK;
  const float* l = lin;
  const float* a = ang;
  if (memory == KDOP_HOST) {
    cudaError_t e;
    float* d = stage(s, 6 * n, &e);
    if (!d) return cuda_fail(s->ctx, e, "staging alloc");
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(d, lin, (size_t)n * 12, cudaMemcpyHostToDevice, s->ctx->stream));
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(d + 3 * n, ang, (size_t)n * 12, cudaMemcpyHostToDevice, s->ctx->stream));
    l = d;
    a = d + 3 * n;
  }
  KDOP_CUDA(s->ctx, kdop::launch_pack3(s, l, s->lin_vel, n, -1));
  KDOP_CUDA(s->ctx, kdop::launch_pack3(s, a, s->ang_vel, n, -1));
  return KDOP_OK;
}

// The contact kernels and the adjoint read the posed vertex array after a
// pose / deform refit.  A mode set by a graph capture whose step has not run
// yet leaves it unwritten: pose the vertices with the current poses first.
static cudaError_t ensure_posed(kdop_scene* s) {
  if (s->refit_mode <= KDOP_REFIT_VERTICES || s->posed_valid) return cudaSuccess;
  cudaError_t e = kdop::launch_world(s, s->refit_mode, s->posed);
  if (e == cudaSuccess) s->posed_valid = true;
  return e;
}

int kdop_refit(kdop_scene* s, int mode) {
  if (!s) return KDOP_ERR_INVALID;
  if (mode < KDOP_REFIT_VERTICES || mode > KDOP_REFIT_DEFORM) return fail(s->ctx, KDOP_ERR_INVALID, "bad refit mode");
  cudaSetDevice(s->ctx->device);
  s->refit_mode = mode;
  KDOP_CUDA(s->ctx, kdop::launch_refit(s, mode));
  if (mode != KDOP_REFIT_VERTICES) s->posed_valid = true;
  return KDOP_OK;
}

int kdop_read_vertices(kdop_scene* s, float* xyz, int64_t cap) {
  if (!s || cap < s->nv || (s->nv > 0 && !xyz)) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  if (s->nv == 0) return KDOP_OK;
  std::vector<float4> h((size_t)s->nv);
  float4* src = s->world;
  if (s->refit_mode > KDOP_REFIT_VERTICES) {
    KDOP_CUDA(s->ctx, ensure_posed(s));
    src = s->posed;
  }
  cudaError_t e = cudaMemcpyAsync(h.data(), src, (size_t)s->nv * sizeof(float4), cudaMemcpyDeviceToHost, s->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "read vertices");
  for (int64_t i = 0; i < s->nv; ++i) {
    xyz[3 * i] = h[i].x;
    xyz[3 * i + 1] = h[i].y;
    xyz[3 * i + 2] = h[i].z;
  }
  return KDOP_OK;
}

}  // extern "C"

int kdop_resolve_traverse_opts(const kdop_scene* s, const kdop_traverse_opts* o, kdop::TravParams& p, int& mode) {
  kdop_traverse_opts d;
  kdop_traverse_opts_default(s, &d);
  if (!o) o = &d;
  mode = o->mode;
  if (mode != KDOP_TRAVERSE_BATCHED && mode != KDOP_TRAVERSE_PLAIN) return KDOP_ERR_INVALID;
  p.block_warps = o->block_warps > 0 ? o->block_warps : d.block_warps;
  p.stack_cap = o->stack_cap > 0 ? o->stack_cap : d.stack_cap;
  p.init_chunk = o->init_chunk > 0 ? o->init_chunk : d.init_chunk;
  p.donate_min = o->donate_min > 0 ? o->donate_min : d.donate_min;
  p.timeout_ns = (long long)(o->timeout_ms > 0 ? o->timeout_ms : 5000) * 1000000ll;
  p.surface_filter = o->surface_filter ? 1 : 0;
  p.load_group = o->load_group > 0 ? o->load_group : d.load_group;
  p.wave_pairs = o->wave_pairs > 0 ? o->wave_pairs : (o->wave_pairs < 0 ? -1 : d.wave_pairs);
  p.smem_carveout = o->smem_carveout > 0 ? o->smem_carveout : (o->smem_carveout < 0 ? -1 : d.smem_carveout);
  if (p.wave_pairs < 0) p.wave_pairs = 0;
  if (p.smem_carveout < 0) p.smem_carveout = 0;
  p.stuck_work = o->test_stuck_work;
  if (p.stuck_work < 0 || p.stuck_work > 1024) return KDOP_ERR_INVALID;
  if (p.smem_carveout > 100) return KDOP_ERR_INVALID;
  if (p.block_warps > 16 || (p.stack_cap & (p.stack_cap - 1)) || p.stack_cap < 64 || p.init_chunk > 32)
    return KDOP_ERR_INVALID;
  if (p.load_group != 1 && p.load_group != 2 && p.load_group != 4 && p.load_group != 8) return KDOP_ERR_INVALID;
  if (kdop::traverse_smem_bytes(p.block_warps, p.stack_cap) > s->ctx->smem_optin) return KDOP_ERR_INVALID;
  return KDOP_OK;
}

// Size class of a scene for the autotuner's cache: floor(log2(tets of all
// its meshes)).
static int tune_size_class(const kdop_scene* s) {
  const int64_t tets = s->t_off.empty() ? 0 : s->t_off.back();
  return tets > 0 ? (int)std::log2((double)tets) : 0;
}

extern "C" {

int kdop_traverse_opts_default(const kdop_scene* s, kdop_traverse_opts* o) {
  if (!o) return KDOP_ERR_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->mode = KDOP_TRAVERSE_BATCHED;
  o->surface_filter = 1;
  o->block_warps = 16;
  o->stack_cap = 512;
  o->init_chunk = 1;
  o->donate_min = 128;
  o->timeout_ms = 5000;
  o->load_group = 4;
  o->wave_pairs = 0;
  o->smem_carveout = 0;
  if (s) {
    // this scene's own autotuned choice, else one cached on the context for
    // the same K and size class
    kdop_scene_ext* x = ext(const_cast<kdop_scene*>(s));
    const kdop_traverse_opts* t = nullptr;
    if (x->has_tuned) {
      t = &x->tuned;
    } else {
      auto it = s->ctx->tuned.find(std::make_pair(s->K, tune_size_class(s)));
      if (it != s->ctx->tuned.end()) t = &it->second;
    }
    if (t) {
      o->block_warps = t->block_warps;
      o->stack_cap = t->stack_cap;
      o->init_chunk = t->init_chunk;
      o->donate_min = t->donate_min;
      o->load_group = t->load_group;
      o->wave_pairs = t->wave_pairs;
      o->smem_carveout = t->smem_carveout;
    }
  }
  return KDOP_OK;
}

static int upload_pairs(kdop_scene* s, int64_t n, const uint32_t* pairs, int memory) {
  kdop_scene_ext* x = ext(s);
  int rc = grow_pairs(s, std::max<int64_t>(n, 1));
  if (rc != KDOP_OK) return rc;
  if (n == 0) {
    x->pairs_host.clear();
    return KDOP_OK;
  }
  if (memory == KDOP_HOST) {
    for (int64_t i = 0; i < 2 * n; ++i)
      if ((int64_t)pairs[i] >= s->n_meshes) return fail(s->ctx, KDOP_ERR_INVALID, "mesh index out of range in pairs");
    x->pairs_host.assign(pairs, pairs + 2 * n);
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->pairs, pairs, (size_t)n * 8, cudaMemcpyHostToDevice, s->ctx->stream));
  } else {
    x->pairs_host.assign((size_t)(2 * n), 0);
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(x->pairs_host.data(), pairs, (size_t)n * 8, cudaMemcpyDeviceToHost,
                                      s->ctx->stream));
    KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    for (int64_t i = 0; i < 2 * n; ++i)
      if ((int64_t)x->pairs_host[i] >= s->n_meshes)
        return fail(s->ctx, KDOP_ERR_INVALID, "mesh index out of range in pairs");
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->pairs, pairs, (size_t)n * 8, cudaMemcpyDeviceToDevice, s->ctx->stream));
  }
  // largest pairs first: the traversal takes root pairs in this order
  std::vector<uint32_t>& ord = x->order_host;
  ord.resize((size_t)n);
  std::vector<int64_t> size((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    uint32_t a = x->pairs_host[2 * i], b = x->pairs_host[2 * i + 1];
    size[i] = (s->t_off[a + 1] - s->t_off[a]) + (s->t_off[b + 1] - s->t_off[b]);
    ord[i] = (uint32_t)i;
  }
  std::stable_sort(ord.begin(), ord.end(), [&](uint32_t i, uint32_t j) { return size[i] > size[j]; });
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->pair_order, ord.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s->ctx->stream));
  return KDOP_OK;
}

int kdop_traverse(kdop_scene* s, int64_t n_pairs, const uint32_t* pairs, int memory, const kdop_traverse_opts* opts) {
  if (!s || n_pairs < 0 || (n_pairs > 0 && !pairs)) return KDOP_ERR_INVALID;
  if (n_pairs >= (int64_t)0x7FFFFFFF) return fail(s->ctx, KDOP_ERR_INVALID, "too many pairs");
  cudaSetDevice(s->ctx->device);
  kdop::TravParams p;
  int mode = 0;
  if (kdop_resolve_traverse_opts(s, opts, p, mode) != KDOP_OK) return fail(s->ctx, KDOP_ERR_INVALID, "bad traversal options");
  int rc = upload_pairs(s, n_pairs, pairs, memory);
  if (rc != KDOP_OK) return rc;
  KDOP_CUDA(s->ctx, kdop::launch_traverse(s, n_pairs, s->pairs, p, mode == KDOP_TRAVERSE_PLAIN));
  s->traversed = true;
  s->contacted = false;
  s->last_pairs = n_pairs;
  s->last_mode = mode;
  s->last_params = p;
  return KDOP_OK;
}

int kdop_broad_phase(kdop_scene* s, const float* positions, int memory, uint32_t* out_pairs, int64_t cap,
                     int64_t* n_pairs) {
  if (!s || !n_pairs || cap < 0 || (cap > 0 && !out_pairs)) return KDOP_ERR_INVALID;
  if (memory != KDOP_HOST && memory != KDOP_DEVICE) return fail(s->ctx, KDOP_ERR_INVALID, "bad memory kind");
  cudaSetDevice(s->ctx->device);
  cudaStream_t st = s->ctx->stream;
  kdop_scene_ext* x = ext(s);
  const int n = s->n_meshes;
  *n_pairs = 0;
  if (!x->radius_bits) {
    KDOP_CUDA(s->ctx, cudaMalloc((void**)&x->radius_bits, (size_t)std::max(n, 1) * 4));
    s->device_bytes += (int64_t)std::max(n, 1) * 4;
    KDOP_CUDA(s->ctx, kdop::launch_mesh_radius(s, x->radius_bits));
  }
  size_t need = kdop::broad_work_bytes(n);
  if (x->broad_work_bytes < need) {
    if (x->broad_work) cudaFree(x->broad_work);
    x->broad_work = nullptr;
    KDOP_CUDA(s->ctx, cudaMalloc(&x->broad_work, need));
    s->device_bytes += (int64_t)need - (int64_t)x->broad_work_bytes;
    x->broad_work_bytes = need;
  }
  const float* pos = positions;
  if (positions && memory == KDOP_HOST) {
    if (!x->broad_pos) {
      KDOP_CUDA(s->ctx, cudaMalloc((void**)&x->broad_pos, (size_t)std::max(n, 1) * 12));
      s->device_bytes += (int64_t)std::max(n, 1) * 12;
    }
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(x->broad_pos, positions, (size_t)n * 12, cudaMemcpyHostToDevice, st));
    pos = x->broad_pos;
  }
  int64_t total = 0;
  KDOP_CUDA(s->ctx, kdop::broad_phase(s, x->radius_bits, pos, x->broad_work, x->broad_pairs, x->broad_cap, &total));
  if (total > x->broad_cap) {
    if (x->broad_pairs) cudaFree(x->broad_pairs);
    x->broad_pairs = nullptr;
    int64_t c = total + total / 4 + 256;
    KDOP_CUDA(s->ctx, cudaMalloc((void**)&x->broad_pairs, (size_t)c * sizeof(uint2)));
    s->device_bytes += (c - x->broad_cap) * (int64_t)sizeof(uint2);
    x->broad_cap = c;
    KDOP_CUDA(s->ctx, kdop::broad_phase(s, x->radius_bits, pos, x->broad_work, x->broad_pairs, x->broad_cap, &total));
  }
  *n_pairs = total;
  if (total > cap) return fail(s->ctx, KDOP_ERR_CAPACITY, "broad phase: output buffer too small");
  if (total > 0)
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(out_pairs, x->broad_pairs, (size_t)total * sizeof(uint2), cudaMemcpyDefault, st));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(st));
  return KDOP_OK;
}

int kdop_traverse_shard(kdop_scene* s, int64_t n_pairs, const uint32_t* pairs, int memory,
                        const kdop_traverse_opts* opts, int rank, int n_ranks, int64_t frontier_min) {
  if (!s || n_pairs < 0 || (n_pairs > 0 && !pairs) || n_ranks < 1 || rank < 0 || rank >= n_ranks ||
      frontier_min < 1 || frontier_min > ((int64_t)1 << 26))
    return s ? fail(s->ctx, KDOP_ERR_INVALID, "bad shard arguments") : KDOP_ERR_INVALID;
  if (n_pairs >= (int64_t)0x7FFFFFFF) return fail(s->ctx, KDOP_ERR_INVALID, "too many pairs");
  cudaSetDevice(s->ctx->device);
  kdop::TravParams p;
  int mode = 0;
  if (kdop_resolve_traverse_opts(s, opts, p, mode) != KDOP_OK || mode != KDOP_TRAVERSE_BATCHED)
    return fail(s->ctx, KDOP_ERR_INVALID, "bad traversal options (shards are batched)");
  int rc = upload_pairs(s, n_pairs, pairs, memory);
  if (rc != KDOP_OK) return rc;
  int64_t ne = 0;
  kdop_scene_ext* x = ext(s);
  size_t before = x->shard_work_bytes;
  cudaError_t e = kdop::launch_traverse_shard(s, n_pairs, s->pairs, p, rank, n_ranks, frontier_min, &x->shard_work,
                                              &x->shard_work_bytes, &ne);
  s->device_bytes += (int64_t)x->shard_work_bytes - (int64_t)before;
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "kdop_traverse_shard");
  s->traversed = true;
  s->contacted = false;
  s->last_pairs = n_pairs;
  s->last_mode = mode;
  s->last_params = p;
  return KDOP_OK;
}

int kdop_get_stats(kdop_scene* s, kdop_stats* st) {
  if (!s || !st) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  const TravCtl& c = *s->ctl_host;
  std::memset(st, 0, sizeof(*st));
  st->n_pairs = s->last_pairs;
  st->n_tests = (int64_t)c.tests;
  st->n_leaf_overlaps = (int64_t)c.leaf_overlaps;
  st->n_candidates = (int64_t)c.n_cand;
  st->n_contacts = s->contacted ? (int64_t)c.n_contacts : 0;
  st->candidate_capacity = s->cand_cap;
  st->contact_capacity = s->contact_cap;
  st->queue_capacity = s->queue_cap;
  st->queue_used = (int64_t)c.q_tail;
  st->device_error = (int32_t)c.error;
  if (c.error & (kdop::DEV_ERR_TIMEOUT | kdop::DEV_ERR_QUEUE_FULL)) {
    // leave the queue clean for the next launch
    KDOP_CUDA(s->ctx, cudaMemsetAsync(s->q_tags, 0, (size_t)s->queue_cap * 4, s->ctx->stream));
    KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  }
  if (c.error & kdop::DEV_ERR_TIMEOUT) return fail(s->ctx, KDOP_ERR_TIMEOUT, "traversal wait timed out");
  if (c.error & kdop::DEV_ERR_QUEUE_FULL) return fail(s->ctx, KDOP_ERR_CAPACITY, "traversal work queue full");
  if (c.error & kdop::DEV_ERR_BAD_INDEX) return fail(s->ctx, KDOP_ERR_INVALID, "bad index on device");
  if ((int64_t)c.n_cand > s->cand_cap) return fail(s->ctx, KDOP_ERR_CAPACITY, "candidate buffer full");
  if (s->contacted && (int64_t)c.n_contacts > s->contact_cap)
    return fail(s->ctx, KDOP_ERR_CAPACITY, "contact buffer full");
  return KDOP_OK;
}

int kdop_reserve(kdop_scene* s, int64_t candidates, int64_t contacts, int64_t queue) {
  if (!s || candidates < 0 || contacts < 0 || queue < 0) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  int rc = KDOP_OK;
  if (candidates) rc = grow_candidates(s, candidates);
  if (rc == KDOP_OK && contacts) rc = grow_contacts(s, contacts);
  if (rc == KDOP_OK && queue) rc = grow_queue(s, queue);
  if (rc == KDOP_OK) KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  return rc;
}

int kdop_set_capacity(kdop_scene* s, int64_t candidates, int64_t contacts, int64_t queue) {
  if (!s || candidates < 0 || contacts < 0 || queue < 0) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  int rc = KDOP_OK;
  if (candidates || contacts || queue) drop_graph(s);
  if (candidates) {
    dfree(s, &s->cand, kdop::kCandCols * s->cand_cap);
    dfree(s, &s->records, s->cand_cap);
    s->cand_cap = 0;
    rc = grow_candidates(s, candidates);
  }
  if (rc == KDOP_OK && contacts) {
    dfree(s, &s->contacts, s->contact_cap);
    s->contact_cap = 0;
    rc = grow_contacts(s, contacts);
  }
  if (rc == KDOP_OK && queue) {
    dfree(s, &s->q_items, s->queue_cap);
    dfree(s, &s->q_tags, s->queue_cap);
    s->queue_cap = 0;
    rc = grow_queue(s, queue);
  }
  s->traversed = s->contacted = false;
  if (rc == KDOP_OK) KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  return rc;
}

int kdop_read_candidates(kdop_scene* s, uint32_t* rows, int64_t cap, int64_t* n_rows) {
  if (!s || !n_rows || (cap > 0 && !rows)) return KDOP_ERR_INVALID;
  if (!s->traversed) return fail(s->ctx, KDOP_ERR_STATE, "no traversal yet");
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  int64_t n = std::min<int64_t>((int64_t)s->ctl_host->n_cand, s->cand_cap);
  *n_rows = n;
  if (n > cap) return fail(s->ctx, KDOP_ERR_CAPACITY, "candidate read buffer too small");
  if (n == 0) return KDOP_OK;
  std::vector<uint32_t> h(3 * (size_t)n);
  for (int k = 0; k < 3; ++k)
    KDOP_CUDA(s->ctx, cudaMemcpyAsync(h.data() + k * n, s->cand + k * s->cand_cap, (size_t)n * 4,
                                      cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  const std::vector<uint32_t>& ph = ext(s)->pairs_host;
  for (int64_t i = 0; i < n; ++i) {
    uint32_t p = h[2 * n + i];
    uint32_t ma = ph[2 * p], mb = ph[2 * p + 1];
    rows[3 * i] = p;
    rows[3 * i + 1] = (uint32_t)((int64_t)h[i] - s->t_off[ma]);
    rows[3 * i + 2] = (uint32_t)((int64_t)h[n + i] - s->t_off[mb]);
  }
  return KDOP_OK;
}

int kdop_sort_results(kdop_scene* s) {
  if (!s) return KDOP_ERR_INVALID;
  if (!s->traversed) return fail(s->ctx, KDOP_ERR_STATE, "kdop_sort_results before kdop_traverse");
  kdop_stats st;
  int rc = kdop_get_stats(s, &st);  // synchronises; reports overflow and device errors
  if (rc != KDOP_OK) return rc;
  int64_t n = std::min<int64_t>(st.n_candidates, s->cand_cap);
  int64_t nc = s->contacted ? std::min<int64_t>(st.n_contacts, s->contact_cap) : 0;
  if (n <= 0) return KDOP_OK;
  kdop_scene_ext* x = ext(s);
  size_t need = kdop::sort_results_bytes(n, nc);
  if (x->sort_work_bytes < need) {
    if (x->sort_work) {
      cudaFree(x->sort_work);
      s->device_bytes -= (int64_t)x->sort_work_bytes;
    }
    x->sort_work = nullptr;
    x->sort_work_bytes = 0;
    KDOP_CUDA(s->ctx, cudaMalloc(&x->sort_work, need));
    x->sort_work_bytes = need;
    s->device_bytes += (int64_t)need;
  }
  KDOP_CUDA(s->ctx, kdop::sort_results(s, n, nc, x->sort_work, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  return KDOP_OK;
}

int kdop_contacts(kdop_scene* s) {
  if (!s) return KDOP_ERR_INVALID;
  if (!s->traversed) return fail(s->ctx, KDOP_ERR_STATE, "kdop_contacts before kdop_traverse");
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, ensure_posed(s));
  KDOP_CUDA(s->ctx, kdop::launch_contacts(s));
  s->contacted = true;
  return KDOP_OK;
}

int kdop_read_contacts(kdop_scene* s, kdop_contact* rows, int64_t cap, int64_t* n_rows) {
  if (!s || !n_rows || (cap > 0 && !rows)) return KDOP_ERR_INVALID;
  if (!s->contacted) return fail(s->ctx, KDOP_ERR_STATE, "no contacts yet");
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  int64_t n = std::min<int64_t>((int64_t)s->ctl_host->n_contacts, s->contact_cap);
  *n_rows = n;
  if (n > cap) return fail(s->ctx, KDOP_ERR_CAPACITY, "contact read buffer too small");
  if (n == 0) return KDOP_OK;
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(rows, s->contacts, (size_t)n * sizeof(kdop_contact), cudaMemcpyDefault,
                                    s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  return KDOP_OK;
}

// ---- contact reduction (prox_collision_detection.h:341-350) ----
static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// The context's grow-only scratch, at least `bytes` long.  Calls on a context
// are serial, so one buffer serves every reduction; growing frees the old
// buffer (cudaFree waits for the work that used it).
static cudaError_t ctx_scratch(kdop_ctx* ctx, size_t bytes, char** p) {
  if (bytes > ctx->scratch_bytes) {
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    cudaError_t e = cudaMalloc((void**)&ctx->scratch, bytes);
    if (e != cudaSuccess) return e;
    ctx->scratch_bytes = bytes;
  }
  *p = ctx->scratch;
  return cudaSuccess;
}

// Bytes reduce_rows needs for n rows: the sort's work, then the kept rows and
// their bodies.
static size_t reduce_rows_bytes(int64_t n) {
  const size_t m = (size_t)std::max<int64_t>(n, 1);
  return align256(kdop::reduce_work_bytes(n)) + align256(m * sizeof(kdop_contact)) + align256(m * sizeof(uint2));
}

// Reduces n device rows with their device bodies in `buf` (reduce_rows_bytes(n)
// bytes), then copies the kept rows (and bodies) to the caller's buffers
// (host or device).
static int reduce_rows(kdop_ctx* ctx, const kdop_contact* rows, const uint2* bodies, int64_t n, char* buf,
                       kdop_contact* out, uint32_t* out_bodies, int64_t cap, int64_t* n_out) {
  const size_t m = (size_t)std::max<int64_t>(n, 1);
  const size_t wb = align256(kdop::reduce_work_bytes(n));
  const size_t rb = align256(m * sizeof(kdop_contact));
  kdop_contact* kept_rows = reinterpret_cast<kdop_contact*>(buf + wb);
  uint2* kept_bodies = reinterpret_cast<uint2*>(buf + wb + rb);
  int64_t kept = 0;
  cudaError_t e = kdop::reduce_contact_rows(ctx, rows, bodies, n, buf, kept_rows, kept_bodies, &kept);
  *n_out = kept;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "reduce_contact_rows");
  if (kept > cap) return fail(ctx, KDOP_ERR_CAPACITY, "reduced contact buffer too small");
  if (kept > 0) {
    e = cudaMemcpyAsync(out, kept_rows, (size_t)kept * sizeof(kdop_contact), cudaMemcpyDefault, ctx->stream);
    if (e == cudaSuccess && out_bodies)
      e = cudaMemcpyAsync(out_bodies, kept_bodies, (size_t)kept * sizeof(uint2), cudaMemcpyDefault, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "reduced contacts copy");
  }
  return KDOP_OK;
}

int kdop_reduce_contact_rows(kdop_ctx* ctx, const kdop_contact* rows, const uint32_t* bodies, int64_t n,
                             kdop_contact* out, uint32_t* out_bodies, int64_t cap, int64_t* n_out) {
  if (!ctx || !n_out || n < 0 || (n > 0 && (!rows || !bodies)) || (cap > 0 && !out)) return KDOP_ERR_INVALID;
  if (n >= ((int64_t)1 << 32) - 1) return fail(ctx, KDOP_ERR_INVALID, "too many contact rows");
  *n_out = 0;
  if (n == 0) return KDOP_OK;
  cudaSetDevice(ctx->device);
  // staged input (rows, bodies), then the reduction's own scratch
  const size_t rb = align256((size_t)n * sizeof(kdop_contact));
  const size_t bb = align256((size_t)n * sizeof(uint2));
  char* in = nullptr;
  KDOP_CUDA(ctx, ctx_scratch(ctx, rb + bb + reduce_rows_bytes(n), &in));
  cudaError_t e = cudaMemcpyAsync(in, rows, (size_t)n * sizeof(kdop_contact), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(in + rb, bodies, (size_t)n * sizeof(uint2), cudaMemcpyDefault, ctx->stream);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(ctx->stream);  // a started copy may still read the caller's rows
    return cuda_fail(ctx, e, "reduce input copy");
  }
  return reduce_rows(ctx, reinterpret_cast<kdop_contact*>(in), reinterpret_cast<uint2*>(in + rb), n, in + rb + bb,
                     out, out_bodies, cap, n_out);
}

int kdop_reduce_contacts(kdop_scene* s, kdop_contact* out, uint32_t* out_bodies, int64_t cap, int64_t* n_out) {
  if (!s || !n_out || (cap > 0 && !out)) return KDOP_ERR_INVALID;
  if (!s->contacted) return fail(s->ctx, KDOP_ERR_STATE, "kdop_reduce_contacts before kdop_contacts");
  kdop_stats st;
  int rc = kdop_get_stats(s, &st);  // synchronises; reports overflow and device errors
  if (rc != KDOP_OK) return rc;
  const int64_t n = std::min<int64_t>(st.n_contacts, s->contact_cap);
  *n_out = 0;
  if (n <= 0) return KDOP_OK;
  // the rows' bodies, then the reduction's own scratch
  const size_t bb = align256((size_t)n * sizeof(uint2));
  char* buf = nullptr;
  KDOP_CUDA(s->ctx, ctx_scratch(s->ctx, bb + reduce_rows_bytes(n), &buf));
  uint2* bodies = reinterpret_cast<uint2*>(buf);
  cudaError_t e = kdop::scene_contact_bodies(s, n, bodies);
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "scene_contact_bodies");
  return reduce_rows(s->ctx, s->contacts, bodies, n, buf + bb, out, out_bodies, cap, n_out);
}

int kdop_contacts_adjoint(kdop_scene* s, const float* dd, const float* dn, float* grad, int memory) {
  if (!s || !dd || !grad) return KDOP_ERR_INVALID;
  if (!s->contacted) return fail(s->ctx, KDOP_ERR_STATE, "adjoint before kdop_contacts");
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, ensure_posed(s));
  if (memory == KDOP_DEVICE) {
    KDOP_CUDA(s->ctx, kdop::launch_adjoint(s, dd, dn, grad));
    return KDOP_OK;
  }
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  int64_t nc = std::min<int64_t>((int64_t)s->ctl_host->n_contacts, s->contact_cap);
  int64_t need = std::max<int64_t>(nc, 1) * 4 + 3 * s->nv;
  cudaError_t e;
  float* d = stage(s, need, &e);
  if (!d) return cuda_fail(s->ctx, e, "staging alloc");
  float* d_dd = d;
  float* d_dn = d + std::max<int64_t>(nc, 1);
  float* d_g = d + 4 * std::max<int64_t>(nc, 1);
  if (nc) KDOP_CUDA(s->ctx, cudaMemcpyAsync(d_dd, dd, (size_t)nc * 4, cudaMemcpyHostToDevice, s->ctx->stream));
  if (nc && dn) KDOP_CUDA(s->ctx, cudaMemcpyAsync(d_dn, dn, (size_t)nc * 12, cudaMemcpyHostToDevice, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(d_g, grad, (size_t)s->nv * 12, cudaMemcpyHostToDevice, s->ctx->stream));
  KDOP_CUDA(s->ctx, kdop::launch_adjoint(s, d_dd, dn ? d_dn : nullptr, d_g));
  KDOP_CUDA(s->ctx, cudaMemcpyAsync(grad, d_g, (size_t)s->nv * 12, cudaMemcpyDeviceToHost, s->ctx->stream));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  return KDOP_OK;
}

int kdop_graph_release(kdop_scene* s) {
  if (!s) return KDOP_ERR_INVALID;
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->graph_exec = nullptr;
  s->graph = nullptr;
  ext(s)->graph_kernels = 0;
  return KDOP_OK;
}

int kdop_graph_capture(kdop_scene* s, int refit_mode, int64_t n_pairs, const uint32_t* pairs, int memory,
                       const kdop_traverse_opts* opts, int flags) {
  if (!s || n_pairs < 0 || (n_pairs > 0 && !pairs)) return KDOP_ERR_INVALID;
  if (refit_mode < KDOP_REFIT_VERTICES || refit_mode > KDOP_REFIT_DEFORM) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  kdop::TravParams p;
  int mode = 0;
  if (kdop_resolve_traverse_opts(s, opts, p, mode) != KDOP_OK) return fail(s->ctx, KDOP_ERR_INVALID, "bad traversal options");
  kdop_graph_release(s);
  int rc = upload_pairs(s, n_pairs, pairs, memory);
  if (rc != KDOP_OK) return rc;
  // settle function attributes outside the capture
  KDOP_CUDA(s->ctx, kdop::traverse_prepare(s->K, kdop::traverse_smem_bytes(p.block_warps, p.stack_cap)));
  KDOP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  long long before = s->ctx->launches;
  // the captured contact kernels take their vertex source from the refit
  // mode: the graph's, not the one of the last direct refit
  const int old_refit_mode = s->refit_mode;
  s->refit_mode = refit_mode;
  cudaError_t eb = cudaStreamBeginCapture(s->ctx->stream, cudaStreamCaptureModeRelaxed);
  if (eb != cudaSuccess) {
    s->refit_mode = old_refit_mode;
    return cuda_fail(s->ctx, eb, "cudaStreamBeginCapture");
  }
  cudaError_t e = cudaSuccess;
  if (flags & 1) e = kdop::launch_motion(s);
  if (e == cudaSuccess) e = kdop::launch_refit(s, refit_mode);
  if (e == cudaSuccess) e = kdop::launch_traverse(s, n_pairs, s->pairs, p, mode == KDOP_TRAVERSE_PLAIN);
  if (e == cudaSuccess) e = kdop::launch_contacts(s);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s->ctx->stream, &g);
  s->ctx->launches = before;
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    s->refit_mode = old_refit_mode;
    return cuda_fail(s->ctx, e != cudaSuccess ? e : e2, "graph capture");
  }
  s->graph = g;
  e = cudaGraphInstantiate(&s->graph_exec, g, 0);
  if (e != cudaSuccess) {
    kdop_graph_release(s);
    s->refit_mode = old_refit_mode;
    return cuda_fail(s->ctx, e, "cudaGraphInstantiate");
  }
  size_t n_nodes = 0;
  cudaGraphGetNodes(g, nullptr, &n_nodes);
  ext(s)->graph_kernels = (int64_t)n_nodes;
  ext(s)->graph_refit_mode = refit_mode;
  s->refit_mode = refit_mode;
  // capturing runs nothing: the posed array holds no step of this graph yet
  s->posed_valid = false;
  s->traversed = true;
  s->contacted = true;
  s->last_pairs = n_pairs;
  s->last_mode = mode;
  s->last_params = p;
  return KDOP_OK;
}

int kdop_graph_launch(kdop_scene* s) {
  if (!s) return KDOP_ERR_INVALID;
  if (!s->graph_exec) return fail(s->ctx, KDOP_ERR_STATE, "no captured graph");
  cudaSetDevice(s->ctx->device);
  KDOP_CUDA(s->ctx, cudaGraphLaunch(s->graph_exec, s->ctx->stream));
  s->ctx->launches += ext(s)->graph_kernels;
  // the step just enqueued refits in the graph's mode: the contacts, the
  // adjoint and read-backs follow it, whatever direct refit ran in between
  s->refit_mode = ext(s)->graph_refit_mode;
  if (s->refit_mode != KDOP_REFIT_VERTICES) s->posed_valid = true;
  return KDOP_OK;
}

// Times one traversal configuration: a checked warm-up run (growing the
// buffers if needed), then `repeats` runs timed one by one; returns the
// median milliseconds per run, or a negative value when the configuration
// cannot run.
static float time_config(kdop_scene* s, int64_t n_pairs, const kdop::TravParams& p, int repeats,
                         std::vector<cudaEvent_t>& ev) {
  if (kdop::traverse_smem_bytes(p.block_warps, p.stack_cap) > s->ctx->smem_optin) return -1.f;
  if (kdop::launch_traverse(s, n_pairs, s->pairs, p, 0) != cudaSuccess) return -1.f;
  kdop_stats st;
  int r = kdop_get_stats(s, &st);
  if (r == KDOP_ERR_CAPACITY) {
    int64_t nc = std::max<int64_t>(st.n_candidates + st.n_candidates / 4, s->cand_cap);
    int64_t nq = (st.device_error & kdop::DEV_ERR_QUEUE_FULL) ? std::max<int64_t>(2 * s->queue_cap, 2 * st.queue_used) : 0;
    if (kdop_reserve(s, nc, 0, nq) != KDOP_OK) return -1.f;
    if (kdop::launch_traverse(s, n_pairs, s->pairs, p, 0) != cudaSuccess) return -1.f;
    r = kdop_get_stats(s, &st);
  }
  if (r != KDOP_OK) return -1.f;
  cudaEventRecord(ev[0], s->ctx->stream);
  for (int k = 0; k < repeats; ++k) {
    kdop::launch_traverse(s, n_pairs, s->pairs, p, 0);
    cudaEventRecord(ev[k + 1], s->ctx->stream);
  }
  if (cudaEventSynchronize(ev[repeats]) != cudaSuccess) return -1.f;
  std::vector<float> ms((size_t)repeats);
  for (int k = 0; k < repeats; ++k) cudaEventElapsedTime(&ms[(size_t)k], ev[k], ev[k + 1]);
  if (kdop_get_stats(s, &st) != KDOP_OK) return -1.f;
  std::nth_element(ms.begin(), ms.begin() + repeats / 2, ms.end());
  return ms[(size_t)repeats / 2];
}

int kdop_autotune(kdop_scene* s, int64_t n_pairs, const uint32_t* pairs, int memory, int repeats,
                  kdop_traverse_opts* best) {
  if (!s || n_pairs < 0 || (n_pairs > 0 && !pairs)) return KDOP_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  // at least five timed runs per configuration, odd so the median is a run
  repeats = std::max(repeats, 5) | 1;
  int rc = upload_pairs(s, n_pairs, pairs, memory);
  if (rc != KDOP_OK) return rc;
  std::vector<cudaEvent_t> ev((size_t)repeats + 1, nullptr);
  for (auto& e : ev) {
    cudaError_t ce = cudaEventCreate(&e);
    if (ce != cudaSuccess) {
      for (auto& f : ev)
        if (f) cudaEventDestroy(f);
      return cuda_fail(s->ctx, ce, "cudaEventCreate");
    }
  }
  // Coordinate descent from the defaults, two sweeps over the knobs.  A
  // challenger replaces the incumbent only when its median is more than 2 %
  // faster, so that run-to-run noise does not flip the choice.
  const float kGain = 0.98f;
  kdop_traverse_opts d;
  kdop_traverse_opts_default(nullptr, &d);
  kdop::TravParams cur;
  int mode = 0;
  kdop_resolve_traverse_opts(s, &d, cur, mode);
  float best_ms = time_config(s, n_pairs, cur, repeats, ev);
  if (best_ms < 0.f) best_ms = 1e30f;
  const std::vector<int> warps = {4, 8, 16}, caps = {128, 256, 512, 1024}, groups = {1, 2, 4, 8},
                         donate = {32, 64, 128, 256}, waves = {0, 16, 64, 128}, carve = {0, 25, 50, 100},
                         chunk = {1, 4};
  for (int sweep = 0; sweep < 2; ++sweep) {
    for (int knob = 0; knob < 7; ++knob) {
      const std::vector<int>& vals = knob == 0 ? warps : knob == 1 ? caps : knob == 2 ? groups
                                   : knob == 3 ? donate : knob == 4 ? waves : knob == 5 ? carve : chunk;
      for (int v : vals) {
        kdop::TravParams p = cur;
        int* f = knob == 0 ? &p.block_warps : knob == 1 ? &p.stack_cap : knob == 2 ? &p.load_group
               : knob == 3 ? &p.donate_min : knob == 4 ? &p.wave_pairs : knob == 5 ? &p.smem_carveout
               : &p.init_chunk;
        if (*f == v) continue;
        *f = v;
        float ms = time_config(s, n_pairs, p, repeats, ev);
        if (ms >= 0.f && ms < kGain * best_ms) {
          best_ms = ms;
          cur = p;
        }
      }
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (best_ms >= 1e30f) return fail(s->ctx, KDOP_ERR_CUDA, "autotune: no configuration ran");
  kdop_traverse_opts bo = d;
  bo.block_warps = cur.block_warps;
  bo.stack_cap = cur.stack_cap;
  bo.init_chunk = cur.init_chunk;
  bo.donate_min = cur.donate_min;
  bo.load_group = cur.load_group;
  bo.wave_pairs = cur.wave_pairs;
  bo.smem_carveout = cur.smem_carveout;
  kdop_scene_ext* x = ext(s);
  x->tuned = bo;
  x->has_tuned = true;
  s->ctx->tuned[std::make_pair(s->K, tune_size_class(s))] = bo;
  if (best) *best = bo;
  return KDOP_OK;
}

}  // extern "C"
