// kdop_cuda_tag.hpp -- drop-in C++ back-end for the reference's kDOP entry
// points, over the C ABI of kdop_cuda.h.
//
// Include it after the reference's kdop headers (kdop_tree.h,
// kdop_test_pair.h, kdop_refit_tree.h, kdop_tandem_traversal.h) and link
// libkdop_cuda.so.  It adds a tag next to kdop::sequential / kdop::dikucl
// (SIMULATION/KDOP/KDOP/include/kdop_tags.h:13-18) and the two overloads the
// narrow phase calls:
//
//   kdop::tandem_traversal(std::vector<TestPair<V,K,T> >&, kdop::cuda const&)
//       replaces kdop_tandem_traversal.h:198-226 (and the OpenCL overload of
//       cl/kdop_cl_tandem_traversal.h:623): every pair's contacts go to its
//       TestPair::m_callback, per pair in the order of its candidate tet pairs
//       sorted by (tet of A, tet of B) on the device (kdop_sort_results),
//       each candidate's contacts in the reference's generation order (the
//       OpenCL path sorted too, kdop_cl_tandem_traversal.h:1773-1788).
//   kdop::refit_tree(Tree<T,K>&, T4Mesh const&, X, Y, Z, kdop::cuda const&)
//       replaces kdop_refit_tree.h:120-162 for every tree make_tree builds:
//       one-chunk trees (mem_bytes = SIZE_MAX, the gProximity set-up) get
//       every node volume from the GPU refit; chunked trees (the narrow
//       phase's default, narrow_object.h:113-128: 8000-byte chunks) get the
//       leaf kDOPs from the GPU and their chunk, super-chunk and root volumes
//       as exact unions of those (min / max per slab), written into every
//       SubTree and tree.m_root as kdop_refit_tree.h:131-161 does.
//
// Device state persists between calls: the meshes of a call are uploaded
// once into a scene cached on the context, keyed by the identity of the
// caller's objects (mesh, X, Y, Z and surface map addresses) and their sizes,
// so the calls of later simulation steps only upload the current positions,
// refit and traverse.  A caller that changes a mesh's topology in place
// (same objects, same counts) or that is about to destroy the context calls
// kdop::cuda_release(ctx) first; up to 16 scenes are kept per context (least
// recently used dropped first).  Volumes and contacts are the reference's bit
// for bit when T = float (the GPU computes in float).
//
// Errors come back as std::runtime_error carrying kdop_last_error().
#ifndef KDOP_CUDA_TAG_HPP
#define KDOP_CUDA_TAG_HPP

#include <algorithm>
#include <cstring>
#include <list>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kdop_cuda.h"

namespace kdop {

// Back-end tag: the CUDA context to run on (created by the caller with
// kdop_ctx_create and kept for the lifetime of the simulation).
struct cuda {
  kdop_ctx* ctx;
  explicit cuda(kdop_ctx* c) : ctx(c) {}
};

namespace cuda_detail {

inline void check(kdop_ctx* ctx, int rc, const char* what) {
  if (rc != KDOP_OK)
    throw std::runtime_error(std::string("kdop ") + what + ": " + kdop_status_string(rc) + " " +
                             kdop_last_error(ctx));
}

typedef mesh_array::TetrahedronAttribute<mesh_array::TetrahedronSurfaceInfo, mesh_array::T4Mesh> SurfaceMap;

// Identity of one caller mesh: its objects and sizes.
struct MeshKey {
  const void* mesh;
  const void* x;
  const void* y;
  const void* z;
  const void* surf;
  int64_t n_verts;
  int64_t n_tets;
  bool operator==(MeshKey const& o) const {
    return mesh == o.mesh && x == o.x && y == o.y && z == o.z && surf == o.surf && n_verts == o.n_verts &&
           n_tets == o.n_tets;
  }
};

// Host copy of one reference mesh's topology in the C ABI's layout.
struct MeshCopy {
  std::vector<float> xyz;
  std::vector<uint32_t> tets;
  std::vector<uint8_t> surf;
  std::vector<uint32_t> order;  // 0..n_tets-1: the tree of make_tree over the mesh as given
};

template <typename T>
void gather_positions(mesh_array::T4Mesh const& mesh, mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& X,
                      mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Y,
                      mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Z, float* out) {
  size_t nv = mesh.vertex_size();
  for (size_t i = 0; i < nv; ++i) {
    mesh_array::Vertex const& v = mesh.vertex(i);
    out[3 * i] = (float)X(v);
    out[3 * i + 1] = (float)Y(v);
    out[3 * i + 2] = (float)Z(v);
  }
}

template <typename T>
MeshCopy copy_mesh(mesh_array::T4Mesh const& mesh, mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& X,
                   mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Y,
                   mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Z, SurfaceMap const* S) {
  MeshCopy c;
  size_t nv = mesh.vertex_size(), nt = mesh.tetrahedron_size();
  c.xyz.resize(3 * nv);
  gather_positions<T>(mesh, X, Y, Z, c.xyz.data());
  c.tets.resize(4 * nt);
  c.surf.assign(nt, 0);
  c.order.resize(nt);
  for (size_t t = 0; t < nt; ++t) c.order[t] = (uint32_t)t;
  for (size_t t = 0; t < nt; ++t) {
    mesh_array::Tetrahedron const& tet = mesh.tetrahedron(t);
    c.tets[4 * t] = (uint32_t)tet.i();
    c.tets[4 * t + 1] = (uint32_t)tet.j();
    c.tets[4 * t + 2] = (uint32_t)tet.k();
    c.tets[4 * t + 3] = (uint32_t)tet.m();
    if (S) {
      mesh_array::TetrahedronSurfaceInfo const& s = (*S)(tet);
      c.surf[t] = (uint8_t)((s.m_i ? 1 : 0) | (s.m_j ? 2 : 0) | (s.m_k ? 4 : 0) | (s.m_m ? 8 : 0));
    }
  }
  return c;
}

// A scene on the device holding a fixed list of caller meshes.
struct CachedScene {
  int K = 0;
  std::vector<MeshKey> keys;
  kdop_scene* scene = nullptr;
  std::vector<int64_t> v_off;  // first vertex of each mesh in the concatenated positions
  std::vector<float> xyz;      // staging of the current positions, all meshes
  uint64_t used = 0;
};

struct ContextCache {
  std::list<CachedScene> scenes;
  uint64_t clock = 0;
};

const size_t kMaxCachedScenes = 16;

inline std::mutex& cache_mutex() {
  static std::mutex m;
  return m;
}
inline std::map<kdop_ctx*, ContextCache>& caches() {
  static std::map<kdop_ctx*, ContextCache> c;
  return c;
}

// The cached scene of (K, keys), created from make() on a miss.  Caller holds
// cache_mutex().
template <typename Make>
CachedScene& scene_for(kdop_ctx* ctx, int K, std::vector<MeshKey> const& keys, Make make) {
  ContextCache& cc = caches()[ctx];
  for (std::list<CachedScene>::iterator it = cc.scenes.begin(); it != cc.scenes.end(); ++it) {
    if (it->K == K && it->keys == keys) {
      it->used = ++cc.clock;
      return *it;
    }
  }
  std::vector<MeshCopy> meshes = make();
  std::vector<kdop_mesh_desc> desc(meshes.size());
  CachedScene cs;
  cs.K = K;
  cs.keys = keys;
  cs.v_off.assign(meshes.size() + 1, 0);
  for (size_t m = 0; m < meshes.size(); ++m) {
    desc[m].n_verts = (int64_t)meshes[m].xyz.size() / 3;
    desc[m].xyz = meshes[m].xyz.data();
    desc[m].n_tets = (int64_t)meshes[m].tets.size() / 4;
    desc[m].tets = meshes[m].tets.data();
    desc[m].surface = meshes[m].surf.data();
    desc[m].leaf_order = meshes[m].order.data();
    cs.v_off[m + 1] = cs.v_off[m] + desc[m].n_verts;
  }
  cs.xyz.resize((size_t)std::max<int64_t>(cs.v_off.back(), 1) * 3);
  check(ctx, kdop_scene_create(ctx, K, (int)desc.size(), desc.data(), &cs.scene), "scene_create");
  if (cc.scenes.size() >= kMaxCachedScenes) {
    std::list<CachedScene>::iterator old = cc.scenes.begin();
    for (std::list<CachedScene>::iterator it = cc.scenes.begin(); it != cc.scenes.end(); ++it)
      if (it->used < old->used) old = it;
    kdop_scene_destroy(old->scene);
    cc.scenes.erase(old);
  }
  cs.used = ++cc.clock;
  cc.scenes.push_back(cs);
  return cc.scenes.back();
}

template <typename T, size_t K>
void set_volume(geometry::DOP<T, K>& d, float const* v) {
  for (size_t s = 0; s < K / 2; ++s) {
    d(s).lower() = (T)v[2 * s];
    d(s).upper() = (T)v[2 * s + 1];
  }
}

// One-chunk tree: every node volume straight from the GPU refit's preorder.
template <typename T, size_t K>
void write_preorder(kdop::SubTree<T, K>& st, size_t idx, float const* vol, size_t& k) {
  kdop::Node<T, K>& n = st.m_nodes[idx];
  set_volume<T, K>(n.m_volume, vol + k * K);
  ++k;
  if (n.is_leaf()) return;
  write_preorder<T, K>(st, n.m_start, vol, k);
  write_preorder<T, K>(st, n.m_end, vol, k);
}

// Chunked tree: the subtree of a branch or super chunk below node idx, leaves
// from `leaf(index)`, internal nodes the union of their children (exact, so
// equal to the reference's bottom-up sweep of kdop_refit_tree.h:24-115).
template <typename T, size_t K, typename Leaf>
void fill_subtree(kdop::SubTree<T, K>& st, size_t idx, Leaf const& leaf) {
  kdop::Node<T, K>& n = st.m_nodes[idx];
  if (n.is_leaf()) {
    leaf(n.m_start, n.m_volume);
    return;
  }
  fill_subtree<T, K, Leaf>(st, n.m_start, leaf);
  fill_subtree<T, K, Leaf>(st, n.m_end, leaf);
  n.m_volume = geometry::make_union(st.m_nodes[n.m_start].m_volume, st.m_nodes[n.m_end].m_volume);
}

}  // namespace cuda_detail

// Drops the device scenes the tag keeps for this context (call before
// kdop_ctx_destroy, or after changing a mesh's topology in place).
inline void cuda_release(kdop_ctx* ctx) {
  std::lock_guard<std::mutex> lock(cuda_detail::cache_mutex());
  std::map<kdop_ctx*, cuda_detail::ContextCache>::iterator it = cuda_detail::caches().find(ctx);
  if (it == cuda_detail::caches().end()) return;
  for (std::list<cuda_detail::CachedScene>::iterator s = it->second.scenes.begin(); s != it->second.scenes.end(); ++s)
    kdop_scene_destroy(s->scene);
  cuda_detail::caches().erase(it);
}

// refit_tree on the GPU (all trees make_tree builds, see the file comment).
template <typename V, size_t K, typename T>
inline void refit_tree(Tree<T, K>& tree, mesh_array::T4Mesh const& mesh,
                       mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& X,
                       mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Y,
                       mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Z, cuda const& tag) {
  const int64_t nt = (int64_t)mesh.tetrahedron_size();
  if (nt == 0 || tree.number_of_levels() == 0) return;
  const int64_t nn = 2 * nt - 1;
  std::vector<float> vol((size_t)nn * K);
  std::vector<int64_t> tet((size_t)nn);
  {
    std::lock_guard<std::mutex> lock(cuda_detail::cache_mutex());
    cuda_detail::MeshKey key = {&mesh, &X, &Y, &Z, 0, (int64_t)mesh.vertex_size(), nt};
    cuda_detail::CachedScene& cs = cuda_detail::scene_for(tag.ctx, (int)K, std::vector<cuda_detail::MeshKey>(1, key),
                                                          [&]() {
      return std::vector<cuda_detail::MeshCopy>(1, cuda_detail::copy_mesh<T>(mesh, X, Y, Z, 0));
    });
    cuda_detail::gather_positions<T>(mesh, X, Y, Z, cs.xyz.data());
    int64_t got = 0;
    int rc = kdop_set_vertices(cs.scene, cs.xyz.data(), cs.v_off.back(), KDOP_HOST);
    if (rc == KDOP_OK) rc = kdop_refit(cs.scene, KDOP_REFIT_VERTICES);
    if (rc == KDOP_OK) rc = kdop_read_tree(cs.scene, 0, nn, vol.data(), tet.data(), &got);
    cuda_detail::check(tag.ctx, rc, "refit_tree");
  }
  if (tree.number_of_levels() == 1 && tree.branches().size() == 1) {
    // one chunk: the GPU tree has the same topology, node for node
    size_t k = 0;
    cuda_detail::write_preorder<T, K>(tree.branches()[0], 0, vol.data(), k);
    tree.m_root = tree.branches()[0].m_nodes[0].m_volume;
    return;
  }
  // chunked: leaf kDOPs by tet, then branches, super chunks and the root
  std::vector<int64_t> leaf_row((size_t)nt, -1);
  for (int64_t k = 0; k < nn; ++k)
    if (tet[(size_t)k] >= 0 && tet[(size_t)k] < nt) leaf_row[(size_t)tet[(size_t)k]] = k;
  const float* vp = vol.data();
  std::vector<SubTree<T, K> >& branches = tree.branches();
  for (size_t c = 0; c < branches.size(); ++c) {
    cuda_detail::fill_subtree<T, K>(branches[c], 0, [&](size_t t, geometry::DOP<T, K>& d) {
      if (t >= (size_t)nt || leaf_row[t] < 0) throw std::runtime_error("kdop::cuda refit_tree: leaf tet out of range");
      cuda_detail::set_volume<T, K>(d, vp + (size_t)leaf_row[t] * K);
    });
  }
  for (size_t h = tree.number_of_levels() - 1; h >= 1; --h) {
    std::vector<SubTree<T, K> >& below = tree.super_chunks(h);
    std::vector<SubTree<T, K> >& level = tree.super_chunks(h - 1);
    for (size_t c = 0; c < level.size(); ++c) {
      cuda_detail::fill_subtree<T, K>(level[c], 0, [&](size_t i, geometry::DOP<T, K>& d) {
        if (i >= below.size()) throw std::runtime_error("kdop::cuda refit_tree: chunk index out of range");
        d = below[i].m_nodes[0].m_volume;
      });
    }
  }
  std::vector<SubTree<T, K> >& top = tree.super_chunks(0);
  tree.m_root = top[0].m_nodes[0].m_volume;
  for (size_t c = 1; c < top.size(); ++c) tree.m_root = geometry::make_union(tree.m_root, top[c].m_nodes[0].m_volume);
}

// tandem_traversal of a pool of test pairs on the GPU.
template <typename V, size_t K, typename T>
inline void tandem_traversal(std::vector<TestPair<V, K, T> >& work_pool, cuda const& tag) {
  if (work_pool.empty()) return;
  typedef TestPair<V, K, T> P;
  // distinct meshes of the pool, by the identity of the caller's objects
  std::vector<cuda_detail::MeshKey> keys;
  std::vector<std::pair<const P*, int> > source;  // (pair, side) that first named each mesh
  std::vector<uint32_t> pairs;
  for (size_t i = 0; i < work_pool.size(); ++i) {
    P const& p = work_pool[i];
    for (int s = 0; s < 2; ++s) {
      cuda_detail::MeshKey k = s == 0 ? cuda_detail::MeshKey{p.m_mesh_a, p.m_x_a, p.m_y_a, p.m_z_a, p.m_surface_map_a,
                                                              (int64_t)p.m_mesh_a->vertex_size(),
                                                              (int64_t)p.m_mesh_a->tetrahedron_size()}
                                      : cuda_detail::MeshKey{p.m_mesh_b, p.m_x_b, p.m_y_b, p.m_z_b, p.m_surface_map_b,
                                                              (int64_t)p.m_mesh_b->vertex_size(),
                                                              (int64_t)p.m_mesh_b->tetrahedron_size()};
      size_t id = 0;
      while (id < keys.size() && !(keys[id] == k)) ++id;
      if (id == keys.size()) {
        keys.push_back(k);
        source.push_back(std::make_pair(&p, s));
      }
      pairs.push_back((uint32_t)id);
    }
  }
  std::vector<uint32_t> cand;
  std::vector<kdop_contact> rows;
  int64_t nc = 0, nr = 0;
  {
    std::lock_guard<std::mutex> lock(cuda_detail::cache_mutex());
    cuda_detail::CachedScene& cs = cuda_detail::scene_for(tag.ctx, (int)K, keys, [&]() {
      std::vector<cuda_detail::MeshCopy> m;
      for (size_t i = 0; i < source.size(); ++i) {
        P const& p = *source[i].first;
        m.push_back(source[i].second == 0
                        ? cuda_detail::copy_mesh<T>(*p.m_mesh_a, *p.m_x_a, *p.m_y_a, *p.m_z_a, p.m_surface_map_a)
                        : cuda_detail::copy_mesh<T>(*p.m_mesh_b, *p.m_x_b, *p.m_y_b, *p.m_z_b, p.m_surface_map_b));
      }
      return m;
    });
    // this step's positions of every mesh, then refit, traversal, contacts
    for (size_t i = 0; i < source.size(); ++i) {
      P const& p = *source[i].first;
      float* out = cs.xyz.data() + 3 * cs.v_off[i];
      if (source[i].second == 0)
        cuda_detail::gather_positions<T>(*p.m_mesh_a, *p.m_x_a, *p.m_y_a, *p.m_z_a, out);
      else
        cuda_detail::gather_positions<T>(*p.m_mesh_b, *p.m_x_b, *p.m_y_b, *p.m_z_b, out);
    }
    kdop_scene* sc = cs.scene;
    int64_t np = (int64_t)work_pool.size();
    int rc = kdop_set_vertices(sc, cs.xyz.data(), cs.v_off.back(), KDOP_HOST);
    if (rc == KDOP_OK) rc = kdop_refit(sc, KDOP_REFIT_VERTICES);
    kdop_stats st;
    std::memset(&st, 0, sizeof(st));
    for (int attempt = 0; attempt < 8 && rc == KDOP_OK; ++attempt) {
      rc = kdop_traverse(sc, np, pairs.data(), KDOP_HOST, 0);
      if (rc == KDOP_OK) rc = kdop_contacts(sc);
      if (rc == KDOP_OK) rc = kdop_get_stats(sc, &st);
      if (rc != KDOP_ERR_CAPACITY) break;
      rc = kdop_reserve(sc, st.n_candidates + st.n_candidates / 4 + 1024, st.n_contacts + st.n_contacts / 4 + 1024,
                        (st.device_error & 2) ? 2 * st.queue_capacity : 0);
      if (rc != KDOP_OK) break;
    }
    if (rc == KDOP_OK) rc = kdop_sort_results(sc);  // candidates by (pair, tet A, tet B), contacts to match
    cand.resize((size_t)st.n_candidates * 3 + 3);
    rows.resize((size_t)st.n_contacts + 1);
    if (rc == KDOP_OK) rc = kdop_read_candidates(sc, cand.data(), st.n_candidates, &nc);
    if (rc == KDOP_OK) rc = kdop_read_contacts(sc, rows.data(), st.n_contacts, &nr);
    cuda_detail::check(tag.ctx, rc, "tandem_traversal");
  }
  for (int64_t r = 0; r < nr; ++r) {
    kdop_contact const& c = rows[(size_t)r];
    P& p = work_pool[cand[3 * (size_t)c.cand]];
    (*p.m_callback)(V::make(c.p[0], c.p[1], c.p[2]), V::make(c.n[0], c.n[1], c.n[2]), (T)c.depth);
  }
}

}  // namespace kdop

#endif
