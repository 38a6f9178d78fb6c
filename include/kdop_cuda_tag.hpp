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
//       replaces kdop_refit_tree.h:120-162 for one-chunk trees (make_tree with
//       mem_bytes = SIZE_MAX, the reference's gProximity set-up): the node
//       volumes are computed on the GPU and written back into the Tree.
//
// Errors come back as std::runtime_error carrying kdop_last_error().
#ifndef KDOP_CUDA_TAG_HPP
#define KDOP_CUDA_TAG_HPP

#include <algorithm>
#include <cstring>
#include <map>
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

// Host copy of one reference mesh in the C ABI's layout.
struct MeshCopy {
  std::vector<float> xyz;
  std::vector<uint32_t> tets;
  std::vector<uint8_t> surf;
  std::vector<uint32_t> order;  // 0..n_tets-1: the tree of make_tree over the mesh as given
};

template <typename T>
MeshCopy copy_mesh(mesh_array::T4Mesh const& mesh, mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& X,
                   mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Y,
                   mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Z,
                   mesh_array::TetrahedronAttribute<mesh_array::TetrahedronSurfaceInfo, mesh_array::T4Mesh> const* S) {
  MeshCopy c;
  size_t nv = mesh.vertex_size(), nt = mesh.tetrahedron_size();
  c.xyz.resize(3 * nv);
  for (size_t i = 0; i < nv; ++i) {
    mesh_array::Vertex const& v = mesh.vertex(i);
    c.xyz[3 * i] = (float)X(v);
    c.xyz[3 * i + 1] = (float)Y(v);
    c.xyz[3 * i + 2] = (float)Z(v);
  }
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

template <typename T, size_t K>
void write_preorder(kdop::SubTree<T, K>& st, size_t idx, float const* vol, size_t& k) {
  kdop::Node<T, K>& n = st.m_nodes[idx];
  for (size_t s = 0; s < K / 2; ++s) {
    n.m_volume(s).lower() = (T)vol[k * K + 2 * s];
    n.m_volume(s).upper() = (T)vol[k * K + 2 * s + 1];
  }
  ++k;
  if (n.is_leaf()) return;
  write_preorder<T, K>(st, n.m_start, vol, k);
  write_preorder<T, K>(st, n.m_end, vol, k);
}

}  // namespace cuda_detail

// refit_tree on the GPU for a one-chunk tree; the tree topology of the scene
// built here equals make_tree's for a mesh already in Morton order.
template <typename V, size_t K, typename T>
inline void refit_tree(Tree<T, K>& tree, mesh_array::T4Mesh const& mesh,
                       mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& X,
                       mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Y,
                       mesh_array::VertexAttribute<T, mesh_array::T4Mesh> const& Z, cuda const& tag) {
  if (tree.number_of_levels() != 1 || tree.branches().size() != 1)
    throw std::runtime_error("kdop::cuda refit_tree: one-chunk trees only (make_tree with mem_bytes = SIZE_MAX)");
  cuda_detail::MeshCopy m = cuda_detail::copy_mesh<T>(mesh, X, Y, Z, 0);
  kdop_mesh_desc d;
  d.n_verts = (int64_t)mesh.vertex_size();
  d.xyz = m.xyz.data();
  d.n_tets = (int64_t)mesh.tetrahedron_size();
  d.tets = m.tets.data();
  d.surface = m.surf.data();
  d.leaf_order = m.order.data();
  kdop_scene* sc = 0;
  cuda_detail::check(tag.ctx, kdop_scene_create(tag.ctx, (int)K, 1, &d, &sc), "scene_create");
  int64_t nn = d.n_tets > 0 ? 2 * d.n_tets - 1 : 0;
  std::vector<float> vol((size_t)std::max<int64_t>(nn, 1) * K);
  std::vector<int64_t> tet((size_t)std::max<int64_t>(nn, 1));
  int64_t got = 0;
  int rc = kdop_refit(sc, KDOP_REFIT_VERTICES);
  if (rc == KDOP_OK) rc = kdop_read_tree(sc, 0, nn, vol.data(), tet.data(), &got);
  kdop_scene_destroy(sc);
  cuda_detail::check(tag.ctx, rc, "refit_tree");
  size_t k = 0;
  cuda_detail::write_preorder<T, K>(tree.branches()[0], 0, vol.data(), k);
  tree.m_root = tree.branches()[0].m_nodes[0].m_volume;
}

// tandem_traversal of a pool of test pairs on the GPU.
template <typename V, size_t K, typename T>
inline void tandem_traversal(std::vector<TestPair<V, K, T> >& work_pool, cuda const& tag) {
  if (work_pool.empty()) return;
  typedef TestPair<V, K, T> P;
  // distinct meshes of the pool (by object identity)
  std::map<const void*, int> index;
  std::vector<cuda_detail::MeshCopy> meshes;
  std::vector<uint32_t> pairs;
  for (size_t i = 0; i < work_pool.size(); ++i) {
    P const& p = work_pool[i];
    const void* keys[2] = {p.m_x_a, p.m_x_b};
    for (int s = 0; s < 2; ++s) {
      if (!index.count(keys[s])) {
        int id = (int)meshes.size();
        index[keys[s]] = id;
        if (s == 0)
          meshes.push_back(cuda_detail::copy_mesh<T>(*p.m_mesh_a, *p.m_x_a, *p.m_y_a, *p.m_z_a, p.m_surface_map_a));
        else
          meshes.push_back(cuda_detail::copy_mesh<T>(*p.m_mesh_b, *p.m_x_b, *p.m_y_b, *p.m_z_b, p.m_surface_map_b));
      }
      pairs.push_back((uint32_t)index[keys[s]]);
    }
  }
  std::vector<kdop_mesh_desc> desc(meshes.size());
  for (size_t m = 0; m < meshes.size(); ++m) {
    desc[m].n_verts = (int64_t)meshes[m].xyz.size() / 3;
    desc[m].xyz = meshes[m].xyz.data();
    desc[m].n_tets = (int64_t)meshes[m].tets.size() / 4;
    desc[m].tets = meshes[m].tets.data();
    desc[m].surface = meshes[m].surf.data();
    desc[m].leaf_order = meshes[m].order.data();
  }
  kdop_scene* sc = 0;
  cuda_detail::check(tag.ctx, kdop_scene_create(tag.ctx, (int)K, (int)desc.size(), desc.data(), &sc),
                     "scene_create");
  int64_t np = (int64_t)work_pool.size();
  // the scene's rest positions are the current ones: refit the volumes there
  int rc = kdop_refit(sc, KDOP_REFIT_VERTICES);
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
  std::vector<uint32_t> cand((size_t)st.n_candidates * 3 + 3);
  std::vector<kdop_contact> rows((size_t)st.n_contacts + 1);
  int64_t nc = 0, nr = 0;
  if (rc == KDOP_OK) rc = kdop_read_candidates(sc, cand.data(), st.n_candidates, &nc);
  if (rc == KDOP_OK) rc = kdop_read_contacts(sc, rows.data(), st.n_contacts, &nr);
  kdop_scene_destroy(sc);
  cuda_detail::check(tag.ctx, rc, "tandem_traversal");
  for (int64_t r = 0; r < nr; ++r) {
    kdop_contact const& c = rows[r];
    P& p = work_pool[cand[3 * c.cand]];
    (*p.m_callback)(V::make(c.p[0], c.p[1], c.p[2]), V::make(c.n[0], c.n[1], c.n[2]), (T)c.depth);
  }
}

}  // namespace kdop

#endif
