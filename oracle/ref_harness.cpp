// Harness around the reference's own CPU (kdop::sequential) collision path.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's headers and MESH_ARRAY sources (see oracle/Makefile) into
// oracle/_ref/libkdop_ref*.so.  Only tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py load it, as the checker or as the timed
// reference arm; the product library never links it.
//
// Two builds come from this one source:
//   REF_RECORD=1  libkdop_ref_record.so: the include guards of
//                 geometry_overlap_dop_dop.h and
//                 kdop_select_contact_point_algorithm.h are pre-defined so that
//                 same-semantics replacements count every kDOP node-pair test
//                 (SIMULATION/KDOP/KDOP/include/kdop_tandem_traversal.h:42,164)
//                 and record every leaf pair that reaches contact generation
//                 (kdop_tandem_traversal.h:116).
//   REF_RECORD=0  libkdop_ref_time.so: the unmodified reference headers, used
//                 to time the reference's per-step hot path.
//
// Both follow the reference's pipeline: scene set-up reorders each mesh
// (Morton, narrow_shape_types.h:172), computes its surface map (:182) and
// builds its tree on the rest positions (narrow_object.h:121); each step
// poses the vertices and refits (narrow_update_kdop_bvh.h:146-171), then runs
// the tandem traversal with contact generation
// (narrow_tetramesh_tetramesh.h:68-85 -> kdop_tandem_traversal.h:199-226).
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>
#include <map>
#include <chrono>
#include <thread>
#include <atomic>
#include <algorithm>
#include <limits>

#include <tiny_math_types.h>
#include <types/geometry_dop.h>
#include <overlap/geometry_overlap_interval_interval.h>

#if REF_RECORD
// ---- counting replacement for geometry_overlap_dop_dop.h:13-25 -------------
#define GEOMETRY_OVERLAP_DOP_DOP_H
namespace refh { extern thread_local long long g_tests; }
namespace geometry {
template <typename T, size_t K>
inline bool overlap_dop_dop(DOP<T, K> const& A, DOP<T, K> const& B) {
  ++refh::g_tests;
  for (size_t k = 0u; k < K / 2; ++k)
    if (!overlap_interval_interval(A(k), B(k))) return false;
  return true;
}
}  // namespace geometry
#endif

#include <geometry.h>

#if REF_RECORD
// ---- recording replacement for kdop_select_contact_point_algorithm.h -------
#define KDOP_SELECT_CONTACT_POINT_ALGORITHM_H
namespace refh {
struct Recorder {
  virtual void leaf_pair(float const* a12, float const* b12) = 0;
  virtual void leaf_pair(double const* a12, double const* b12) = 0;
  virtual ~Recorder() {}
};
extern thread_local Recorder* g_recorder;
}  // namespace refh
namespace kdop {
class SelectContactPointAlgorithm {
 public:
  template <typename V>
  static bool call_algorithm(geometry::Tetrahedron<V> const& A, geometry::Tetrahedron<V> const& B,
                             geometry::ContactsCallback<V>& callback,
                             std::vector<bool> const& surface_A, std::vector<bool> const& surface_B) {
    typedef typename V::real_type T;
    T a[12], b[12];
    for (int v = 0; v < 4; ++v)
      for (int c = 0; c < 3; ++c) {
        a[3 * v + c] = A.p(v)(c);
        b[3 * v + c] = B.p(v)(c);
      }
    if (refh::g_recorder) refh::g_recorder->leaf_pair(a, b);
    // kdop_select_contact_point_algorithm.h:30 default choice
    return geometry::contacts_tetrahedron_tetrahedron(A, B, callback, surface_A, surface_B,
                                                      geometry::MOST_OPPOSING_SURFACES());
  }
};
}  // namespace kdop
#endif

#include <mesh_array.h>
#include <mesh_array_compute_surface_map.h>
#include <kdop_tree.h>
#include <kdop_make_tree.h>
#include <kdop_refit_tree.h>
#include <kdop_mesh_reorder.h>
#include <kdop_test_pair.h>
#include <kdop_tandem_traversal.h>
#include <broad.h>
#include <prox_math_policy.h>
#include <prox_contact_point.h>

namespace refh {
#if REF_RECORD
thread_local long long g_tests = 0;
thread_local Recorder* g_recorder = 0;
#endif

using mesh_array::T4Mesh;

template <typename T>
struct Mesh {
  T4Mesh mesh;
  mesh_array::VertexAttribute<T, T4Mesh> X, Y, Z;
  mesh_array::TetrahedronAttribute<mesh_array::TetrahedronSurfaceInfo, T4Mesh> surf;
  std::vector<T> rest;  // rest positions in this mesh's vertex order
};

template <typename T>
static void make_mesh(Mesh<T>& m, int nv, float const* xyz, int nt, unsigned const* tets) {
  m.mesh.clear();
  m.mesh.set_capacity(nv, nt);
  for (int i = 0; i < nv; ++i) m.mesh.push_vertex();
  for (int t = 0; t < nt; ++t)
    m.mesh.push_tetrahedron(m.mesh.vertex(tets[4 * t + 0]), m.mesh.vertex(tets[4 * t + 1]),
                            m.mesh.vertex(tets[4 * t + 2]), m.mesh.vertex(tets[4 * t + 3]));
  m.X.bind(m.mesh);
  m.Y.bind(m.mesh);
  m.Z.bind(m.mesh);
  for (int i = 0; i < nv; ++i) {
    mesh_array::Vertex const& v = m.mesh.vertex(i);
    m.X(v) = (T)xyz[3 * i + 0];
    m.Y(v) = (T)xyz[3 * i + 1];
    m.Z(v) = (T)xyz[3 * i + 2];
  }
}

// Copy the current X, Y, Z as the rest positions.
template <typename T>
static void keep_rest(Mesh<T>& m) {
  size_t N = m.mesh.vertex_size();
  m.rest.resize(3 * N);
  for (size_t n = 0; n < N; ++n) {
    mesh_array::Vertex const& v = m.mesh.vertex(n);
    m.rest[3 * n] = m.X(v);
    m.rest[3 * n + 1] = m.Y(v);
    m.rest[3 * n + 2] = m.Z(v);
  }
}

// The rigid transform of narrow::update_kdop_bvh
// (SIMULATION/NARROW/NARROW/include/narrow_update_kdop_bvh.h:154-165):
// X = tiny::rotate(q, rest) + p for every vertex, q = (w, x, y, z).
template <typename T>
static void pose_mesh(Mesh<T>& m, float const* q, float const* p) {
  typedef tiny::MathTypes<T> M;
  typedef typename M::vector3_type V;
  typename M::quaternion_type Q((T)q[0], (T)q[1], (T)q[2], (T)q[3]);
  V P = V::make((T)p[0], (T)p[1], (T)p[2]);
  size_t N = m.mesh.vertex_size();
  for (size_t n = 0; n < N; ++n) {
    mesh_array::Vertex const& v = m.mesh.vertex(n);
    V r0 = V::make(m.rest[3 * n], m.rest[3 * n + 1], m.rest[3 * n + 2]);
    V r = tiny::rotate(Q, r0) + P;
    m.X(v) = r(0);
    m.Y(v) = r(1);
    m.Z(v) = r(2);
  }
}

// Copy the reference's Morton-reordered mesh (kdop_mesh_reorder.h:173-353,
// selected as the default at :364-387) into `out`.
template <typename T>
static void reorder_mesh(Mesh<T> const& in, Mesh<T>& out) {
  kdop::mesh_reorder<T>(in.mesh, in.X, in.Y, in.Z, out.mesh, out.X, out.Y, out.Z);
}

// Key of a tetrahedron by the bit patterns of its 12 coordinates.
struct Key {
  uint32_t w[12];
  bool operator<(Key const& o) const { return std::memcmp(w, o.w, sizeof(w)) < 0; }
};
template <typename T>
static Key key_of(T const* c12) {
  Key k;
  for (int i = 0; i < 12; ++i) {
    float f = (float)c12[i];
    std::memcpy(&k.w[i], &f, 4);
  }
  return k;
}
template <typename T>
static Key key_of_mesh_tet(Mesh<T> const& m, size_t t) {
  mesh_array::Tetrahedron const& tet = m.mesh.tetrahedron(t);
  size_t vi[4] = {tet.i(), tet.j(), tet.k(), tet.m()};
  float c[12];
  for (int v = 0; v < 4; ++v) {
    mesh_array::Vertex const& vv = m.mesh.vertex(vi[v]);
    c[3 * v + 0] = (float)m.X(vv);
    c[3 * v + 1] = (float)m.Y(vv);
    c[3 * v + 2] = (float)m.Z(vv);
  }
  return key_of(c);
}

template <typename T>
struct StoreCallback : public geometry::ContactsCallback<typename tiny::MathTypes<T>::vector3_type> {
  typedef typename tiny::MathTypes<T>::vector3_type V;
  std::vector<double> rows;  // p3 n3 d pair
  long long current_pair;
  StoreCallback() : current_pair(-1) {}
  void operator()(V const& p, V const& n, T const& d) {
    rows.push_back((double)p(0)); rows.push_back((double)p(1)); rows.push_back((double)p(2));
    rows.push_back((double)n(0)); rows.push_back((double)n(1)); rows.push_back((double)n(2));
    rows.push_back((double)d);
    rows.push_back((double)current_pair);
  }
};

template <typename T>
struct CountCallback : public geometry::ContactsCallback<typename tiny::MathTypes<T>::vector3_type> {
  typedef typename tiny::MathTypes<T>::vector3_type V;
  std::vector<float> rows;  // the PROX callback appends a contact record per call
  void operator()(V const& p, V const& n, T const& d) {
    rows.push_back((float)p(0)); rows.push_back((float)p(1)); rows.push_back((float)p(2));
    rows.push_back((float)n(0)); rows.push_back((float)n(1)); rows.push_back((float)n(2));
    rows.push_back((float)d);
  }
};

#if REF_RECORD
template <typename T>
struct PairRecorder : public Recorder {
  std::map<Key, unsigned> const* mapA;
  std::map<Key, unsigned> const* mapB;
  std::vector<unsigned> pairs;
  StoreCallback<T>* cb;
  long long missing;
  PairRecorder() : mapA(0), mapB(0), cb(0), missing(0) {}
  template <typename R>
  void rec(R const* a, R const* b) {
    std::map<Key, unsigned>::const_iterator ia = mapA->find(key_of(a));
    std::map<Key, unsigned>::const_iterator ib = mapB->find(key_of(b));
    if (ia == mapA->end() || ib == mapB->end()) { ++missing; return; }
    if (cb) cb->current_pair = (long long)(pairs.size() / 2);
    pairs.push_back(ia->second);
    pairs.push_back(ib->second);
  }
  void leaf_pair(float const* a, float const* b) { rec(a, b); }
  void leaf_pair(double const* a, double const* b) { rec(a, b); }
};
#endif

template <size_t K>
struct KTag {};

// Preorder walk of the reference tree (one chunk level).  Emits, per node,
// K floats of slabs (lo,hi interleaved) and the tet index (leaf) or -1.
template <typename T, size_t K>
static void walk(kdop::SubTree<T, K> const& st, size_t idx, std::vector<float>& vols,
                 std::vector<long long>& leaf) {
  kdop::Node<T, K> const& n = st.m_nodes[idx];
  for (size_t k = 0; k < K / 2; ++k) {
    vols.push_back((float)n.m_volume(k).lower());
    vols.push_back((float)n.m_volume(k).upper());
  }
  if (n.is_leaf()) {
    leaf.push_back((long long)n.m_start);
    return;
  }
  leaf.push_back(-1);
  walk<T, K>(st, n.m_start, vols, leaf);
  walk<T, K>(st, n.m_end, vols, leaf);
}

// Scene set-up of one mesh: reorder (optional), surface map, tree on rest.
template <typename T, size_t K>
static void setup_mesh(int nv, float const* rest, int nt, unsigned const* tets, int reorder,
                       unsigned long long mem_bytes, Mesh<T>& out, kdop::Tree<T, K>& tree) {
  typedef typename tiny::MathTypes<T>::vector3_type V;
  if (reorder) {
    Mesh<T> raw;
    make_mesh(raw, nv, rest, nt, tets);
    reorder_mesh(raw, out);
  } else {
    make_mesh(out, nv, rest, nt, tets);
  }
  mesh_array::compute_surface_map(out.mesh, out.X, out.Y, out.Z, out.surf);
  keep_rest(out);
  tree = kdop::make_tree<V, K, T>((size_t)mem_bytes, out.mesh, out.X, out.Y, out.Z, kdop::sequential());
}

#if REF_RECORD
// One mesh pair through set-up and one simulation step, recording the leaf
// pairs (in the caller's tet numbering), the contacts and the test count.
template <size_t K>
static int traverse_k(unsigned long long mem_bytes, int reorder, int nvA, float const* restA, float const* qA,
                      float const* pA, int ntA, unsigned const* tetsA, int nvB, float const* restB, float const* qB,
                      float const* pB, int ntB, unsigned const* tetsB, long long cap_pairs, unsigned* out_pairs,
                      long long* out_npairs, long long cap_contacts, float* out_contacts, long long* out_ncontacts,
                      long long* out_tests, long long cap_nodes, float* out_volsA, long long* out_leafA,
                      long long* out_nnodesA) {
  typedef float T;
  typedef tiny::MathTypes<T>::vector3_type V;
  Mesh<T> a, b;
  kdop::Tree<T, K> ta, tb;
  setup_mesh<T, K>(nvA, restA, ntA, tetsA, reorder, mem_bytes, a, ta);
  setup_mesh<T, K>(nvB, restB, ntB, tetsB, reorder, mem_bytes, b, tb);
  pose_mesh(a, qA, pA);
  kdop::refit_tree<V, K, T>(ta, a.mesh, a.X, a.Y, a.Z, kdop::sequential());
  pose_mesh(b, qB, pB);
  kdop::refit_tree<V, K, T>(tb, b.mesh, b.X, b.Y, b.Z, kdop::sequential());

  // caller's tet numbering, keyed by the posed coordinates of the input meshes
  Mesh<T> a0, b0;
  make_mesh(a0, nvA, restA, ntA, tetsA);
  make_mesh(b0, nvB, restB, ntB, tetsB);
  keep_rest(a0);
  keep_rest(b0);
  pose_mesh(a0, qA, pA);
  pose_mesh(b0, qB, pB);
  std::map<Key, unsigned> mapA, mapB;
  for (int t = 0; t < ntA; ++t) mapA[key_of_mesh_tet(a0, (size_t)t)] = (unsigned)t;
  for (int t = 0; t < ntB; ++t) mapB[key_of_mesh_tet(b0, (size_t)t)] = (unsigned)t;

  if (out_volsA && ta.number_of_levels() == 1 && ta.branches().size() == 1) {
    std::vector<float> vols;
    std::vector<long long> leaf;
    walk<T, K>(ta.branches()[0], 0, vols, leaf);
    *out_nnodesA = (long long)leaf.size();
    if ((long long)leaf.size() <= cap_nodes) {
      std::memcpy(out_volsA, vols.data(), vols.size() * sizeof(float));
      for (size_t i = 0; i < leaf.size(); ++i) {
        long long t = leaf[i];
        if (t >= 0) {
          std::map<Key, unsigned>::const_iterator it = mapA.find(key_of_mesh_tet(a, (size_t)t));
          t = (it == mapA.end()) ? -2 : (long long)it->second;
        }
        out_leafA[i] = t;
      }
    }
  }

  StoreCallback<T> cb;
  PairRecorder<T> rec;
  rec.mapA = &mapA;
  rec.mapB = &mapB;
  rec.cb = &cb;
  std::vector<kdop::TestPair<V, K, T> > pool;
  pool.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf, cb));
  g_tests = 0;
  g_recorder = &rec;
  kdop::tandem_traversal<V, K, T>(pool, kdop::sequential());
  g_recorder = 0;
  *out_tests = g_tests;
  long long np = (long long)rec.pairs.size() / 2;
  *out_npairs = np;
  if (np <= cap_pairs && out_pairs) std::memcpy(out_pairs, rec.pairs.data(), rec.pairs.size() * sizeof(unsigned));
  long long nc = (long long)cb.rows.size() / 8;
  *out_ncontacts = nc;
  if (nc <= cap_contacts && out_contacts)
    for (size_t i = 0; i < cb.rows.size(); ++i) out_contacts[i] = (float)cb.rows[i];
  return rec.missing ? -3 : 0;
}
#endif


// Contacts of explicit tet pairs with the reference's MOST_OPPOSING_SURFACES
// algorithm (geometry_contacts_tetrahedron_tetrahedron.h:1313-1345), in T.
template <typename T>
static int contacts_pairs_t(float const* xyzA, unsigned const* tetsA, unsigned char const* surfA,
                            float const* xyzB, unsigned const* tetsB, unsigned char const* surfB,
                            long long n_pairs, unsigned const* pairs, long long cap, double* out,
                            long long* out_n) {
  typedef typename tiny::MathTypes<T>::vector3_type V;
  StoreCallback<T> cb;
  for (long long i = 0; i < n_pairs; ++i) {
    unsigned const* ta = tetsA + 4 * (size_t)pairs[2 * i];
    unsigned const* tb = tetsB + 4 * (size_t)pairs[2 * i + 1];
    V pa[4], pb[4];
    for (int v = 0; v < 4; ++v) {
      pa[v] = V::make((T)xyzA[3 * ta[v]], (T)xyzA[3 * ta[v] + 1], (T)xyzA[3 * ta[v] + 2]);
      pb[v] = V::make((T)xyzB[3 * tb[v]], (T)xyzB[3 * tb[v] + 1], (T)xyzB[3 * tb[v] + 2]);
    }
    std::vector<bool> sA(4), sB(4);
    unsigned char fa = surfA[pairs[2 * i]], fb = surfB[pairs[2 * i + 1]];
    for (int v = 0; v < 4; ++v) {
      sA[v] = (fa >> v) & 1;
      sB[v] = (fb >> v) & 1;
    }
    if (!fa || !fb) continue;  // kdop_tandem_traversal.h:61-88
    geometry::Tetrahedron<V> const A = geometry::make_tetrahedron(pa[0], pa[1], pa[2], pa[3]);
    geometry::Tetrahedron<V> const B = geometry::make_tetrahedron(pb[0], pb[1], pb[2], pb[3]);
    cb.current_pair = i;
    geometry::contacts_tetrahedron_tetrahedron(A, B, cb, sA, sB, geometry::MOST_OPPOSING_SURFACES());
  }
  long long nc = (long long)cb.rows.size() / 8;
  *out_n = nc;
  if (nc <= cap && out) std::memcpy(out, cb.rows.data(), cb.rows.size() * sizeof(double));
  return 0;
}

// ---- timing of the unmodified reference path --------------------------------
// Untimed scene set-up: reorder, surface map and make_tree on the rest
// positions of every mesh in use.  Timed, per mesh pair, the reference's
// simulation-step hot path: rigid transform + refit_tree of both meshes
// (narrow_update_kdop_bvh.h:146-171) and tandem_traversal with contact
// generation (kdop_tandem_traversal.h:199-226).  Pairs run on `threads`
// threads, one pair at a time per thread.
template <size_t K>
static int time_pairs_k(unsigned long long mem_bytes, int n_meshes, long long const* v_off, float const* xyz,
                        float const* quat, float const* pos, long long const* t_off, unsigned const* tets,
                        long long n_pairs, unsigned const* pairs, int threads, int repeats, double* out_seconds,
                        long long* out_contacts) {
  typedef float T;
  typedef tiny::MathTypes<T>::vector3_type V;
  std::vector<Mesh<T>*> meshes(n_meshes, (Mesh<T>*)0);
  std::vector<kdop::Tree<T, K>*> trees(n_meshes, (kdop::Tree<T, K>*)0);
  std::vector<char> used(n_meshes, 0);
  for (long long p = 0; p < n_pairs; ++p) used[pairs[2 * p]] = used[pairs[2 * p + 1]] = 1;
  if (threads < 1) threads = 1;
  // untimed set-up (reorder, surface map, make_tree on the rest positions), meshes in parallel
  {
    std::atomic<int> nm(0);
    auto setup = [&]() {
      for (;;) {
        int m = nm.fetch_add(1);
        if (m >= n_meshes) break;
        if (!used[m]) continue;
        int nv = (int)(v_off[m + 1] - v_off[m]);
        int nt = (int)(t_off[m + 1] - t_off[m]);
        std::vector<unsigned> lt(tets + 4 * t_off[m], tets + 4 * t_off[m + 1]);
        meshes[m] = new Mesh<T>();
        trees[m] = new kdop::Tree<T, K>();
        setup_mesh<T, K>(nv, xyz + 3 * v_off[m], nt, lt.data(), 1, mem_bytes, *meshes[m], *trees[m]);
      }
    };
    int ns = (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (int i = 0; i < ns; ++i) th.push_back(std::thread(setup));
    for (size_t i = 0; i < th.size(); ++i) th[i].join();
  }
  std::vector<long long> contacts(threads, 0);
  std::atomic<long long> next(0);
  auto worker = [&](int tid) {
    for (;;) {
      long long p = next.fetch_add(1);
      if (p >= n_pairs) break;
      unsigned ia = pairs[2 * p], ib = pairs[2 * p + 1];
      Mesh<T>& A = *meshes[ia];
      Mesh<T>& B = *meshes[ib];
      pose_mesh(A, quat + 4 * ia, pos + 3 * ia);
      kdop::refit_tree<V, K, T>(*trees[ia], A.mesh, A.X, A.Y, A.Z, kdop::sequential());
      pose_mesh(B, quat + 4 * ib, pos + 3 * ib);
      kdop::refit_tree<V, K, T>(*trees[ib], B.mesh, B.X, B.Y, B.Z, kdop::sequential());
      CountCallback<T> cb;
      std::vector<kdop::TestPair<V, K, T> > pool;
      pool.push_back(kdop::TestPair<V, K, T>(*trees[ia], *trees[ib], A.mesh, B.mesh, A.X, B.X, A.Y, B.Y, A.Z,
                                             B.Z, A.surf, B.surf, cb));
      kdop::tandem_traversal<V, K, T>(pool, kdop::sequential());
      contacts[tid] += (long long)cb.rows.size() / 7;
    }
  };
  // `repeats` timed simulation steps over all pairs
  for (int r = 0; r < std::max(repeats, 1); ++r) {
    next = 0;
    for (int i = 0; i < threads; ++i) contacts[i] = 0;
    auto t0 = std::chrono::steady_clock::now();
    if (threads == 1) {
      worker(0);
    } else {
      std::vector<std::thread> th;
      for (int i = 0; i < threads; ++i) th.push_back(std::thread(worker, i));
      for (size_t i = 0; i < th.size(); ++i) th[i].join();
    }
    auto t1 = std::chrono::steady_clock::now();
    out_seconds[r] = std::chrono::duration<double>(t1 - t0).count();
  }
  long long c = 0;
  for (int i = 0; i < threads; ++i) c += contacts[i];
  *out_contacts = c;
  for (int m = 0; m < n_meshes; ++m) {
    delete trees[m];
    delete meshes[m];
  }
  return 0;
}

}  // namespace refh

extern "C" {

int ref_surface_map(int nv, float const* xyz, int nt, unsigned const* tets, unsigned char* out_surf) {
  refh::Mesh<float> m;
  refh::make_mesh(m, nv, xyz, nt, tets);
  mesh_array::compute_surface_map(m.mesh, m.X, m.Y, m.Z, m.surf);
  for (int t = 0; t < nt; ++t) {
    mesh_array::TetrahedronSurfaceInfo const& s = m.surf(m.mesh.tetrahedron(t));
    out_surf[t] = (unsigned char)((s.m_i ? 1 : 0) | (s.m_j ? 2 : 0) | (s.m_k ? 4 : 0) | (s.m_m ? 8 : 0));
  }
  return 0;
}

int ref_mesh_reorder(int nv, float const* xyz, int nt, unsigned const* tets, float* out_xyz, unsigned* out_tets) {
  refh::Mesh<float> a, b;
  refh::make_mesh(a, nv, xyz, nt, tets);
  refh::reorder_mesh(a, b);
  if ((int)b.mesh.vertex_size() != nv || (int)b.mesh.tetrahedron_size() != nt) return -1;
  for (int i = 0; i < nv; ++i) {
    mesh_array::Vertex const& v = b.mesh.vertex(i);
    out_xyz[3 * i + 0] = b.X(v);
    out_xyz[3 * i + 1] = b.Y(v);
    out_xyz[3 * i + 2] = b.Z(v);
  }
  for (int t = 0; t < nt; ++t) {
    mesh_array::Tetrahedron const& tt = b.mesh.tetrahedron(t);
    out_tets[4 * t + 0] = (unsigned)tt.i();
    out_tets[4 * t + 1] = (unsigned)tt.j();
    out_tets[4 * t + 2] = (unsigned)tt.k();
    out_tets[4 * t + 3] = (unsigned)tt.m();
  }
  return 0;
}

// tiny::rotate(q, r) + p (narrow_update_kdop_bvh.h:160), q = (w, x, y, z).
int ref_rotate(float const* q, float const* p, int nv, float const* xyz, float* out) {
  refh::Mesh<float> m;
  std::vector<unsigned> none(4, 0);
  refh::make_mesh(m, nv, xyz, 0, none.data());
  refh::keep_rest(m);
  refh::pose_mesh(m, q, p);
  for (int i = 0; i < nv; ++i) {
    mesh_array::Vertex const& v = m.mesh.vertex(i);
    out[3 * i] = m.X(v);
    out[3 * i + 1] = m.Y(v);
    out[3 * i + 2] = m.Z(v);
  }
  return 0;
}

// Unit direction table of DirectionTableHelper<V,K/2>::make()
// (geometry_direction_table.h:124-176), as float triples.
int ref_direction_table(int K, float* out) {
  typedef tiny::MathTypes<float>::vector3_type V;
#define REFH_DT(N)                                                          \
  {                                                                         \
    geometry::DirectionTable<V, N> D = geometry::DirectionTableHelper<V, N>::make(); \
    for (size_t i = 0; i < N; ++i)                                          \
      for (int c = 0; c < 3; ++c) out[3 * i + c] = D(i)(c);                 \
    return (int)N;                                                          \
  }
  switch (K) {
    case 6: REFH_DT(3)
    case 8: REFH_DT(4)
    case 12: REFH_DT(6)
    case 14: REFH_DT(7)
    case 18: REFH_DT(9)
    case 20: REFH_DT(10)
    case 26: REFH_DT(13)
  }
#undef REFH_DT
  return -1;
}

int ref_contacts_pairs(int fp64, float const* xyzA, unsigned const* tetsA, unsigned char const* surfA,
                       float const* xyzB, unsigned const* tetsB, unsigned char const* surfB, long long n_pairs,
                       unsigned const* pairs, long long cap, double* out, long long* out_n) {
  if (fp64)
    return refh::contacts_pairs_t<double>(xyzA, tetsA, surfA, xyzB, tetsB, surfB, n_pairs, pairs, cap, out, out_n);
  return refh::contacts_pairs_t<float>(xyzA, tetsA, surfA, xyzB, tetsB, surfB, n_pairs, pairs, cap, out, out_n);
}

#if REF_RECORD
int ref_traverse(int K, unsigned long long mem_bytes, int reorder, int nvA, float const* restA, float const* qA,
                 float const* pA, int ntA, unsigned const* tetsA, int nvB, float const* restB, float const* qB,
                 float const* pB, int ntB, unsigned const* tetsB, long long cap_pairs, unsigned* out_pairs,
                 long long* out_npairs, long long cap_contacts, float* out_contacts, long long* out_ncontacts,
                 long long* out_tests, long long cap_nodes, float* out_volsA, long long* out_leafA,
                 long long* out_nnodesA) {
#define REFH_TR(KK)                                                                                      \
  case KK:                                                                                               \
    return refh::traverse_k<KK>(mem_bytes, reorder, nvA, restA, qA, pA, ntA, tetsA, nvB, restB, qB, pB, \
                                ntB, tetsB, cap_pairs, out_pairs, out_npairs, cap_contacts, out_contacts,\
                                out_ncontacts, out_tests, cap_nodes, out_volsA, out_leafA, out_nnodesA);
  switch (K) {
    REFH_TR(6) REFH_TR(8) REFH_TR(12) REFH_TR(14) REFH_TR(18) REFH_TR(20) REFH_TR(26)
  }
#undef REFH_TR
  return -1;
}
#endif

int ref_time_pairs(int K, unsigned long long mem_bytes, int n_meshes, long long const* v_off, float const* xyz,
                   float const* quat, float const* pos, long long const* t_off, unsigned const* tets,
                   long long n_pairs, unsigned const* pairs, int threads, int repeats, double* out_seconds,
                   long long* out_contacts) {
#define REFH_TP(KK)                                                                                  \
  case KK:                                                                                           \
    return refh::time_pairs_k<KK>(mem_bytes, n_meshes, v_off, xyz, quat, pos, t_off, tets, n_pairs,  \
                                  pairs, threads, repeats, out_seconds, out_contacts);
  switch (K) {
    REFH_TP(6) REFH_TP(8) REFH_TP(12) REFH_TP(14) REFH_TP(18) REFH_TP(20) REFH_TP(26)
  }
#undef REFH_TP
  return -1;
}


// Broad phase of the reference (broad_find_overlaps.h): every body a box of
// its position +- its bounding radius (prox_rigid_body.h:159-172); overlapping
// body pairs (lower index first, lexicographically sorted) by the all-pair
// (algorithm 0) or the grid (1) algorithm.
struct RefBox : public broad::Object<float> {
  float x, y, z, r;
  void get_box(float& mx, float& my, float& mz, float& Mx, float& My, float& Mz) const {
    mx = x - r;
    my = y - r;
    mz = z - r;
    Mx = x + r;
    My = y + r;
    Mz = z + r;
  }
};

int ref_broad_pairs(int n, float const* pos, float const* radius, int algorithm, unsigned* out, long long cap,
                    long long* n_out) {
  util::LogInfo::console() = false;
  util::LogInfo::on() = false;
  std::vector<RefBox> boxes((size_t)n);
  broad::System<float> sys;
  for (int i = 0; i < n; ++i) {
    boxes[i].x = pos[3 * i];
    boxes[i].y = pos[3 * i + 1];
    boxes[i].z = pos[3 * i + 2];
    boxes[i].r = radius[i];
    sys.connect(&boxes[i]);
  }
  std::vector<std::pair<broad::Object<float>*, broad::Object<float>*> > overlaps;
  float eff = 0.f;
  if (algorithm == 1) {
    sys.compute_optimal_cell_spacing();
    broad::find_overlaps(sys, overlaps, eff, broad::grid_algorithm());
  } else {
    broad::find_overlaps(sys, overlaps, eff, broad::all_pair_algorithm());
  }
  *n_out = (long long)overlaps.size();
  if ((long long)overlaps.size() > cap) return -2;
  for (size_t k = 0; k < overlaps.size(); ++k) {
    out[2 * k] = (unsigned)(static_cast<RefBox*>(overlaps[k].first) - boxes.data());
    out[2 * k + 1] = (unsigned)(static_cast<RefBox*>(overlaps[k].second) - boxes.data());
  }
  return 0;
}

// Bounding radius of a mesh about its body origin: max |r0| over the rest
// vertices (narrow_shape_types.h:189-206).
float ref_mesh_radius(int nv, float const* xyz) {
  typedef tiny::MathTypes<float>::vector3_type V;
  float r = 0.f;
  for (int i = 0; i < nv; ++i) {
    V const r0 = V::make(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    r = std::max(r, tiny::norm(r0));
  }
  return r;
}

// PROX's contact point reduction (prox_collision_detection.h:341-350) on
// rows of (p, n, depth) with the bodies (a, b) of each row, through the
// reference's own ContactPoint comparisons (prox_contact_point.h:91-194),
// std::sort and std::unique.  out_rows: 7 floats and out_bodies: 2 ids per
// kept row, in the reduced order.
int ref_reduce_contacts(long long n, float const* rows, unsigned const* bodies, int n_bodies, float* out_rows,
                        unsigned* out_bodies, long long* n_out) {
  typedef prox::MathPolicy<float> M;
  typedef M::vector3_type V;
  std::vector<prox::RigidBody<M> > body((size_t)std::max(n_bodies, 1));
  std::vector<prox::ContactPoint<M> > c((size_t)n);
  for (long long i = 0; i < n; ++i) {
    float const* r = rows + 7 * i;
    c[i].set_position(V::make(r[0], r[1], r[2]));
    c[i].set_normal(V::make(r[3], r[4], r[5]));
    c[i].set_depth(r[6]);
    c[i].set_body_i(&body[bodies[2 * i]]);
    c[i].set_body_j(&body[bodies[2 * i + 1]]);
  }
  std::sort(c.begin(), c.end());
  c.erase(std::unique(c.begin(), c.end()), c.end());
  *n_out = (long long)c.size();
  for (size_t k = 0; k < c.size(); ++k) {
    for (int j = 0; j < 3; ++j) {
      out_rows[7 * k + j] = c[k].get_position()(j);
      out_rows[7 * k + 3 + j] = c[k].get_normal()(j);
    }
    out_rows[7 * k + 6] = c[k].get_depth();
    out_bodies[2 * k] = (unsigned)(c[k].get_body_i() - body.data());
    out_bodies[2 * k + 1] = (unsigned)(c[k].get_body_j() - body.data());
  }
  return 0;
}

}  // extern "C"
