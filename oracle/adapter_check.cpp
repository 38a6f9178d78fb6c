// adapter_check.cpp -- TEST INFRASTRUCTURE: the reference's own narrow-phase
// calls run once with kdop::sequential and once with the kdop::cuda tag of
// include/kdop_cuda_tag.hpp (the drop-in binding), on the same meshes.
// Exits 0 when the GPU back-end reproduces the reference: refitted node
// volumes bit for bit and the contacts reported through each pair's
// ContactsCallback as the same multiset of (p, n, d) bit patterns.
//
// Built by `make -C oracle adapter` against the reference's headers and
// libkdop_cuda.so; run by tests/test_gpu_adapter.py on a GPU.
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>

#include <tiny_math_types.h>
#include <geometry.h>
#include <mesh_array.h>
#include <mesh_array_compute_surface_map.h>
#include <kdop_tree.h>
#include <kdop_make_tree.h>
#include <kdop_refit_tree.h>
#include <kdop_mesh_reorder.h>
#include <kdop_test_pair.h>
#include <kdop_tandem_traversal.h>

#include "../include/kdop_cuda_tag.hpp"

typedef tiny::MathTypes<float> MT;
typedef MT::vector3_type V;
typedef float T;
using mesh_array::T4Mesh;
typedef mesh_array::VertexAttribute<T, T4Mesh> Attr;

struct Body {
  T4Mesh raw, mesh;
  Attr X0, Y0, Z0, rX, rY, rZ, X, Y, Z;
  mesh_array::TetrahedronAttribute<mesh_array::TetrahedronSurfaceInfo, T4Mesh> surf;
};

// n^3 cubes, 6 Kuhn tets each, centred on the origin.
static void lattice(Body& b, int n) {
  int m = n + 1;
  b.raw.set_capacity(m * m * m, 6 * n * n * n);
  for (int i = 0; i < m * m * m; ++i) b.raw.push_vertex();
  static const int kuhn[6][4] = {{0, 1, 3, 7}, {0, 1, 7, 5}, {0, 4, 5, 7}, {0, 3, 2, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}};
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        int c[8];
        for (int q = 0; q < 8; ++q) c[q] = (i + (q & 1)) + m * ((j + ((q >> 1) & 1)) + m * (k + ((q >> 2) & 1)));
        for (int t = 0; t < 6; ++t)
          b.raw.push_tetrahedron(b.raw.vertex(c[kuhn[t][0]]), b.raw.vertex(c[kuhn[t][1]]), b.raw.vertex(c[kuhn[t][2]]),
                                 b.raw.vertex(c[kuhn[t][3]]));
      }
  b.rX.bind(b.raw);
  b.rY.bind(b.raw);
  b.rZ.bind(b.raw);
  for (int z = 0; z < m; ++z)
    for (int y = 0; y < m; ++y)
      for (int x = 0; x < m; ++x) {
        mesh_array::Vertex const& v = b.raw.vertex(x + m * (y + m * z));
        b.rX(v) = x - n / 2.0f;
        b.rY(v) = y - n / 2.0f;
        b.rZ(v) = z - n / 2.0f;
      }
  // scene set-up as the narrow phase does it: Morton reorder, surface map
  kdop::mesh_reorder<T>(b.raw, b.rX, b.rY, b.rZ, b.mesh, b.X0, b.Y0, b.Z0);
  mesh_array::compute_surface_map(b.mesh, b.X0, b.Y0, b.Z0, b.surf);
  b.X.bind(b.mesh);
  b.Y.bind(b.mesh);
  b.Z.bind(b.mesh);
}

static void pose(Body& b, MT::quaternion_type const& q, V const& p) {
  for (size_t i = 0; i < b.mesh.vertex_size(); ++i) {
    mesh_array::Vertex const& v = b.mesh.vertex(i);
    V r = tiny::rotate(q, V::make(b.X0(v), b.Y0(v), b.Z0(v))) + p;
    b.X(v) = r(0);
    b.Y(v) = r(1);
    b.Z(v) = r(2);
  }
}

struct Rows : public geometry::ContactsCallback<V> {
  std::vector<uint32_t> bits;
  void operator()(V const& p, V const& n, T const& d) {
    float r[7] = {p(0), p(1), p(2), n(0), n(1), n(2), d};
    uint32_t u[7];
    std::memcpy(u, r, sizeof(r));
    bits.insert(bits.end(), u, u + 7);
  }
  std::vector<std::vector<uint32_t> > sorted() const {
    std::vector<std::vector<uint32_t> > v;
    for (size_t i = 0; i < bits.size(); i += 7) v.push_back(std::vector<uint32_t>(bits.begin() + i, bits.begin() + i + 7));
    std::sort(v.begin(), v.end());
    return v;
  }
};

template <size_t K>
static int run(kdop_ctx* ctx, int n, float pen, float angle) {
  Body a, b;
  lattice(a, n);
  lattice(b, n);
  kdop::Tree<T, K> ta = kdop::make_tree<V, K, T>((size_t)-1, a.mesh, a.X0, a.Y0, a.Z0, kdop::sequential());
  kdop::Tree<T, K> tb = kdop::make_tree<V, K, T>((size_t)-1, b.mesh, b.X0, b.Y0, b.Z0, kdop::sequential());
  MT::quaternion_type qa(1.f, 0.f, 0.f, 0.f);
  float s = std::sin(angle / 2), c = std::cos(angle / 2);
  MT::quaternion_type qb(c, s * 0.267f, s * 0.535f, s * 0.802f);
  pose(a, qa, V::make(0.f, 0.f, 0.f));
  pose(b, qb, V::make((float)n - pen, 0.f, 0.f));

  // refit: sequential vs cuda, node volumes bit for bit
  kdop::Tree<T, K> ta_cuda = ta, tb_cuda = tb;
  kdop::refit_tree<V, K, T>(ta, a.mesh, a.X, a.Y, a.Z, kdop::sequential());
  kdop::refit_tree<V, K, T>(tb, b.mesh, b.X, b.Y, b.Z, kdop::sequential());
  kdop::cuda tag(ctx);
  kdop::refit_tree<V, K, T>(ta_cuda, a.mesh, a.X, a.Y, a.Z, tag);
  kdop::refit_tree<V, K, T>(tb_cuda, b.mesh, b.X, b.Y, b.Z, tag);
  int bad = 0;
  for (int w = 0; w < 2; ++w) {
    kdop::SubTree<T, K> const& s1 = (w ? tb : ta).branches()[0];
    kdop::SubTree<T, K> const& s2 = (w ? tb_cuda : ta_cuda).branches()[0];
    for (size_t i = 0; i < s1.m_nodes.size(); ++i) {
      if (s1.m_nodes[i].is_undefined()) continue;
      for (size_t k = 0; k < K / 2; ++k)
        if (std::memcmp(&s1.m_nodes[i].m_volume(k), &s2.m_nodes[i].m_volume(k), sizeof(geometry::Interval<T>)))
          ++bad;
    }
  }

  // traversal + contacts: sequential vs cuda, through the callbacks
  Rows r_seq, r_cuda;
  std::vector<kdop::TestPair<V, K, T> > pool_seq, pool_cuda;
  pool_seq.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf,
                                             r_seq));
  pool_cuda.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf,
                                              r_cuda));
  kdop::tandem_traversal<V, K, T>(pool_seq, kdop::sequential());
  kdop::tandem_traversal<V, K, T>(pool_cuda, tag);
  bool same = r_seq.sorted() == r_cuda.sorted();
  std::printf("K=%d n=%d: %d volume mismatches, contacts %zu (reference) vs %zu (cuda), %s\n", (int)K, n, bad,
              r_seq.bits.size() / 7, r_cuda.bits.size() / 7, same ? "identical" : "DIFFERENT");
  return (bad == 0 && same && !r_seq.bits.empty()) ? 0 : 1;
}

int main() {
  kdop_ctx* ctx = 0;
  int rc = kdop_ctx_create(0, &ctx);
  if (rc != KDOP_OK) {
    std::printf("kdop_ctx_create failed: %s\n", kdop_status_string(rc));
    return 2;
  }
  int fails = 0;
  fails += run<14>(ctx, 4, 0.3f, 0.05f);
  fails += run<26>(ctx, 5, 0.2f, 0.08f);
  fails += run<8>(ctx, 3, 0.4f, 0.03f);
  kdop_ctx_destroy(ctx);
  std::printf(fails ? "FAIL\n" : "OK\n");
  return fails ? 1 : 0;
}
