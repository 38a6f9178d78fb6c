// adapter_check.cpp -- TEST INFRASTRUCTURE: the reference's own narrow-phase
// calls run once with kdop::sequential and once with the kdop::cuda tag of
// include/kdop_cuda_tag.hpp (the drop-in binding), on the same meshes.
// Exits 0 when the GPU back-end reproduces the reference: refitted node
// volumes bit for bit and the contacts reported through each pair's
// ContactsCallback as the same multiset of (p, n, d) bit patterns.
//
// Built by `make -C oracle adapter` against the reference's headers and
// libkdop_cuda.so; run by tests/test_gpu_adapter.py on a GPU.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
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

// Bitwise comparison of every defined node volume of every chunk level and of
// the root kDOP.
template <size_t K>
static int volume_mismatches(kdop::Tree<T, K> const& a, kdop::Tree<T, K> const& b) {
  int bad = 0;
  if (a.number_of_levels() != b.number_of_levels()) return 1 << 20;
  for (size_t h = 0; h < a.number_of_levels(); ++h) {
    std::vector<kdop::SubTree<T, K> > const& la = a.super_chunks(h);
    std::vector<kdop::SubTree<T, K> > const& lb = b.super_chunks(h);
    if (la.size() != lb.size()) return 1 << 20;
    for (size_t c = 0; c < la.size(); ++c)
      for (size_t i = 0; i < la[c].m_nodes.size(); ++i) {
        if (la[c].m_nodes[i].is_undefined()) continue;
        for (size_t k = 0; k < K / 2; ++k)
          if (std::memcmp(&la[c].m_nodes[i].m_volume(k), &lb[c].m_nodes[i].m_volume(k), sizeof(geometry::Interval<T>)))
            ++bad;
      }
  }
  for (size_t k = 0; k < K / 2; ++k)
    if (std::memcmp(&a.m_root(k), &b.m_root(k), sizeof(geometry::Interval<T>))) ++bad;
  return bad;
}

// make_tree with mem_bytes (SIZE_MAX: one chunk; 8000: the narrow phase's
// default chunked tree), then `steps` simulation steps in which body B moves:
// refit_tree and tandem_traversal once with kdop::sequential and once with
// the kdop::cuda tag (whose device scenes persist between the steps).
template <size_t K>
static int run(kdop_ctx* ctx, int n, float pen, float angle, size_t mem_bytes, int steps) {
  Body a, b;
  lattice(a, n);
  lattice(b, n);
  kdop::Tree<T, K> ta = kdop::make_tree<V, K, T>(mem_bytes, a.mesh, a.X0, a.Y0, a.Z0, kdop::sequential());
  kdop::Tree<T, K> tb = kdop::make_tree<V, K, T>(mem_bytes, b.mesh, b.X0, b.Y0, b.Z0, kdop::sequential());
  kdop::Tree<T, K> ta_cuda = ta, tb_cuda = tb;
  MT::quaternion_type qa(1.f, 0.f, 0.f, 0.f);
  float s = std::sin(angle / 2), c = std::cos(angle / 2);
  MT::quaternion_type qb(c, s * 0.267f, s * 0.535f, s * 0.802f);
  kdop::cuda tag(ctx);
  int fails = 0;
  for (int step = 0; step < steps; ++step) {
    pose(a, qa, V::make(0.f, 0.f, 0.f));
    pose(b, qb, V::make((float)n - pen - 0.05f * (float)step, 0.02f * (float)step, 0.f));
    // refit: sequential vs cuda, every node volume of every level bit for bit
    kdop::refit_tree<V, K, T>(ta, a.mesh, a.X, a.Y, a.Z, kdop::sequential());
    kdop::refit_tree<V, K, T>(tb, b.mesh, b.X, b.Y, b.Z, kdop::sequential());
    kdop::refit_tree<V, K, T>(ta_cuda, a.mesh, a.X, a.Y, a.Z, tag);
    kdop::refit_tree<V, K, T>(tb_cuda, b.mesh, b.X, b.Y, b.Z, tag);
    int bad = volume_mismatches<K>(ta, ta_cuda) + volume_mismatches<K>(tb, tb_cuda);

    // traversal + contacts: sequential vs cuda, through the callbacks
    Rows r_seq, r_cuda;
    std::vector<kdop::TestPair<V, K, T> > pool_seq, pool_cuda;
    pool_seq.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf,
                                               r_seq));
    pool_cuda.push_back(kdop::TestPair<V, K, T>(ta_cuda, tb_cuda, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z,
                                                a.surf, b.surf, r_cuda));
    kdop::tandem_traversal<V, K, T>(pool_seq, kdop::sequential());
    kdop::tandem_traversal<V, K, T>(pool_cuda, tag);
    bool same = r_seq.sorted() == r_cuda.sorted();
    std::printf("K=%d n=%d %s (%zu levels, %zu chunks) step %d: %d volume mismatches, contacts %zu (reference) vs "
                "%zu (cuda), %s\n",
                (int)K, n, mem_bytes == (size_t)-1 ? "one chunk" : "chunked", ta.number_of_levels(),
                ta.branches().size(), step, bad, r_seq.bits.size() / 7, r_cuda.bits.size() / 7,
                same ? "identical" : "DIFFERENT");
    if (!(bad == 0 && same && !r_seq.bits.empty())) ++fails;
  }
  return fails;
}

// Pools whose mesh sets change between steps: bodies A, B, C (chunked
// trees); the pool holds {A-B, A-C} (A shared: one device mesh for it), then
// {A-B}, then {A-B, A-C} again (the tag's cached scene of the first pool is
// reused).  Each pair's callback must receive the sequential back-end's
// contacts.
template <size_t K>
static int run_pools(kdop_ctx* ctx, int n) {
  Body a, b, c;
  lattice(a, n);
  lattice(b, n);
  lattice(c, n);
  kdop::Tree<T, K> ta = kdop::make_tree<V, K, T>(8000, a.mesh, a.X0, a.Y0, a.Z0, kdop::sequential());
  kdop::Tree<T, K> tb = kdop::make_tree<V, K, T>(8000, b.mesh, b.X0, b.Y0, b.Z0, kdop::sequential());
  kdop::Tree<T, K> tc = kdop::make_tree<V, K, T>(8000, c.mesh, c.X0, c.Y0, c.Z0, kdop::sequential());
  MT::quaternion_type q0(1.f, 0.f, 0.f, 0.f), qb(0.9998f, 0.0053f, 0.0107f, 0.016f),
      qc(0.9997f, -0.012f, 0.0081f, 0.02f);
  kdop::cuda tag(ctx);
  int fails = 0;
  const int pools[3] = {2, 1, 2};
  for (int step = 0; step < 3; ++step) {
    pose(a, q0, V::make(0.f, 0.f, 0.f));
    pose(b, qb, V::make((float)n - 0.3f - 0.05f * (float)step, 0.f, 0.f));
    pose(c, qc, V::make(0.f, (float)n - 0.25f, 0.02f * (float)step));
    kdop::refit_tree<V, K, T>(ta, a.mesh, a.X, a.Y, a.Z, kdop::sequential());
    kdop::refit_tree<V, K, T>(tb, b.mesh, b.X, b.Y, b.Z, kdop::sequential());
    kdop::refit_tree<V, K, T>(tc, c.mesh, c.X, c.Y, c.Z, kdop::sequential());
    Rows seq[2], gpu[2];
    std::vector<kdop::TestPair<V, K, T> > ps, pg;
    ps.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf, seq[0]));
    pg.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf, gpu[0]));
    if (pools[step] == 2) {
      ps.push_back(kdop::TestPair<V, K, T>(ta, tc, a.mesh, c.mesh, a.X, c.X, a.Y, c.Y, a.Z, c.Z, a.surf, c.surf,
                                           seq[1]));
      pg.push_back(kdop::TestPair<V, K, T>(ta, tc, a.mesh, c.mesh, a.X, c.X, a.Y, c.Y, a.Z, c.Z, a.surf, c.surf,
                                           gpu[1]));
    }
    kdop::tandem_traversal<V, K, T>(ps, kdop::sequential());
    kdop::tandem_traversal<V, K, T>(pg, tag);
    for (int i = 0; i < pools[step]; ++i) {
      bool same = seq[i].sorted() == gpu[i].sorted() && !seq[i].bits.empty();
      std::printf("K=%d n=%d pool of %d pairs, step %d, pair %d: contacts %zu (reference) vs %zu (cuda), %s\n",
                  (int)K, n, pools[step], step, i, seq[i].bits.size() / 7, gpu[i].bits.size() / 7,
                  same ? "identical" : "DIFFERENT");
      if (!same) ++fails;
    }
  }
  return fails;
}

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Times `steps` narrow-phase steps of two n^3-cell bodies with the default
// chunked trees (8000 bytes, narrow_object.h:113-128): pose of B, refit_tree
// of both bodies, tandem_traversal with contacts; once with kdop::sequential
// and once with the kdop::cuda tag.  Prints milliseconds per step.
template <size_t K>
static int time_loop(kdop_ctx* ctx, int n, int steps) {
  Body a, b;
  lattice(a, n);
  lattice(b, n);
  kdop::Tree<T, K> ta = kdop::make_tree<V, K, T>(8000, a.mesh, a.X0, a.Y0, a.Z0, kdop::sequential());
  kdop::Tree<T, K> tb = kdop::make_tree<V, K, T>(8000, b.mesh, b.X0, b.Y0, b.Z0, kdop::sequential());
  MT::quaternion_type qa(1.f, 0.f, 0.f, 0.f), qb(0.9998f, 0.0053f, 0.0107f, 0.016f);
  pose(a, qa, V::make(0.f, 0.f, 0.f));
  kdop::cuda tag(ctx);
  size_t contacts[2] = {0, 0};
  double ms[2];
  for (int backend = 0; backend < 2; ++backend) {
    // one untimed step (the tag's scenes are created in it), then the loop
    double t0 = 0;
    for (int step = -1; step < steps; ++step) {
      if (step == 0) t0 = now_ms();
      pose(b, qb, V::make((float)n - 0.3f - 0.001f * (float)step, 0.f, 0.f));
      Rows r;
      std::vector<kdop::TestPair<V, K, T> > pool;
      pool.push_back(kdop::TestPair<V, K, T>(ta, tb, a.mesh, b.mesh, a.X, b.X, a.Y, b.Y, a.Z, b.Z, a.surf, b.surf, r));
      if (backend == 0) {
        kdop::refit_tree<V, K, T>(ta, a.mesh, a.X, a.Y, a.Z, kdop::sequential());
        kdop::refit_tree<V, K, T>(tb, b.mesh, b.X, b.Y, b.Z, kdop::sequential());
        kdop::tandem_traversal<V, K, T>(pool, kdop::sequential());
      } else {
        kdop::refit_tree<V, K, T>(ta, a.mesh, a.X, a.Y, a.Z, tag);
        kdop::refit_tree<V, K, T>(tb, b.mesh, b.X, b.Y, b.Z, tag);
        kdop::tandem_traversal<V, K, T>(pool, tag);
      }
      contacts[backend] += r.bits.size() / 7;
    }
    ms[backend] = (now_ms() - t0) / steps;
  }
  std::printf("loop K=%d n=%d (%zu tets per body, %zu chunks): %d steps, sequential %.3f ms/step, "
              "kdop::cuda %.3f ms/step, contacts %zu vs %zu\n",
              (int)K, n, a.mesh.tetrahedron_size(), ta.branches().size(), steps, ms[0], ms[1], contacts[0],
              contacts[1]);
  return contacts[0] == contacts[1] && contacts[0] > 0 ? 0 : 1;
}

int main(int argc, char** argv) {
  kdop_ctx* ctx = 0;
  int rc = kdop_ctx_create(0, &ctx);
  if (rc != KDOP_OK) {
    std::printf("kdop_ctx_create failed: %s\n", kdop_status_string(rc));
    return 2;
  }
  int fails = 0;
  if (argc > 1 && std::strcmp(argv[1], "--time") == 0) {
    int steps = argc > 2 ? std::atoi(argv[2]) : 100;
    int n = argc > 3 ? std::atoi(argv[3]) : 16;
    fails += time_loop<8>(ctx, n, steps);
  } else {
    const size_t one = (size_t)-1;
    fails += run<14>(ctx, 4, 0.3f, 0.05f, one, 2);
    fails += run<26>(ctx, 5, 0.2f, 0.08f, one, 1);
    fails += run<8>(ctx, 3, 0.4f, 0.03f, one, 1);
    // the narrow phase's default 8000-byte chunks: several branches, a super
    // chunk level above them at n = 12 (K = 8: 2 levels)
    fails += run<8>(ctx, 6, 0.4f, 0.03f, 8000, 3);
    fails += run<8>(ctx, 12, 0.3f, 0.02f, 8000, 2);
    fails += run<14>(ctx, 8, 0.3f, 0.04f, 8000, 2);
    fails += run_pools<8>(ctx, 6);
  }
  kdop::cuda_release(ctx);
  kdop_ctx_destroy(ctx);
  std::printf(fails ? "FAIL\n" : "OK\n");
  return fails ? 1 : 0;
}
