// kdop_build.cpp -- host-side construction of the scene's kDOP trees.
//
// The topology equals the reference's one-chunk tree (make_tree with
// mem_bytes = SIZE_MAX, SIMULATION/KDOP/KDOP/include/kdop_make_tree.h:191-288)
// built over the Morton-reordered mesh (kdop_mesh_reorder.h:173-353): leaves
// are single tets in Morton order of their centroids and every internal node
// splits its tet range at the index median floor((first + last) / 2)
// (kdop_make_tree.h:85).  Only the storage differs: all trees of a scene form
// one forest laid out level by level (breadth first, level d of every tree
// contiguous, trees in mesh order), so the refit can sweep whole levels with
// coalesced accesses and the two children of a node are adjacent.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

#include "kdop_internal.h"

namespace kdop {

// Unit direction tables of geometry_direction_table.h:54-176, computed with the
// same float operations as tiny's unit() (v * (1 / sqrt(v . v))).
static void put_dir(float* o, int i, float x, float y, float z, bool normalise) {
  if (normalise) {
    float d = 0.0f;
    d = d + x * x;
    d = d + y * y;
    d = d + z * z;
    float l = std::sqrt(d);
    if (l > 0.0f) {
      float inv = 1.0f / l;
      x = x * inv;
      y = y * inv;
      z = z * inv;
    }
  }
  o[3 * i] = x;
  o[3 * i + 1] = y;
  o[3 * i + 2] = z;
}
static int dirs3(float* o, int at) {
  put_dir(o, at, 1, 0, 0, false);
  put_dir(o, at + 1, 0, 1, 0, false);
  put_dir(o, at + 2, 0, 0, 1, false);
  return at + 3;
}
static int dirs4(float* o, int at) {
  put_dir(o, at, 1, 1, 1, true);
  put_dir(o, at + 1, 1, 1, -1, true);
  put_dir(o, at + 2, 1, -1, 1, true);
  put_dir(o, at + 3, 1, -1, -1, true);
  return at + 4;
}
static int dirs6(float* o, int at) {
  put_dir(o, at, 1, 1, 0, true);
  put_dir(o, at + 1, 1, -1, 0, true);
  put_dir(o, at + 2, 1, 0, 1, true);
  put_dir(o, at + 3, 0, 1, 1, true);
  put_dir(o, at + 4, -1, 0, 1, true);
  put_dir(o, at + 5, 0, -1, 1, true);
  return at + 6;
}

int direction_table(int K, float* o) {
  switch (K) {
    case 6: return dirs3(o, 0);
    case 8: return dirs4(o, 0);
    case 12: return dirs6(o, 0);
    case 14: return dirs4(o, dirs3(o, 0));
    case 18: return dirs6(o, dirs3(o, 0));
    case 20: return dirs6(o, dirs4(o, 0));
    case 26: return dirs6(o, dirs4(o, dirs3(o, 0)));
  }
  return -1;
}

// The integer scale of kdop_mesh_reorder.h's quantisation: min over the
// three axes of (int)((float)(2^21 - 1) / (max - min)).  Returns false when a
// quotient is not finite or beyond int range (the reference converts it
// anyway; the host then keeps whatever its own conversion gives).
bool morton_scale(const float* mn, const float* mx, int& scale) {
  const int KB = (int)(sizeof(unsigned long long) * 8) / 3;
  bool ok = true;
  for (int d = 0; d < 3; ++d) {
    float q = (float)((1 << KB) - 1) / (mx[d] - mn[d]);
    if (!(q < 2147483520.0f && q > -2147483520.0f)) ok = false;
    int v = (int)q;
    scale = d == 0 ? v : std::min(scale, v);
  }
  return ok;
}

// Morton order of kdop_mesh_reorder.h:173-353, with its arithmetic: float
// centroid sums scaled by the double 0.25, 21-bit quantisation with an integer
// scale, the initial maximum numeric_limits<float>::min(), and std::sort on the
// codes (whose order of equal codes is what the reference's std::sort gives).
void morton_order(const float* xyz, int64_t nt, const uint32_t* tets, std::vector<uint32_t>& perm) {
  perm.resize(nt);
  if (nt <= 0) return;
  std::vector<float> c(3 * (size_t)nt);
  float mn[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
                 std::numeric_limits<float>::max()};
  float mx[3] = {std::numeric_limits<float>::min(), std::numeric_limits<float>::min(),
                 std::numeric_limits<float>::min()};
  for (int64_t t = 0; t < nt; ++t) {
    const uint32_t* q = tets + 4 * t;
    for (int d = 0; d < 3; ++d) {
      float s = xyz[3 * (size_t)q[0] + d] + xyz[3 * (size_t)q[1] + d];
      s = s + xyz[3 * (size_t)q[2] + d];
      s = s + xyz[3 * (size_t)q[3] + d];
      float v = (float)(0.25 * (double)s);
      c[3 * t + d] = v;
      mn[d] = std::min(mn[d], v);
      mx[d] = std::max(mx[d], v);
    }
  }
  const int KB = (int)(sizeof(unsigned long long) * 8) / 3;
  int scale = 0;
  morton_scale(mn, mx, scale);
  std::vector<std::pair<uint32_t, unsigned long long> > mc((size_t)nt);
  for (int64_t t = 0; t < nt; ++t) {
    unsigned long long x = (unsigned long long)(float)(int)((c[3 * t + 0] - mn[0]) * (float)scale);
    unsigned long long y = (unsigned long long)(float)(int)((c[3 * t + 1] - mn[1]) * (float)scale);
    unsigned long long z = (unsigned long long)(float)(int)((c[3 * t + 2] - mn[2]) * (float)scale);
    unsigned long long code = 0;
    for (unsigned long k = 0; k < (unsigned long)KB; ++k) {
      code |= ((x >> k) & 1ull) << (3 * k);
      code |= ((y >> k) & 1ull) << (3 * k + 1);
      code |= ((z >> k) & 1ull) << (3 * k + 2);
    }
    mc[(size_t)t] = std::make_pair((uint32_t)t, code);
  }
  std::sort(mc.begin(), mc.end(),
            [](const std::pair<uint32_t, unsigned long long>& a, const std::pair<uint32_t, unsigned long long>& b) {
              return a.second < b.second;
            });
  for (int64_t t = 0; t < nt; ++t) perm[(size_t)t] = mc[(size_t)t].first;
}

// Boundary faces by face counting (mesh_array_compute_surface_map.h:41-76):
// the face opposite local vertex v is on the boundary iff no other tet has
// the same three vertices.
void surface_map(int64_t nt, const uint32_t* tets, uint8_t* surf) {
  struct Face {
    uint32_t a, b, c;
    uint32_t tf;  // tet * 4 + face
  };
  std::vector<Face> f(4 * (size_t)nt);
  for (int64_t t = 0; t < nt; ++t) {
    surf[t] = 0;
    for (int k = 0; k < 4; ++k) {
      uint32_t v[3];
      int n = 0;
      for (int i = 0; i < 4; ++i)
        if (i != k) v[n++] = tets[4 * t + i];
      std::sort(v, v + 3);
      f[4 * t + k] = Face{v[0], v[1], v[2], (uint32_t)(4 * t + k)};
    }
  }
  std::sort(f.begin(), f.end(), [](const Face& x, const Face& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.c < y.c;
  });
  size_t i = 0, n = f.size();
  while (i < n) {
    size_t j = i + 1;
    while (j < n && f[j].a == f[i].a && f[j].b == f[i].b && f[j].c == f[i].c) ++j;
    if (j - i == 1) surf[f[i].tf >> 2] |= (uint8_t)(1u << (f[i].tf & 3));
    i = j;
  }
}

namespace {
struct TreeLevels {
  std::vector<uint32_t> perm;
  std::vector<std::vector<std::pair<uint32_t, uint32_t> > > levels;  // (first, last) per node
};

void build_levels(const float* xyz, int64_t nt, const uint32_t* tets, const uint32_t* order, TreeLevels& tl) {
  if (order)
    tl.perm.assign(order, order + nt);
  else
    morton_order(xyz, nt, tets, tl.perm);
  tl.levels.clear();
  if (nt <= 0) return;
  std::vector<std::pair<uint32_t, uint32_t> > cur(1, std::make_pair(0u, (uint32_t)(nt - 1)));
  while (!cur.empty()) {
    std::vector<std::pair<uint32_t, uint32_t> > nxt;
    for (size_t i = 0; i < cur.size(); ++i) {
      uint32_t first = cur[i].first, last = cur[i].second;
      if (last > first) {
        // kdop_make_tree.h:85: mid = floor((first + last) / 2)
        uint32_t mid = (uint32_t)std::floor(((double)first + (double)last) / 2.0);
        nxt.push_back(std::make_pair(first, mid));
        nxt.push_back(std::make_pair(mid + 1, last));
      }
    }
    tl.levels.push_back(std::move(cur));
    cur = std::move(nxt);
  }
}

}  // namespace

int build_forest(const std::vector<const float*>& xyz, const std::vector<int64_t>& n_verts,
                 const std::vector<const uint32_t*>& tets, const std::vector<int64_t>& n_tets,
                 const std::vector<const uint32_t*>& orders, const std::vector<int64_t>& t_off, ForestBuild& out) {
  (void)n_verts;
  int nm = (int)tets.size();
  std::vector<TreeLevels> trees((size_t)nm);
  parallel_for(nm, [&](int m) { build_levels(xyz[m], n_tets[m], tets[m], orders[m], trees[m]); });
  int depth = 0;
  for (int m = 0; m < nm; ++m) depth = std::max(depth, (int)trees[m].levels.size());
  // pre[m][d]: nodes of trees < m at level d
  std::vector<std::vector<int64_t> > pre((size_t)nm, std::vector<int64_t>((size_t)depth + 1, 0));
  out.level_off.assign((size_t)depth + 1, 0);
  std::vector<int64_t> tot((size_t)depth, 0);
  for (int d = 0; d < depth; ++d) {
    int64_t acc = 0;
    for (int m = 0; m < nm; ++m) {
      pre[m][d] = acc;
      if (d < (int)trees[m].levels.size()) acc += (int64_t)trees[m].levels[d].size();
    }
    tot[d] = acc;
  }
  // Twin records need every sibling pair at an even index: levels >= 1 hold
  // whole sibling pairs, so an even root level suffices (one padding node,
  // a copy of the first root's topology, when the count is odd).
  const int64_t n_roots = depth > 0 ? tot[0] : 0;
  if (n_roots & 1) tot[0] += 1;
  for (int d = 0; d < depth; ++d) out.level_off[d + 1] = out.level_off[d] + tot[d];
  int64_t nn = out.level_off[depth];
  if (nn >= (int64_t)(LEAF_BIT_HOST >> 1)) return -1;  // node indices use 30 bits
  out.topo.assign(2 * (size_t)nn, 0);
  out.root.assign((size_t)nm, 0xFFFFFFFFu);
  out.depth = depth > 0 ? depth - 1 : 0;
  parallel_for(nm, [&](int m) {
    TreeLevels& tl = trees[m];
    if (tl.levels.empty()) return;
    out.root[m] = (uint32_t)(out.level_off[0] + pre[m][0]);
    for (size_t d = 0; d < tl.levels.size(); ++d) {
      int64_t base = out.level_off[d] + pre[m][d];
      int64_t child = (d + 1 < tl.levels.size()) ? out.level_off[d + 1] + pre[m][d + 1] : 0;
      const std::vector<std::pair<uint32_t, uint32_t> >& L = tl.levels[d];
      for (size_t i = 0; i < L.size(); ++i) {
        uint32_t* tp = &out.topo[2 * (size_t)(base + (int64_t)i)];
        if (L[i].second > L[i].first) {
          tp[0] = (uint32_t)child;
          tp[1] = (uint32_t)(child + 1);
          child += 2;
        } else {
          uint32_t t = (uint32_t)(t_off[m] + tl.perm[L[i].first]);
          tp[0] = t;
          tp[1] = t;
        }
      }
    }
    std::vector<uint32_t>().swap(tl.perm);
    std::vector<std::vector<std::pair<uint32_t, uint32_t> > >().swap(tl.levels);
  });
  if (n_roots & 1) {
    // the padding slot ending the root level repeats the first root's
    // topology (refitted like it, never reached by a traversal)
    out.topo[2 * (size_t)n_roots] = out.topo[0];
    out.topo[2 * (size_t)n_roots + 1] = out.topo[1];
  }
  return 0;
}

// Level layout of the forest from the tet counts alone.  The index-median
// split halves a range into ceil(s/2), floor(s/2), so the sizes at depth d
// are floor or ceil of n / 2^d: depths 0 .. L = floor(log2 n) are complete
// (2^d nodes) and depth L + 1 holds the 2 (n - 2^L) children of the size-2
// nodes of depth L.  pre[d * (nm + 1) + m] = nodes of trees < m at level d.
int forest_layout(const std::vector<int64_t>& n_tets, ForestBuild& out, std::vector<int64_t>& pre,
                  std::vector<int32_t>& lg) {
  const int nm = (int)n_tets.size();
  lg.assign((size_t)nm, -1);
  int levels = 0;
  for (int m = 0; m < nm; ++m) {
    int64_t n = n_tets[m];
    if (n <= 0) continue;
    int L = 0;
    while ((int64_t(1) << (L + 1)) <= n) ++L;
    lg[m] = L;
    levels = std::max(levels, L + 1 + ((int64_t(1) << L) < n ? 1 : 0));
  }
  auto count = [&](int m, int d) -> int64_t {
    int L = lg[m];
    if (L < 0) return 0;
    if (d <= L) return int64_t(1) << d;
    if (d == L + 1) return 2 * (n_tets[m] - (int64_t(1) << L));
    return 0;
  };
  pre.assign((size_t)levels * (nm + 1), 0);
  std::vector<int64_t> tot((size_t)levels, 0);
  for (int d = 0; d < levels; ++d) {
    int64_t acc = 0;
    for (int m = 0; m < nm; ++m) {
      pre[(size_t)d * (nm + 1) + m] = acc;
      acc += count(m, d);
    }
    pre[(size_t)d * (nm + 1) + nm] = acc;
    tot[d] = acc;
  }
  if (levels > 0 && (tot[0] & 1)) tot[0] += 1;  // even root level (twin records)
  out.level_off.assign((size_t)levels + 1, 0);
  for (int d = 0; d < levels; ++d) out.level_off[d + 1] = out.level_off[d] + tot[d];
  if (out.level_off[levels] >= (int64_t)(LEAF_BIT_HOST >> 1)) return -1;
  out.root.assign((size_t)nm, 0xFFFFFFFFu);
  for (int m = 0; m < nm; ++m)
    if (lg[m] >= 0) out.root[m] = (uint32_t)pre[m];
  out.depth = levels > 0 ? levels - 1 : 0;
  out.topo.clear();
  return 0;
}

}  // namespace kdop
