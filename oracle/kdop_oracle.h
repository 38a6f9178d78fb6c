/*
 * kdop_oracle.h -- CPU restatement of the reference's kDOP collision path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA library is compared
 * against.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py load it; the product library never links or calls it.
 *
 * Parity pin: every function here is checked against the reference's own
 * code, compiled from its sources into oracle/_ref/ (oracle/ref_harness.cpp),
 * and against the fixtures in tests/golden/ generated from it.
 *
 * Conventions shared with the CUDA library:
 *   - vertices are xyz triples (float), tets are 4 vertex indices (uint32),
 *   - a kDOP of K faces is K/2 slabs stored as (lo, hi) pairs, slab order =
 *     direction-table order,
 *   - surface flags: bit v of surf[t] set <=> the face opposite local vertex v
 *     of tet t lies on the mesh boundary.
 * Suffix _f = single precision (the reference's FP32 path), _d = double.
 */
#ifndef KDOP_ORACLE_H
#define KDOP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Number of contact-candidate descriptors per tet pair (8 vertex tests +
 * 6 edges x 4 planes x 2 directions). */
#define OR_NCAND 56

typedef struct {
  int32_t face_a;  /* face of A whose normal is the contact normal, -1: none */
  int32_t face_b;  /* opposing face of B chosen together with face_a */
  int32_t imin;    /* candidate code (0..55) attaining min p.n */
  int32_t imax;    /* candidate code attaining max p.n */
  int32_t ncontacts; /* unique contacts reported */
  int32_t overlap; /* exact tet-tet SAT overlap */
  uint64_t cand_mask; /* bit c set: contact candidate c was generated */
} or_record;

int or_dirs_f(int K, float* out);
int or_dirs_d(int K, double* out);

void or_leaf_dops_f(int K, const float* xyz, int64_t nt, const uint32_t* tets, float* out);
void or_leaf_dops_d(int K, const float* xyz, int64_t nt, const uint32_t* tets, double* out);

/* Morton order of kdop_mesh_reorder.h:173-353: perm[i] = caller's tet index
 * placed at position i.  Ties (equal codes) resolve by tet index. */
int or_morton_order(const float* xyz, int64_t nv, int64_t nt, const uint32_t* tets, uint32_t* perm);

/* Median-split tree of kdop_make_tree.h:58-121 over perm (one chunk).  Nodes in
 * preorder; left[i] = index of left child (right = the next subtree), or -1 for
 * a leaf whose tet is tet[i].  Returns the node count (2 nt - 1). */
int64_t or_build_tree(int64_t nt, const uint32_t* perm, int64_t* left, int64_t* right, int64_t* tet);

/* Bottom-up refit (kdop_refit_tree.h:24-115): vol[node*K + 2s + {0,1}]. */
void or_refit_f(int K, const float* xyz, const uint32_t* tets, int64_t nnodes, const int64_t* left,
                const int64_t* right, const int64_t* tet, float* vol);

/* Tandem traversal (kdop_tandem_traversal.h:19-157) from the two roots,
 * after the root test of :164.  Surface-filtered leaf pairs (A tet, B tet) are
 * written in traversal order.  *tests counts overlap_dop_dop calls including
 * the root test; *leaf_overlaps counts overlapping leaf pairs before the
 * surface filter.  Returns 0, or -1 when cap is exceeded (counts stay exact). */
int or_traverse_f(int K, const float* volA, const int64_t* leftA, const int64_t* rightA, const int64_t* tetA,
                  const uint8_t* surfA, const float* volB, const int64_t* leftB, const int64_t* rightB,
                  const int64_t* tetB, const uint8_t* surfB, int64_t cap, uint32_t* out_pairs,
                  int64_t* npairs, int64_t* tests, int64_t* leaf_overlaps);

/* One mesh pair end to end: Morton order and tree build on the rest
 * positions restA/restB (NULL: the world positions), refit on the world
 * positions xyzA/xyzB, traversal. */
int or_run_pair_f(int K, int64_t nvA, const float* xyzA, const float* restA, int64_t ntA, const uint32_t* tetsA,
                  const uint8_t* surfA, int64_t nvB, const float* xyzB, const float* restB, int64_t ntB,
                  const uint32_t* tetsB, const uint8_t* surfB, int64_t cap, uint32_t* out_pairs, int64_t* npairs,
                  int64_t* tests, int64_t* leaf_overlaps);

/* Many independent mesh pairs with a thread pool (threads <= 0: all cores).
 * Meshes are concatenated: vertices xyz[v_off[m]..v_off[m+1]), tets likewise
 * with mesh-local vertex indices; rest (or NULL) gives the tree-building
 * positions.  out_pairs rows are (pair, a, b). */
int or_run_pairs_f(int K, int n_meshes, const int64_t* v_off, const float* xyz, const float* rest, const int64_t* t_off,
                   const uint32_t* tets, const uint8_t* surf, int64_t n_pairs, const uint32_t* pairs,
                   int threads, int64_t cap, uint32_t* out_pairs, int64_t* npairs, int64_t* tests_per_pair,
                   int64_t* pairs_per_pair);

/* Face-adjacency surface map (mesh_array_compute_surface_map.h:41-76). */
int or_surface_map(int64_t nv, int64_t nt, const uint32_t* tets, uint8_t* surf);

/* Contacts of the MOST_OPPOSING_SURFACES algorithm
 * (geometry_contacts_tetrahedron_tetrahedron.h:1313-1345) for explicit tet
 * pairs.  Rows of out: p.xyz, n.xyz, depth, pair index.  rec (optional) gets
 * one decision record per pair. */
int or_contacts_f(const float* xyzA, const uint32_t* tetsA, const uint8_t* surfA, const float* xyzB,
                  const uint32_t* tetsB, const uint8_t* surfB, int64_t n_pairs, const uint32_t* pairs,
                  int64_t cap, float* out, int64_t* n_out, or_record* rec);
int or_contacts_d(const float* xyzA, const uint32_t* tetsA, const uint8_t* surfA, const float* xyzB,
                  const uint32_t* tetsB, const uint8_t* surfB, int64_t n_pairs, const uint32_t* pairs,
                  int64_t cap, double* out, int64_t* n_out, or_record* rec);
/* Same, vertex positions given in double. */
int or_contacts_dd(const double* xyzA, const uint32_t* tetsA, const uint8_t* surfA, const double* xyzB,
                   const uint32_t* tetsB, const uint8_t* surfB, int64_t n_pairs, const uint32_t* pairs,
                   int64_t cap, double* out, int64_t* n_out, or_record* rec);

/* Depth of a pair with its discrete decisions frozen to rec (double), and the
 * gradient of  gd*depth + gn.n  with respect to the 8 vertices
 * (A0..A3, B0..B3, xyz each) into g24. */
double or_frozen_depth_d(const double* a12, const double* b12, const or_record* rec, double* n_out);
void or_depth_grad_d(const double* a12, const double* b12, const or_record* rec, double gd, const double* gn,
                     double* g24);

/* Batched forms of the two above over n pairs (a12/b12: n x 12, gd: n,
 * gn: n x 3, g24: n x 24, normal: n x 3 or NULL). */
void or_frozen_batch_d(int64_t n, const double* a12, const double* b12, const or_record* rec, double* depth,
                       double* normal);
void or_depth_grad_batch_d(int64_t n, const double* a12, const double* b12, const or_record* rec, const double* gd,
                           const double* gn, double* g24);

/* tiny::rotate(q, r) + p with q = (w, x, y, z) (tiny_quaternion_functions.h:149-152). */
void or_rotate_f(const float* q, const float* p, int64_t nv, const float* xyz, float* out);

/* Deformation of the deforming benchmark: x + a*sin(w*(x+y+z) + phase) on all
 * three coordinates, with the project's own sine (or_sin_f). */
float or_sin_f(float x);
void or_deform_f(float amp, float w, float phase, int64_t nv, const float* xyz, float* out);

#ifdef __cplusplus
}
#endif
#endif
