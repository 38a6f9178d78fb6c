/*
 * kdop_cuda.h -- C ABI of the B200 (sm_100a) kDOP BVH collision library.
 *
 * The library stands in for the reference's SIMULATION/KDOP entry points
 * (diku-dk/bvh-tvcg18):
 *
 *   kdop::make_tree<V,K,T>(mem_bytes, mesh, X, Y, Z, sequential)
 *       SIMULATION/KDOP/KDOP/include/kdop_make_tree.h:191-288
 *       preceded by kdop::mesh_reorder (Morton), kdop_mesh_reorder.h:364-387
 *       and mesh_array::compute_surface_map, mesh_array_compute_surface_map.h:41-76
 *         -> kdop_scene_create
 *   kdop::refit_tree<V,K,T>(tree, mesh, X, Y, Z, tag)
 *       kdop_refit_tree.h:120-162 (CPU), cl/kdop_cl_refit_tree.h:53-283 (OpenCL)
 *       with the rigid transform of narrow_update_kdop_bvh.h:154-165 and
 *       narrow_cl_transform_vertices.cl:5-45 done on the device in the same call
 *         -> kdop_set_vertices / kdop_set_poses / kdop_refit
 *   kdop::tandem_traversal<V,K,T>(std::vector<TestPair>&, tag)
 *       kdop_tandem_traversal.h:160-226 (CPU),
 *       cl/kdop_cl_tandem_traversal.h:623-1796 (OpenCL),
 *       cl/gproximity/kdop_cl_gproximity_tandem_traversal.h:164 (work queues)
 *         -> kdop_traverse (candidate tet pairs) + kdop_contacts (contacts)
 *   geometry::ContactsCallback<V>::operator()(p, n, d)
 *       contacts/geometry_contacts_callback.h:8-23
 *         -> rows of kdop_read_contacts
 *
 * Conventions
 *   - A scene owns the device copies of a set of meshes (vertices, tets,
 *     boundary-face map) and one kDOP tree per mesh.  K is one of
 *     6, 8, 12, 14, 18, 20, 26 (the reference's DirectionTableHelper sets).
 *   - Vertices are float xyz triples, tets are 4 mesh-local uint32 vertex
 *     indices with positive orientation, surface[t] bit v set <=> the face
 *     opposite local vertex v of tet t is on the mesh boundary.
 *   - Pointers tagged `memory` are host pointers for KDOP_HOST and device
 *     pointers (on the scene's device) for KDOP_DEVICE.
 *   - Every call returns a kdop_status; nothing aborts the process.  Work is
 *     enqueued on the context's stream; calls that return statistics
 *     synchronise that stream.
 *   - One context per host thread at a time: calls on one context are not
 *     thread-safe.
 */
#ifndef KDOP_CUDA_H
#define KDOP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KDOP_API_VERSION 1

typedef enum {
  KDOP_OK = 0,
  KDOP_ERR_INVALID = -1,  /* bad argument (sizes, K, null pointer, index range) */
  KDOP_ERR_CAPACITY = -2, /* an output or work buffer was too small; the call
                             reports the required size and can be retried */
  KDOP_ERR_CUDA = -3,     /* a CUDA runtime call failed (see kdop_last_error) */
  KDOP_ERR_TIMEOUT = -4,  /* a bounded device-side wait gave up */
  KDOP_ERR_NOMEM = -5,    /* device or host allocation failed */
  KDOP_ERR_STATE = -6     /* call out of order (e.g. contacts before traverse) */
} kdop_status;

typedef enum { KDOP_HOST = 0, KDOP_DEVICE = 1 } kdop_memory;

typedef struct kdop_ctx kdop_ctx;
typedef struct kdop_scene kdop_scene;

int kdop_api_version(void);
const char* kdop_status_string(int status);
/* Message of the last failure on ctx (empty string if none). */
const char* kdop_last_error(const kdop_ctx* ctx);

/* ---- context --------------------------------------------------------------- */
int kdop_ctx_create(int device, kdop_ctx** out);
int kdop_ctx_destroy(kdop_ctx* ctx);
/* cudaStream_t to enqueue on (NULL: the context's own non-blocking stream). */
int kdop_ctx_set_stream(kdop_ctx* ctx, void* cuda_stream);
void* kdop_ctx_stream(const kdop_ctx* ctx);
int kdop_ctx_synchronize(kdop_ctx* ctx);

/* ---- scene: meshes + trees (replaces mesh_reorder + make_tree) ------------ */
typedef struct {
  int64_t n_verts;
  const float* xyz;        /* host, n_verts * 3: rest positions (also the initial world positions) */
  int64_t n_tets;
  const uint32_t* tets;    /* host, n_tets * 4, mesh-local vertex indices */
  const uint8_t* surface;  /* host, n_tets boundary-face bits, or NULL to compute them */
  const uint32_t* leaf_order; /* host, n_tets: the tets in leaf order (a permutation), or
                                 NULL for the Morton order of the rest positions */
} kdop_mesh_desc;

/* Builds one tree per mesh on the host with the reference's topology
 * (Morton order of tet centroids, index-median split, 1 tet per leaf: the
 * one-chunk tree of make_tree with mem_bytes = SIZE_MAX) and uploads meshes
 * and trees.  Leaves keep the caller's tet numbering.  A leaf_order of
 * 0, 1, ..., n_tets-1 reproduces make_tree's tree of a mesh as given (the
 * reference reorders meshes before building, kdop_mesh_reorder.h:364-387). */
int kdop_scene_create(kdop_ctx* ctx, int K, int n_meshes, const kdop_mesh_desc* meshes, kdop_scene** out);

/* Where the trees are built.  Both give the same trees (the reference's
 * make_tree over the Morton-reordered mesh):
 *   KDOP_BUILD_DEVICE (kdop_scene_create's choice): Morton codes and their
 *     sort on the GPU, topology written by one GPU thread per node; a mesh
 *     with equal Morton codes (whose order std::sort leaves to itself) or a
 *     caller-given leaf_order takes its leaf order from the host;
 *   KDOP_BUILD_HOST: everything on the host (std::sort per mesh). */
enum { KDOP_BUILD_DEVICE = 0, KDOP_BUILD_HOST = 1 };
int kdop_scene_create_ex(kdop_ctx* ctx, int K, int n_meshes, const kdop_mesh_desc* meshes, int build,
                         kdop_scene** out);
int kdop_scene_destroy(kdop_scene* scene);

typedef struct {
  int32_t K;
  int32_t n_meshes;
  int64_t n_verts;
  int64_t n_tets;
  int64_t n_nodes;
  int32_t depth;        /* deepest level index over all trees */
  int32_t node_bytes;   /* bytes per node record: 4 K + 8 rounded up to 16 */
  int64_t device_bytes; /* device memory held by the scene */
  int32_t build;        /* KDOP_BUILD_DEVICE or KDOP_BUILD_HOST */
  int32_t host_orders;  /* device build: meshes whose leaf order came from the host */
} kdop_scene_info;
int kdop_scene_get_info(const kdop_scene* scene, kdop_scene_info* info);

/* Node records of the scene's trees in the reference's preorder (node,
 * left subtree, right subtree) for mesh `mesh`: vol[n*K + 2s] = lower,
 * vol[n*K + 2s + 1] = upper of slab s; tet[n] = leaf tet (mesh-local) or -1.
 * Synchronises.  `cap` = room in nodes; *n_nodes gets 2 n_tets - 1. */
int kdop_read_tree(kdop_scene* scene, int mesh, int64_t cap, float* vol, int64_t* tet, int64_t* n_nodes);

/* ---- positions and refit (replaces refit_tree + update_kdop_bvh) ---------- */
/* World positions of all meshes, concatenated in mesh order (n_verts_total*3). */
int kdop_set_vertices(kdop_scene* scene, const float* xyz, int64_t n_verts_total, int memory);
/* Per-mesh rigid pose: quat (w,x,y,z) n_meshes*4, pos n_meshes*3. */
int kdop_set_poses(kdop_scene* scene, const float* quat, const float* pos, int memory);
/* Rest-space displacement applied before the pose in KDOP_REFIT_DEFORM:
 * x += amp * sin(w * (x + y + z) + phase) on all three coordinates. */
int kdop_set_deformation(kdop_scene* scene, float amp, float w, float phase);

typedef enum {
  KDOP_REFIT_VERTICES = 0, /* refit from the world positions of kdop_set_vertices */
  KDOP_REFIT_POSE = 1,     /* world = rotate(q, rest) + p, computed by the refit on the device */
  KDOP_REFIT_DEFORM = 2    /* world = rotate(q, rest + displacement) + p, likewise */
} kdop_refit_mode;
/* Bottom-up refit of every tree of the scene; the mode also fixes how the
 * contact kernels obtain world positions until the next refit. */
int kdop_refit(kdop_scene* scene, int mode);
/* Copies the world positions (n_verts_total*3) to host memory: the
 * kdop_set_vertices positions in KDOP_REFIT_VERTICES mode, else the ones the
 * last pose / deform refit computed (posed with the current poses when the
 * mode was set by a captured graph that has not run yet). */
int kdop_read_vertices(kdop_scene* scene, float* xyz, int64_t cap_verts);

/* ---- tandem traversal (replaces tandem_traversal) ------------------------- */
typedef enum {
  KDOP_TRAVERSE_BATCHED = 0, /* all pairs in one persistent launch with a global work queue */
  KDOP_TRAVERSE_PLAIN = 1    /* one launch per mesh pair */
} kdop_traverse_mode;

typedef struct {
  int32_t mode;           /* kdop_traverse_mode */
  int32_t surface_filter; /* 1: emit only pairs whose tets both have a boundary
                             face (kdop_tandem_traversal.h:56-88); 0: every
                             overlapping leaf pair */
  int32_t block_warps;    /* warps per block (0: tuned default) */
  int32_t stack_cap;      /* node-pair entries per warp stack, power of two (0: default) */
  int32_t init_chunk;     /* root pairs taken per queue claim (0: default) */
  int32_t donate_min;     /* stack size from which a warp gives work to idle warps (0: default) */
  int32_t timeout_ms;     /* bound of every device-side wait (0: 5000) */
  int32_t load_group;     /* expansion shape (0: default 4): 1 = one 32-byte chunk pair per lane
                             and one batch of entries per step, 2 = two batches per step,
                             4 = two chunk pairs per lane (half the lanes per entry),
                             8 = 4 with two batches per step */
  int32_t wave_pairs;     /* pairs per persistent launch, largest first (0: all pairs in one launch) */
  int32_t smem_carveout;  /* shared-memory share of the L1/shared array in percent (0: driver choice) */
  int32_t test_stuck_work; /* test hook, normally 0: this many extra work units that never complete,
                              so every waiting warp gives up after timeout_ms and the call reports
                              KDOP_ERR_TIMEOUT (exercises the bounded waits without a GPU fault) */
} kdop_traverse_opts;

/* Fills opts with the defaults, or with the autotuned choice: the scene's own
 * (kdop_autotune on this scene), else one cached on the scene's context by
 * kdop_autotune on another scene of the same K and size class (floor(log2)
 * of the scene's total tet count). */
int kdop_traverse_opts_default(const kdop_scene* scene, kdop_traverse_opts* opts);

typedef struct {
  int64_t n_pairs;          /* mesh pairs traversed */
  int64_t n_tests;          /* kDOP node-pair tests, counted as the reference
                               counts its overlap_dop_dop calls (root test of
                               :164 included) */
  int64_t n_leaf_overlaps;  /* overlapping leaf pairs before the surface filter */
  int64_t n_candidates;     /* candidate tet pairs emitted */
  int64_t n_contacts;       /* contacts of the last kdop_contacts */
  int64_t candidate_capacity;
  int64_t contact_capacity;
  int64_t queue_capacity;
  int64_t queue_used;       /* work-queue slots used by the last traversal */
  int32_t device_error;     /* bit set of device-side errors (0: none) */
  int32_t reserved;
} kdop_stats;

/* Broad phase (replaces broad::find_overlaps, SIMULATION/BROAD/BROAD/include/
 * broad_find_overlaps.h:44-125; its all-pair and grid algorithms report the
 * same set): the mesh pairs (i, j), i < j, whose boxes overlap, sorted
 * lexicographically -- the pair list kdop_traverse takes.  A mesh's box is
 * its position +- its bounding radius (prox_rigid_body.h:159-172), the radius
 * the largest |rest vertex| (narrow_shape_types.h:189-206); boxes overlap
 * unless one's max is strictly below the other's min on an axis.
 * positions: n_meshes * 3 floats in `memory`, or NULL for the positions of
 * kdop_set_poses.  out_pairs: room for `cap` pairs, host or device memory;
 * *n_pairs = pairs found (KDOP_ERR_CAPACITY when above cap).  Synchronises. */
int kdop_broad_phase(kdop_scene* scene, const float* positions, int memory, uint32_t* out_pairs, int64_t cap,
                     int64_t* n_pairs);

/* Enqueues the traversal of n_pairs mesh pairs (pairs[2i] = mesh A, pairs[2i+1]
 * = mesh B).  Asynchronous: read results with kdop_get_stats.  opts NULL =
 * defaults. */
int kdop_traverse(kdop_scene* scene, int64_t n_pairs, const uint32_t* pairs, int memory,
                  const kdop_traverse_opts* opts);

/* One shard of a traversal, for splitting few large pairs (one huge pair
 * included) over ranks or GPUs.  The node-pair tree of the given pairs is
 * expanded breadth first until at least frontier_min node pairs are pending
 * (the tests and leaf pairs of that expansion count on shard 0); the pending
 * pairs are sorted -- the same list on every rank -- and dealt round-robin,
 * and this call traverses shard `rank` of `n_ranks` from its share.  The
 * shards' candidate rows and test counts together equal kdop_traverse's
 * (each candidate on exactly one shard); kdop_contacts etc. then work on the
 * shard's rows.  With n_ranks = 1 it is kdop_traverse seeded by the frontier.
 * Batched mode only.  Synchronises.  The sharded (multi-GPU) use of the
 * reference's single-pair traversal (kdop_tandem_traversal.h:161-196) has no
 * counterpart there. */
int kdop_traverse_shard(kdop_scene* scene, int64_t n_pairs, const uint32_t* pairs, int memory,
                        const kdop_traverse_opts* opts, int rank, int n_ranks, int64_t frontier_min);
/* Synchronises and reads the counters of the last traversal/contacts.
 * Returns KDOP_ERR_CAPACITY when candidates, contacts or the work queue
 * overflowed (stats then hold the required sizes), KDOP_ERR_TIMEOUT when a
 * device wait gave up. */
int kdop_get_stats(kdop_scene* scene, kdop_stats* stats);
/* Grows the scene's candidate / contact / queue buffers (0 = keep). */
int kdop_reserve(kdop_scene* scene, int64_t candidates, int64_t contacts, int64_t queue);
/* Sets the three capacities exactly (0 = keep), e.g. to bound device memory. */
int kdop_set_capacity(kdop_scene* scene, int64_t candidates, int64_t contacts, int64_t queue);

/* Tandem traversal that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc while they
 * run -- a plugin inside a host application whose own allocator must own
 * every byte of device memory, simulators that reserve a fixed
 * device-memory budget or arena once at start-up, and real-time loops that
 * must not risk an allocation failure (or an allocator's device-wide
 * synchronisation) in the middle of a step.
 *
 * The caller passes device memory only: pairs (n_pairs * 2 mesh indices),
 * candidates (3 * cap uint32: tets of A | tets of B | pair indices; tet
 * indices are scene-global, i.e. mesh m's tets start at the tet count of the
 * meshes before m) and counters (4 uint64: candidates found -- more than cap
 * means the rows were cut --, node-pair tests, overlapping leaf pairs, device
 * error bits).  The traversal's control block and work queue live in a static
 * device array of 1.25 MiB per GPU (a queue of 65,536 entries) that every GPU
 * loading the library keeps until the process exits; a run that needs more
 * queue entries sets error bit 2 in counters[3] and is incomplete (use
 * kdop_traverse then).  cap above 2^32 - 16 or n_pairs of 2^31 - 1 or more
 * are rejected with KDOP_ERR_CAPACITY.  Calls share the array, so calls that
 * overlap on the GPU (other streams, other threads) race; each call clears the
 * parts that must start at zero.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress, once per device): make that
 * first call before any stream capture.  Asynchronous on the scene's stream. */
int kdop_traverse_noalloc(kdop_scene* scene, int64_t n_pairs, const uint32_t* pairs, uint32_t* candidates,
                          int64_t cap, unsigned long long* counters, const kdop_traverse_opts* opts);

/* Candidate rows (pair index, mesh-local tet of A, mesh-local tet of B) in the
 * device's emission order; sort them for a canonical order. Synchronises. */
int kdop_read_candidates(kdop_scene* scene, uint32_t* rows, int64_t cap_rows, int64_t* n_rows);

/* ---- contacts (replaces SelectContactPointAlgorithm + ContactsCallback) ---- */
typedef struct {
  float p[3];     /* contact point, world space */
  float n[3];     /* contact normal (unit, outward from A's face) */
  float depth;    /* penetration measure, <= 0 when overlapping */
  uint32_t cand;  /* candidate row index the contact came from */
} kdop_contact;

/* MOST_OPPOSING_SURFACES contacts
 * (geometry_contacts_tetrahedron_tetrahedron.h:1313-1345) of every candidate
 * of the last traversal, from the vertex positions of the last refit: the
 * posed (and deformed) positions it computed in KDOP_REFIT_POSE /
 * KDOP_REFIT_DEFORM mode, the kdop_set_vertices positions in
 * KDOP_REFIT_VERTICES mode.  kdop_contacts_adjoint differentiates with
 * respect to the same positions.  Asynchronous. */
int kdop_contacts(kdop_scene* scene);
/* Contacts grouped by candidate (rows of one candidate are contiguous, in the
 * reference's reporting order).  `rows` may be host or device memory (a
 * device buffer gets a device-to-device copy).  Synchronises. */
int kdop_read_contacts(kdop_scene* scene, kdop_contact* rows, int64_t cap_rows, int64_t* n_rows);

/* Contact point reduction of PROX (prox_collision_detection.h:341-350):
 * the contact rows sorted by ContactPoint::operator< (prox_contact_point.h:
 * 135-194: body i, body j, p.y, p.x, p.z, n.y, n.x, n.z, depth, each by
 * float `<`), then std::unique with ContactPoint::operator== (:91-133: same
 * bodies and every component within working_precision<float>() =
 * 10 FLT_EPSILON, tiny_precision.h:21-24), which keeps a row only when it
 * differs from the last row kept.  The kept rows go to `out` (and their
 * bodies, 2 uint32 per row, to `out_bodies` unless NULL) in that order; host
 * or device memory.  *n_out = rows kept; KDOP_ERR_CAPACITY (nothing written)
 * when that exceeds cap.  Rows whose nine key fields all compare equal keep
 * their input order (std::sort leaves it unspecified; such rows can differ
 * only in the sign of a zero and in `cand`, and all but the first are
 * dropped).  Synchronises.  The sort's scratch is device memory the context
 * keeps for later calls (allocated when a call needs more than it holds,
 * freed by kdop_ctx_destroy).
 *
 * kdop_reduce_contacts: the scene's contacts of the last kdop_contacts, the
 * bodies of a row being the meshes (A, B) of its candidate's pair.
 * kdop_reduce_contact_rows: any n rows (host or device) with their bodies. */
int kdop_reduce_contacts(kdop_scene* scene, kdop_contact* out, uint32_t* out_bodies, int64_t cap, int64_t* n_out);
int kdop_reduce_contact_rows(kdop_ctx* ctx, const kdop_contact* rows, const uint32_t* bodies, int64_t n,
                             kdop_contact* out, uint32_t* out_bodies, int64_t cap, int64_t* n_out);

/* Puts the last traversal's results in a reproducible order, on the device:
 * candidate rows by (pair, tet of A, tet of B) and, after kdop_contacts, the
 * contact rows grouped by candidate in that order (each candidate's rows in
 * the reference's reporting order), their `cand` fields, and the records the
 * adjoint reads, to match.  Replaces the OpenCL back-end's result sort
 * (cl/kdop_cl_tandem_traversal.h:1773-1788; the sequential back-end reports
 * in traversal order).  Synchronises; not for stream capture. */
int kdop_sort_results(kdop_scene* scene);

/* Adjoint of contact generation with the pair set and every discrete choice
 * of the last kdop_contacts held fixed: given dL/d(depth) and dL/d(normal)
 * per contact row (n_contacts and n_contacts*3 floats; dn may be NULL),
 * ADDS dL/d(world vertex position) into grad (n_verts_total*3 floats).
 * All three pointers share `memory`. */
int kdop_contacts_adjoint(kdop_scene* scene, const float* d_depth, const float* d_normal, float* grad,
                          int memory);

/* ---- one collision step in a CUDA graph ------------------------------------ */
/* Per-step pose integration for the captured step: each step p += lin_vel,
 * q = normalise(q + 0.5 (0, ang_vel) q), deformation phase += phase_rate. */
int kdop_set_motion(kdop_scene* scene, const float* lin_vel, const float* ang_vel, float phase_rate, int memory);
/* Captures [motion update?] + refit(mode) + traversal + contacts into a CUDA
 * graph over the given mesh pairs.  flags bit 0: include the motion update. */
/* Buffers must be large enough before capture (kdop_reserve): a capture
 * holds buffer addresses, and any later reallocation drops the graph. */
int kdop_graph_capture(kdop_scene* scene, int refit_mode, int64_t n_pairs, const uint32_t* pairs, int memory,
                       const kdop_traverse_opts* opts, int flags);
int kdop_graph_launch(kdop_scene* scene);
int kdop_graph_release(kdop_scene* scene);

/* ---- autotuner --------------------------------------------------------------- */
/* Times traversal configurations on the given pairs -- coordinate descent,
 * two sweeps, over block warps {4,8,16}, stack capacity {128..1024}, load
 * group {1,2,4,8}, donation threshold {32..256}, wave pairs {0,16,64,128},
 * shared-memory carveout {0,25,50,100} and root chunk {1,4}, starting from
 * the defaults -- and caches the fastest for this scene and, on the scene's
 * context, for its K and size class (see kdop_traverse_opts_default).  Each
 * configuration is the median of max(repeats, 5) (rounded up to odd) runs
 * timed one by one; a challenger replaces the incumbent only when more than
 * 2 % faster.  best (optional) receives the choice.  Synchronises. */
int kdop_autotune(kdop_scene* scene, int64_t n_pairs, const uint32_t* pairs, int memory, int repeats,
                  kdop_traverse_opts* best);

/* Number of kernel launches this context has enqueued so far. */
int64_t kdop_ctx_launch_count(const kdop_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
