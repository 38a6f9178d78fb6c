"""Synthetic tetrahedral-lattice scenes for the kDOP collision path.

No public dataset is used by the reference's collision benchmarks; every
workload here is a seeded lattice of unit cubes split into 6 tetrahedra each,
with the shapes, sizes, jitter and poses of the five benchmark configurations
(small pair, large pair, 512 uneven pairs, 64 deforming pairs, 256 pairs for
differentiation).

Vertex (i, j, k) of an n^3-cell lattice has index i + (n+1) (j + (n+1) k) and
sits at (i, j, k) - n/2, so each mesh is centred on the origin.  Cube corner c
(bit0 = x, bit1 = y, bit2 = z) is split into the six Kuhn tetrahedra
(0,1,3,7), (0,1,7,5), (0,4,5,7), (0,3,2,7), (0,2,6,7), (0,6,4,7), all of
positive orientation as the reference's tet-tet test requires
(geometry_overlap_tetrahedron_tetrahedron.h:59-60).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

KUHN = np.array([[0, 1, 3, 7], [0, 1, 7, 5], [0, 4, 5, 7],
                 [0, 3, 2, 7], [0, 2, 6, 7], [0, 6, 4, 7]], dtype=np.int64)

SUPPORTED_K = (6, 8, 12, 14, 18, 20, 26)


@dataclasses.dataclass
class Mesh:
    """One tetrahedral mesh: rest vertices, tets and the boundary-face map."""
    xyz: np.ndarray      # (nv, 3) float32 rest positions
    tets: np.ndarray     # (nt, 4) uint32 vertex indices
    surf: np.ndarray     # (nt,) uint8, bit v = face opposite vertex v is boundary

    @property
    def n_verts(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])


@dataclasses.dataclass
class Scene:
    """Meshes, one rigid pose per mesh and the mesh pairs to test."""
    name: str
    K: int
    meshes: List[Mesh]
    quat: np.ndarray     # (n_meshes, 4) float32, (w, x, y, z)
    pos: np.ndarray      # (n_meshes, 3) float32
    pairs: np.ndarray    # (n_pairs, 2) uint32 mesh indices (A, B)
    extra: dict = dataclasses.field(default_factory=dict)

    @property
    def n_tets(self) -> int:
        return sum(m.n_tets for m in self.meshes)


_TOPOLOGY = {}


def lattice_topology(n: int):
    """(rest xyz float64, tets, surface map) of the n^3-cell lattice, cached."""
    if n not in _TOPOLOGY:
        m = n + 1
        g = np.arange(m, dtype=np.float64)
        z, y, x = np.meshgrid(g, g, g, indexing="ij")
        xyz = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1) - n / 2.0
        ci = np.arange(n)
        ck, cj, cii = np.meshgrid(ci, ci, ci, indexing="ij")
        base = (cii + m * (cj + m * ck)).ravel()
        corner = np.array([(c & 1) + m * ((c >> 1) & 1) + m * m * ((c >> 2) & 1) for c in range(8)])
        tets = (base[:, None, None] + corner[KUHN][None, :, :]).reshape(-1, 4).astype(np.uint32)
        for a in (xyz, tets):
            a.setflags(write=False)
        surf = _lattice_surface(n, tets)
        surf.setflags(write=False)
        _TOPOLOGY[n] = (xyz, tets, surf)
    return _TOPOLOGY[n]


def _lattice_surface(n: int, tets: np.ndarray) -> np.ndarray:
    # boundary faces of the Kuhn lattice: a face is on the boundary iff its
    # three vertices lie on one face of the cube [0, n]^3 (a face strictly
    # inside the cube always has a second tet); checked against face counting
    # in the tests.
    if n <= 8:
        return surface_map(tets)
    m = n + 1
    v = tets.astype(np.int64)
    coords = np.stack([v % m, (v // m) % m, v // (m * m)], axis=-1)  # (nt, 4, 3)
    surf = np.zeros(tets.shape[0], np.uint8)
    for k in range(4):
        others = [u for u in range(4) if u != k]
        c = coords[:, others, :]  # (nt, 3, 3)
        on = np.zeros(tets.shape[0], bool)
        for d in range(3):
            col = c[:, :, d]
            on |= np.all(col == 0, axis=1) | np.all(col == n, axis=1)
        surf |= on.astype(np.uint8) << k
    return surf


def lattice(n: int, jitter: float = 0.0, rng: Optional[np.random.Generator] = None) -> Mesh:
    """n^3 cubes x 6 Kuhn tets, centred on the origin, optional uniform jitter."""
    xyz, tets, surf = lattice_topology(n)
    if jitter:
        xyz = xyz + rng.uniform(-jitter, jitter, size=xyz.shape)
    return Mesh(xyz.astype(np.float32), tets, surf)


def skip_lattice(n: int, jitter: float, rng: np.random.Generator) -> None:
    """Advances rng past the draws lattice(n, jitter, rng) would take (one
    64-bit output per uniform double) without building the mesh."""
    if jitter:
        rng.bit_generator.advance(3 * (n + 1) ** 3)


def surface_map(tets: np.ndarray) -> np.ndarray:
    """Boundary faces by face counting (mesh_array_compute_surface_map.h:41-76):
    the face opposite local vertex v of a tet is on the boundary when no other
    tet shares its three vertices."""
    nt = tets.shape[0]
    surf = np.zeros(nt, dtype=np.uint8)
    if nt == 0:
        return surf
    faces = []
    for v in range(4):
        others = [u for u in range(4) if u != v]
        faces.append(np.sort(tets[:, others].astype(np.int64), axis=1))
    f = np.concatenate(faces, axis=0)  # (4 nt, 3)
    _, inv, cnt = np.unique(f, axis=0, return_inverse=True, return_counts=True)
    inv = inv.reshape(-1)
    boundary = (cnt[inv] == 1).reshape(4, nt)
    for v in range(4):
        surf |= (boundary[v].astype(np.uint8) << v)
    return surf


def random_quaternion(rng: np.random.Generator) -> np.ndarray:
    """Uniform random unit quaternion (w, x, y, z), Shoemake's method."""
    u1, u2, u3 = rng.uniform(0.0, 1.0, size=3)
    a, b = math.sqrt(1.0 - u1), math.sqrt(u1)
    x = a * math.sin(2 * math.pi * u2)
    y = a * math.cos(2 * math.pi * u2)
    z = b * math.sin(2 * math.pi * u3)
    w = b * math.cos(2 * math.pi * u3)
    return np.array([w, x, y, z], dtype=np.float32)


def axis_angle_quaternion(axis, angle: float) -> np.ndarray:
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    s = math.sin(angle / 2)
    return np.array([math.cos(angle / 2), axis[0] * s, axis[1] * s, axis[2] * s], dtype=np.float32)


def _identity(n: int):
    q = np.zeros((n, 4), dtype=np.float32)
    q[:, 0] = 1.0
    return q, np.zeros((n, 3), dtype=np.float32)


def _touching_poses(rng, n: int, q, p, ia: int, ib: int, pen=(0.1, 0.5), max_deg: float = 5.0):
    """A at the origin; B face to face with A along a random axis direction,
    penetrating by U(pen) cells, turned by at most max_deg degrees."""
    q[ia] = (1.0, 0.0, 0.0, 0.0)
    p[ia] = 0.0
    q[ib] = axis_angle_quaternion(rng.normal(size=3), math.radians(max_deg) * rng.uniform(-1.0, 1.0))
    axis = int(rng.integers(0, 3))
    sign = 1.0 if rng.uniform() < 0.5 else -1.0
    d = np.zeros(3)
    d[axis] = sign * (n - rng.uniform(pen[0], pen[1]))
    p[ib] = d


def touching_pair(n: int = 4, seed: int = 11, K: int = 14, jitter: float = 0.0) -> Scene:
    """Two n^3-cell lattices face to face with a small penetration: a
    contact-rich case for contact generation."""
    rng = np.random.default_rng(seed)
    a = lattice(n, jitter, rng)
    b = lattice(n, jitter, rng)
    q, p = _identity(2)
    _touching_poses(rng, n, q, p, 0, 1)
    return Scene(f"touching pair of {n}^3-cell lattices, k={K}", K, [a, b], q, p, np.array([[0, 1]], np.uint32))


def config1() -> Scene:
    """Two 10^3-cell lattices (6000 tets each); B rotated by a random
    quaternion (seed 0) and translated by (0.3, 0.1, 0) cells; k = 14."""
    rng = np.random.default_rng(0)
    a = lattice(10)
    b = lattice(10)
    q, p = _identity(2)
    q[1] = random_quaternion(rng)
    p[1] = (0.3, 0.1, 0.0)
    return Scene("config1: 2 x 10^3-cell lattices (6000 tets), k=14", 14, [a, b], q, p,
                 np.array([[0, 1]], dtype=np.uint32))


def config2(n: int = 64) -> Scene:
    """Two n^3-cell lattices (n=64: 1,572,864 tets each), vertices jittered by
    U(-0.2, 0.2) (seed 1); B translated by n/2 cells along x (half the volume
    overlaps) and turned by a seeded rotation of at most 10 degrees; k = 26."""
    rng = np.random.default_rng(1)
    a = lattice(n, 0.2, rng)
    b = lattice(n, 0.2, rng)
    q, p = _identity(2)
    ax = rng.normal(size=3)
    q[1] = axis_angle_quaternion(ax, math.radians(10.0) * rng.uniform(0.0, 1.0))
    p[1] = (n / 2.0, 0.0, 0.0)
    return Scene(f"config2: 2 x {n}^3-cell jittered lattices ({6 * n ** 3} tets each), k=26", 26, [a, b], q, p,
                 np.array([[0, 1]], dtype=np.uint32))


def _pair_poses(rng, n: int, q, p, ia: int, ib: int):
    q[ia] = random_quaternion(rng)
    q[ib] = random_quaternion(rng)
    radius = n * math.sqrt(3.0) / 2.0
    d = rng.uniform(0.0, 1.0) * radius
    u = rng.normal(size=3)
    u /= np.linalg.norm(u)
    p[ia] = 0.0
    p[ib] = d * u


def config3(n_pairs: int = 512, seed: int = 2, min_tets: float = 1e3, max_tets: float = 2e5,
            jitter: float = 0.15, K: int = 14, keep=None) -> Scene:
    """n_pairs mesh pairs; per pair a tet count T drawn log-uniformly from
    [1e3, 2e5] and both meshes n^3 cells with n = round((T/6)^(1/3)); vertex
    jitter +-0.15; random rotations, centroids U(0,1) mesh radii apart; k = 14.

    keep (optional): the pair indices to build.  The random stream is the
    same as for the whole scene (the jitter of the other pairs' meshes is
    skipped, not drawn), so the kept pairs equal those of config3(n_pairs,
    seed); the returned scene holds only them, renumbered in the given order,
    with extra['pair_ids'] the global indices and extra['pair_tets'] the tet
    count of both meshes of every pair of the whole scene."""
    rng = np.random.default_rng(seed)
    keep_set = None if keep is None else set(int(k) for k in keep)
    built = {}
    pair_tets = np.zeros(n_pairs, np.int64)
    q, p = _identity(2 * n_pairs)
    cache = {}
    for i in range(n_pairs):
        T = math.exp(rng.uniform(math.log(min_tets), math.log(max_tets)))
        n = max(1, int(round((T / 6.0) ** (1.0 / 3.0))))
        if keep_set is None or i in keep_set:
            built[i] = [lattice(n, jitter, rng) for _ in range(2)]
        else:
            for _ in range(2):
                skip_lattice(n, jitter, rng)
        _pair_poses(rng, n, q, p, 2 * i, 2 * i + 1)
        pair_tets[i] = 2 * 6 * n ** 3
        cache[n] = cache.get(n, 0) + 1
    ids = list(range(n_pairs)) if keep is None else [int(k) for k in keep]
    meshes: List[Mesh] = []
    sel = []
    for i in ids:
        meshes += built[i]
        sel += [2 * i, 2 * i + 1]
    pairs = np.arange(2 * len(ids), dtype=np.uint32).reshape(-1, 2)
    sel = np.array(sel, np.int64)
    return Scene(f"config3: {n_pairs} pairs, 1k-200k tets log-uniform, k={K}", K, meshes, q[sel].copy(),
                 p[sel].copy(), pairs, {"sizes": cache, "pair_ids": np.array(ids, np.int64),
                                        "pair_tets": pair_tets})


def subset(sc: Scene, pair_ids) -> Scene:
    """The pairs pair_ids of a scene (and their meshes), renumbered in order."""
    ids = [int(i) for i in pair_ids]
    used: List[int] = []
    index = {}
    pairs = np.zeros((len(ids), 2), np.uint32)
    for k, i in enumerate(ids):
        for s in range(2):
            m = int(sc.pairs[i, s])
            if m not in index:
                index[m] = len(used)
                used.append(m)
            pairs[k, s] = index[m]
    extra = dict(sc.extra)
    for key in ("lin_vel", "ang_vel"):
        if key in extra:
            extra[key] = np.asarray(extra[key])[used].copy()
    extra["pair_ids"] = np.array(ids, np.int64)
    return Scene(sc.name, sc.K, [sc.meshes[m] for m in used], sc.quat[used].copy(), sc.pos[used].copy(), pairs,
                 extra)


def config4(n_pairs: int = 64, n: int = 40, seed: int = 3, K: int = 18) -> Scene:
    """n_pairs pairs of n^3-cell lattices (n=40: 384,000 tets each) for the
    deforming, graph-captured benchmark, posed face to face (penetrating
    0.1-0.5 cells) so that contacts exist; per mesh a random rigid velocity
    (seed 3) stored in extra['lin_vel'] / extra['ang_vel']; k = 18."""
    rng = np.random.default_rng(seed)
    base = lattice(n)
    meshes = [Mesh(base.xyz, base.tets, base.surf) for _ in range(2 * n_pairs)]
    q, p = _identity(2 * n_pairs)
    pairs = np.zeros((n_pairs, 2), dtype=np.uint32)
    for i in range(n_pairs):
        _touching_poses(rng, n, q, p, 2 * i, 2 * i + 1)
        pairs[i] = (2 * i, 2 * i + 1)
    lin = rng.uniform(-0.05, 0.05, size=(2 * n_pairs, 3)).astype(np.float32)
    ang = rng.uniform(-0.01, 0.01, size=(2 * n_pairs, 3)).astype(np.float32)
    return Scene(f"config4: {n_pairs} pairs of {n}^3-cell lattices ({6 * n ** 3} tets), deforming, k={K}", K,
                 meshes, q, p, pairs,
                 {"lin_vel": lin, "ang_vel": ang, "amp": 0.1, "L": float(n), "phase_rate": 0.05})


def config5(n_pairs: int = 256, n: int = 20, seed: int = 4, K: int = 14) -> Scene:
    """n_pairs pairs of n^3-cell lattices (n=20: 48,000 tets each) in random
    overlapping poses (seed 4): face to face, penetrating 0.1-0.5 cells, turned
    by up to 5 degrees, so that the most-opposing-surfaces contact algorithm
    reports contacts; for differentiation of contact depths; k = 14."""
    rng = np.random.default_rng(seed)
    base = lattice(n)
    meshes = [Mesh(base.xyz, base.tets, base.surf) for _ in range(2 * n_pairs)]
    q, p = _identity(2 * n_pairs)
    pairs = np.zeros((n_pairs, 2), dtype=np.uint32)
    for i in range(n_pairs):
        _touching_poses(rng, n, q, p, 2 * i, 2 * i + 1)
        pairs[i] = (2 * i, 2 * i + 1)
    return Scene(f"config5: {n_pairs} pairs of {n}^3-cell lattices ({6 * n ** 3} tets), k={K}", K, meshes, q, p,
                 pairs)


def small_batch(n_pairs: int = 8, n_lo: int = 2, n_hi: int = 6, seed: int = 7, K: int = 14,
                jitter: float = 0.15) -> Scene:
    """A few small uneven pairs with the pose model of config3 (test sizes)."""
    rng = np.random.default_rng(seed)
    meshes: List[Mesh] = []
    q, p = _identity(2 * n_pairs)
    pairs = np.zeros((n_pairs, 2), dtype=np.uint32)
    for i in range(n_pairs):
        n = int(rng.integers(n_lo, n_hi + 1))
        meshes.append(lattice(n, jitter, rng))
        meshes.append(lattice(int(rng.integers(n_lo, n_hi + 1)), jitter, rng))
        _pair_poses(rng, n, q, p, 2 * i, 2 * i + 1)
        pairs[i] = (2 * i, 2 * i + 1)
    return Scene(f"small batch of {n_pairs} pairs", K, meshes, q, p, pairs)


def concat(meshes: List[Mesh]):
    """Concatenate meshes: (v_off, xyz, t_off, tets (mesh-local ids), surf)."""
    v_off = np.zeros(len(meshes) + 1, dtype=np.int64)
    t_off = np.zeros(len(meshes) + 1, dtype=np.int64)
    for i, m in enumerate(meshes):
        v_off[i + 1] = v_off[i] + m.n_verts
        t_off[i + 1] = t_off[i] + m.n_tets
    xyz = np.concatenate([m.xyz for m in meshes], axis=0) if meshes else np.zeros((0, 3), np.float32)
    tets = np.concatenate([m.tets for m in meshes], axis=0) if meshes else np.zeros((0, 4), np.uint32)
    surf = np.concatenate([m.surf for m in meshes], axis=0) if meshes else np.zeros((0,), np.uint8)
    return v_off, np.ascontiguousarray(xyz), t_off, np.ascontiguousarray(tets), np.ascontiguousarray(surf)
