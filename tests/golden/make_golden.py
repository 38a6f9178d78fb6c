"""Generate tests/golden/*.npz from the reference's own CPU code.

Run in a container where the reference sources are mounted and the harness is
built (`make -C oracle ref REF_ROOT=<reference checkout>`):

    python tests/golden/make_golden.py

Every array comes out of oracle/_ref/libkdop_ref_record.so, i.e. the
reference's make_tree / refit_tree / tandem_traversal / mesh_reorder /
compute_surface_map / contacts_tetrahedron_tetrahedron / tiny::rotate compiled
from its sources.  The fixtures pin the CPU oracle (oracle/kdop_oracle.c) and,
through it, the CUDA library on machines where the reference is absent.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "bvh-tvcg18_b200"))

from oracle.pyoracle import Reference  # noqa: E402
from kdop_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sorted_pairs(p: np.ndarray) -> np.ndarray:
    if p.size == 0:
        return p.reshape(0, 2)
    o = np.lexsort((p[:, 1], p[:, 0]))
    return p[o]


def reduction_rows(rng, n_base=600, n_bodies=3):
    """Contact rows (n, 7: p, n, depth) and bodies (n, 2) for the reduction."""
    eps = np.float32(np.float32(np.finfo(np.float32).eps) * np.float32(10))
    base = rng.uniform(-1, 1, (n_base, 7)).astype(np.float32)
    bodies = rng.integers(0, n_bodies, (n_base, 2)).astype(np.uint32)
    k = n_base // 2
    src = rng.integers(0, n_base, k)
    near = base[src] + (rng.integers(-4, 5, (k, 7)) * (np.float32(0.3) * eps)).astype(np.float32)
    near[: k // 5] = base[src[: k // 5]]
    chains = []
    for c in range(20):
        r0 = rng.uniform(-1, 1, 7).astype(np.float32)
        steps = np.arange(6, dtype=np.float32)[:, None] * (np.float32(0.9) * eps)
        chains.append(r0 + steps * np.array([0, 1, 0, 0, 0, 0, 0], np.float32))
    chain = np.concatenate(chains)
    chain_b = np.repeat(rng.integers(0, n_bodies, (20, 2)), 6, axis=0).astype(np.uint32)
    rows = np.concatenate([base, near, chain]).astype(np.float32)
    b = np.concatenate([bodies, bodies[src], chain_b]).astype(np.uint32)
    z = rng.integers(0, len(rows), 40)
    rows[z[:20], 1] = np.float32(0.0)
    rows[z[20:], 1] = np.float32(-0.0)
    perm = rng.permutation(len(rows))
    return rows[perm], b[perm]


def main():
    R = Reference()
    g = {}
    for K in scenes.SUPPORTED_K:
        g[f"dirs_{K}"] = R.direction_table(K)

    # rigid transform (tiny::rotate + translation)
    rng = np.random.default_rng(123)
    xyz = rng.uniform(-5, 5, size=(64, 3)).astype(np.float32)
    q = scenes.random_quaternion(rng)
    p = rng.uniform(-2, 2, size=3).astype(np.float32)
    g["rotate_q"], g["rotate_p"], g["rotate_in"] = q, p, xyz
    g["rotate_out"] = R.rotate(q, p, xyz)

    # surface map and Morton order of a jittered 4^3 lattice
    m = scenes.lattice(4, 0.2, np.random.default_rng(5))
    g["lat4_xyz"], g["lat4_tets"] = m.xyz, m.tets
    g["lat4_surf"] = R.surface_map(m.xyz, m.tets)
    ox, ot = R.mesh_reorder(m.xyz, m.tets)
    g["lat4_reorder_xyz"], g["lat4_reorder_tets"] = ox, ot

    # config 1 (two 10^3 lattices, k = 14): pair list, node-pair tests, tree A
    sc = scenes.config1()
    A, B = sc.meshes
    xa = R.rotate(sc.quat[0], sc.pos[0], A.xyz)
    xb = R.rotate(sc.quat[1], sc.pos[1], B.xyz)
    r = R.traverse(14, A.xyz, sc.quat[0], sc.pos[0], A.tets, B.xyz, sc.quat[1], sc.pos[1], B.tets,
                   want_volumes=True)
    g["c1_xyzB"] = xb
    g["c1_pairs"] = sorted_pairs(r["pairs"])
    g["c1_tests"] = np.int64(r["tests"])
    g["c1_ncontacts"] = np.int64(len(r["contacts"]))
    g["c1_volA_sha"] = np.array(sha(r["volumes"]))
    g["c1_volA_head"] = r["volumes"][:64]
    g["c1_leafA"] = r["leaf"]
    r8 = R.traverse(14, A.xyz, sc.quat[0], sc.pos[0], A.tets, B.xyz, sc.quat[1], sc.pos[1], B.tets,
                    mem_bytes=8000)
    g["c1_chunked_pairs_sha"] = np.array(sha(sorted_pairs(r8["pairs"])))
    g["c1_chunked_tests"] = np.int64(r8["tests"])

    # contact-rich touching pairs, several K
    for seed, K in [(0, 14), (1, 14), (2, 26), (3, 18), (4, 8)]:
        sc = scenes.touching_pair(n=4, seed=seed, K=K)
        A, B = sc.meshes
        xa = R.rotate(sc.quat[0], sc.pos[0], A.xyz)
        xb = R.rotate(sc.quat[1], sc.pos[1], B.xyz)
        r = R.traverse(K, A.xyz, sc.quat[0], sc.pos[0], A.tets, B.xyz, sc.quat[1], sc.pos[1], B.tets)
        key = f"t{seed}"
        g[f"{key}_K"] = np.int64(K)
        g[f"{key}_xyzA"], g[f"{key}_xyzB"] = xa, xb
        g[f"{key}_pairs_trav"] = r["pairs"]
        g[f"{key}_tests"] = np.int64(r["tests"])
        g[f"{key}_contacts_f32"] = r["contacts"]
        g[f"{key}_contacts_f64"] = R.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, r["pairs"], fp64=True)
    # broad phase: 300 bodies, positions on a coarse grid so that some boxes
    # touch exactly (equal max and min count as overlapping), radii of the
    # meshes of a small batch
    rng = np.random.default_rng(77)
    pos = (rng.integers(0, 24, size=(300, 3)) * 0.5).astype(np.float32)
    rad = np.float32(0.25) * rng.integers(1, 5, size=300).astype(np.float32)
    g["broad_pos"], g["broad_radius"] = pos, rad
    g["broad_pairs"] = R.broad_pairs(pos, rad, 0)
    g["broad_pairs_grid"] = R.broad_pairs(pos, rad, 1)
    sb = scenes.small_batch(n_pairs=4, seed=9)
    g["radius_xyz"] = np.concatenate([m.xyz for m in sb.meshes])
    g["radius_n"] = np.array([m.n_verts for m in sb.meshes], np.int64)
    g["radius_out"] = np.array([R.mesh_radius(m.xyz) for m in sb.meshes], np.float32)
    # contact reduction: rows with near duplicates (offsets of whole multiples
    # of 0.3 working precisions, inside and beyond it), exact copies, signed
    # zeros and chains along p.y whose links are within the tolerance but
    # whose ends are not, over three bodies
    rr, rb = reduction_rows(np.random.default_rng(91))
    g["reduce_rows"], g["reduce_bodies"] = rr, rb
    g["reduce_out_rows"], g["reduce_out_bodies"] = R.reduce_contacts(rr, rb)
    np.savez_compressed(os.path.join(OUT, "reference_golden.npz"), **g)
    print("wrote", os.path.join(OUT, "reference_golden.npz"), os.path.getsize(os.path.join(OUT, "reference_golden.npz")),
          "bytes")


if __name__ == "__main__":
    main()
