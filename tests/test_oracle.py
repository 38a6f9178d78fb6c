"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference's compiled CPU path) and, where
the reference harness is built, against the reference directly."""
import hashlib

import numpy as np
import pytest

from conftest import sorted_rows, world_xyz
from kdop_b200 import scenes


def preorder(left, right, tet, vol):
    order, leaf = [], []
    stack = [0]
    while stack:
        i = stack.pop()
        order.append(i)
        leaf.append(tet[i] if left[i] < 0 else -1)
        if left[i] >= 0:
            stack.append(right[i])
            stack.append(left[i])
    return vol[order], np.array(leaf)


@pytest.mark.parametrize("K", scenes.SUPPORTED_K)
def test_direction_tables_bit_exact(oracle, golden, K):
    assert oracle.dirs(K).tobytes() == golden[f"dirs_{K}"].tobytes()


def test_rotate_bit_exact(oracle, golden):
    out = oracle.rotate(golden["rotate_q"], golden["rotate_p"], golden["rotate_in"])
    assert out.tobytes() == golden["rotate_out"].tobytes()


def test_surface_map(oracle, golden):
    tets = golden["lat4_tets"]
    assert np.array_equal(oracle.surface_map(golden["lat4_xyz"].shape[0], tets), golden["lat4_surf"])
    assert np.array_equal(scenes.surface_map(tets), golden["lat4_surf"])


def test_morton_order_matches_reference_reorder(oracle, golden):
    xyz, tets = golden["lat4_xyz"], golden["lat4_tets"]
    perm = oracle.morton_order(xyz, tets)
    mine = xyz[tets[perm]].reshape(-1, 12)
    ref = golden["lat4_reorder_xyz"][golden["lat4_reorder_tets"]].reshape(-1, 12)
    assert np.array_equal(mine, ref)


def test_config1_pairs_tests_and_tree(oracle, golden):
    sc = scenes.config1()
    A, B = sc.meshes
    xb = world_xyz(oracle, sc, 1)
    assert xb.tobytes() == golden["c1_xyzB"].tobytes()
    xa = world_xyz(oracle, sc, 0)
    pairs, tests, _ = oracle.run_pair(14, xa, A.tets, A.surf, xb, B.tets, B.surf, restA=A.xyz, restB=B.xyz)
    assert np.array_equal(sorted_rows(pairs), golden["c1_pairs"])
    assert tests == int(golden["c1_tests"])
    # whole tree of A: node volumes in preorder, bit for bit
    perm = oracle.morton_order(A.xyz, A.tets)
    left, right, tet = oracle.build_tree(perm)
    vol = oracle.refit(14, xa, A.tets, left, right, tet)
    pv, leaf = preorder(left, right, tet, vol)
    assert hashlib.sha256(pv.tobytes()).hexdigest() == str(golden["c1_volA_sha"])
    assert np.array_equal(leaf, golden["c1_leafA"])


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 4])
def test_touching_pairs_contacts(oracle, golden, seed):
    key = f"t{seed}"
    K = int(golden[f"{key}_K"])
    sc = scenes.touching_pair(n=4, seed=seed, K=K)
    A, B = sc.meshes
    xa, xb = golden[f"{key}_xyzA"], golden[f"{key}_xyzB"]
    assert world_xyz(oracle, sc, 1).tobytes() == xb.tobytes()
    pairs, tests, _ = oracle.run_pair(K, xa, A.tets, A.surf, xb, B.tets, B.surf, restA=A.xyz, restB=B.xyz)
    # same traversal order as the reference's recursion
    assert np.array_equal(pairs, golden[f"{key}_pairs_trav"])
    assert tests == int(golden[f"{key}_tests"])
    cf, _ = oracle.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, pairs, "f")
    assert len(cf) > 0
    assert cf.tobytes() == golden[f"{key}_contacts_f32"].tobytes()
    cd, _ = oracle.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, pairs, "d")
    assert np.array_equal(cd, golden[f"{key}_contacts_f64"])


def test_sine_accuracy(oracle):
    xs = np.linspace(-40.0, 40.0, 2001, dtype=np.float32)
    ys = np.array([oracle.sin(float(x)) for x in xs])
    assert np.max(np.abs(ys - np.sin(xs.astype(np.float64)))) < 2e-6


@pytest.mark.parametrize("K,seed", [(6, 1), (8, 2), (12, 3), (14, 4), (18, 5), (20, 6), (26, 7)])
def test_oracle_against_reference_random(oracle, reference, K, seed):
    rng = np.random.default_rng(seed)
    a = scenes.lattice(int(rng.integers(2, 5)), 0.15, rng)
    b = scenes.lattice(int(rng.integers(2, 5)), 0.15, rng)
    q = scenes.random_quaternion(rng)
    p = rng.uniform(-1.5, 1.5, size=3).astype(np.float32)
    xb = oracle.rotate(q, p, b.xyz)
    assert xb.tobytes() == reference.rotate(q, p, b.xyz).tobytes()
    q0, p0 = np.float32([1, 0, 0, 0]), np.float32([0, 0, 0])
    r = reference.traverse(K, a.xyz, q0, p0, a.tets, b.xyz, q, p, b.tets)
    pairs, tests, _ = oracle.run_pair(K, a.xyz, a.tets, a.surf, xb, b.tets, b.surf, restA=a.xyz, restB=b.xyz)
    assert np.array_equal(pairs, r["pairs"])
    assert tests == r["tests"]
    cf, _ = oracle.contacts(a.xyz, a.tets, a.surf, xb, b.tets, b.surf, pairs, "f")
    assert cf.tobytes() == r["contacts"].tobytes()


def test_broad_phase_oracle_against_golden(oracle, golden):
    pos, rad = golden["broad_pos"], golden["broad_radius"]
    got = oracle.broad_pairs(pos, rad)
    assert np.array_equal(got, golden["broad_pairs"])
    # the reference's grid algorithm reports the same sorted set
    assert np.array_equal(golden["broad_pairs_grid"], golden["broad_pairs"])
    xyz, n = golden["radius_xyz"], golden["radius_n"]
    off = np.concatenate([[0], np.cumsum(n)])
    r = np.array([oracle.mesh_radius(xyz[off[i]:off[i + 1]]) for i in range(len(n))], np.float32)
    assert np.array_equal(r.view(np.uint32), golden["radius_out"].view(np.uint32))


def test_broad_phase_oracle_against_reference_random(oracle, reference):
    rng = np.random.default_rng(5)
    for n in (1, 2, 17, 150):
        pos = (rng.random((n, 3)) * 10).astype(np.float32)
        rad = (rng.random(n) * 1.5 + 0.05).astype(np.float32)
        want = reference.broad_pairs(pos, rad, 0)
        assert np.array_equal(oracle.broad_pairs(pos, rad), want)
        assert np.array_equal(reference.broad_pairs(pos, rad, 1), want)


def _rows_equal(a, b):
    # float == (a signed zero equals its opposite, as the reference's `<` treats it)
    return a.shape == b.shape and bool(np.all(a == b))


def test_contact_reduction_oracle_against_golden(oracle, golden):
    rows, bodies = golden["reduce_rows"], golden["reduce_bodies"]
    got_r, got_b, _ = oracle.reduce_contacts(rows, bodies)
    assert _rows_equal(got_r, golden["reduce_out_rows"])
    assert np.array_equal(got_b, golden["reduce_out_bodies"])
    # the fixture exercises every case: removals, chains, signed zeros
    assert len(golden["reduce_out_rows"]) < len(rows)


def test_contact_reduction_oracle_against_reference_random(oracle, reference):
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent / "golden"))
    from make_golden import reduction_rows
    for seed, n_base, nb in ((1, 5, 1), (2, 40, 2), (3, 900, 4), (4, 3000, 1)):
        rows, bodies = reduction_rows(np.random.default_rng(seed), n_base=n_base, n_bodies=nb)
        want_r, want_b = reference.reduce_contacts(rows, bodies)
        got_r, got_b, _ = oracle.reduce_contacts(rows, bodies)
        assert _rows_equal(got_r, want_r) and np.array_equal(got_b, want_b)
