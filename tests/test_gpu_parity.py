"""CUDA library (through its C ABI) against the CPU oracle / golden fixtures.

Bars: node volumes, candidate pair sets and node-pair test counts bit-exact /
exact; FP32 contacts bit-exact against the reference's FP32 path; contact
depths and normals within 1e-5 relative of the FP64 oracle on pairs whose
discrete decisions agree.
"""
import numpy as np
import pytest

import kdop_b200 as kd
from conftest import sorted_rows, world_xyz
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def oracle_tree(oracle, K, rest, world, tets):
    """Tree built on the rest positions, refitted on the world positions, in preorder."""
    perm = oracle.morton_order(rest, tets)
    left, right, tet = oracle.build_tree(perm)
    vol = oracle.refit(K, world, tets, left, right, tet)
    order, leaf = [], []
    stack = [0]
    while stack:
        i = stack.pop()
        order.append(i)
        leaf.append(tet[i] if left[i] < 0 else -1)
        if left[i] >= 0:
            stack += [right[i], left[i]]
    return vol[order], np.array(leaf)


def scene_world(oracle, sc):
    return [world_xyz(oracle, sc, i) for i in range(len(sc.meshes))]


def oracle_pairs(oracle, sc, worlds, filt=True):
    rows, tests = [], 0
    for pi, (a, b) in enumerate(sc.pairs):
        A, B = sc.meshes[a], sc.meshes[b]
        sa = A.surf if filt else np.full(A.n_tets, 15, np.uint8)
        sb = B.surf if filt else np.full(B.n_tets, 15, np.uint8)
        p, t, _ = oracle.run_pair(sc.K, worlds[a], A.tets, sa, worlds[b], B.tets, sb, restA=A.xyz, restB=B.xyz)
        tests += t
        if len(p):
            rows.append(np.column_stack([np.full(len(p), pi, np.uint32), p]))
    rows = np.concatenate(rows) if rows else np.zeros((0, 3), np.uint32)
    return sorted_rows(rows), tests


@pytest.mark.parametrize("K", scenes.SUPPORTED_K)
def test_refit_bit_exact_all_K(ctx, oracle, K):
    rng = np.random.default_rng(K)
    m = scenes.lattice(5, 0.2, rng)
    q = scenes.random_quaternion(rng)
    p = np.float32([0.5, -1.0, 2.0])
    sc = kd.DeviceScene(ctx, K, [m])
    # vertices mode
    xw = oracle.rotate(q, p, m.xyz)
    sc.set_vertices(xw)
    sc.refit(kd.REFIT_VERTICES)
    vol, tet = sc.read_tree(0)
    ovol, oleaf = oracle_tree(oracle, K, m.xyz, xw, m.tets)
    assert np.array_equal(tet, oleaf)
    assert vol.tobytes() == ovol.tobytes()
    # fused pose mode gives the same bits
    sc.set_poses(q[None, :], p[None, :])
    sc.refit(kd.REFIT_POSE)
    vol2, _ = sc.read_tree(0)
    assert vol2.tobytes() == ovol.tobytes()
    assert sc.read_vertices().tobytes() == xw.tobytes()


def test_refit_deform_mode_bit_exact(ctx, oracle):
    m = scenes.lattice(4)
    q = scenes.axis_angle_quaternion([1, 2, 3], 0.3)
    p = np.float32([0.1, 0.2, 0.3])
    sc = kd.DeviceScene(ctx, 18, [m])
    sc.set_poses(q[None], p[None])
    amp, w, phase = 0.1, np.float32(2 * np.pi / 4), 0.35
    sc.set_deformation(amp, float(w), phase)
    sc.refit(kd.REFIT_DEFORM)
    xw = oracle.rotate(q, p, oracle.deform(amp, float(w), phase, m.xyz))
    assert sc.read_vertices().tobytes() == xw.tobytes()
    vol, _ = sc.read_tree(0)
    ovol, _ = oracle_tree(oracle, 18, m.xyz, xw, m.tets)
    assert vol.tobytes() == ovol.tobytes()


def test_config1_against_golden(ctx, oracle, golden):
    sc = scenes.config1()
    ds = kd.DeviceScene(ctx, 14, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    for mode in (kd.TRAVERSE_BATCHED, kd.TRAVERSE_PLAIN):
        st = ds.traverse_sync(sc.pairs, ds.opts(mode=mode))
        rows = ds.candidates()
        assert np.array_equal(sorted_rows(rows[:, 1:]), golden["c1_pairs"])
        assert st.n_tests == int(golden["c1_tests"])
    vol, tet = ds.read_tree(0)
    assert np.array_equal(tet, golden["c1_leafA"])
    assert vol[:64].tobytes() == golden["c1_volA_head"].tobytes()


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 4])
def test_touching_pairs_contacts_bit_exact(ctx, oracle, golden, seed):
    key = f"t{seed}"
    K = int(golden[f"{key}_K"])
    sc = scenes.touching_pair(n=4, seed=seed, K=K)
    ds = kd.DeviceScene(ctx, K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    assert st.n_tests == int(golden[f"{key}_tests"])
    rows = ds.candidates()
    ref_pairs = golden[f"{key}_pairs_trav"]
    assert np.array_equal(sorted_rows(rows[:, 1:]), sorted_rows(ref_pairs))
    # contacts: group the device rows by candidate, order candidates as the
    # reference's traversal visited them, then compare bit for bit
    c = ds.read_contacts()
    cand = rows[c["cand"], 1:]
    index = {(int(a), int(b)): i for i, (a, b) in enumerate(ref_pairs)}
    order = np.array([index[(int(a), int(b))] for a, b in cand])
    perm = np.lexsort((np.arange(len(c)), order))
    dev = np.column_stack([c["p"], c["n"], c["depth"][:, None], order[:, None].astype(np.float32)])[perm]
    ref = golden[f"{key}_contacts_f32"]
    assert dev.shape == ref.shape
    assert dev.tobytes() == ref.tobytes()
    A, B = sc.meshes
    check_against_fp64(oracle, dev, golden[f"{key}_contacts_f64"], golden[f"{key}_xyzA"], A, golden[f"{key}_xyzB"],
                       B, ref_pairs)


def test_contacts_use_the_positions_of_the_last_refit(ctx):
    """After a pose refit, contacts (and the adjoint) read the world positions
    that refit computed -- the ones the traversal saw -- so a pose change
    between refit and kdop_contacts does not mix two poses; the same rows come
    back as from the world positions uploaded and refitted in vertex mode."""
    sc = scenes.touching_pair(n=4, seed=2, K=14)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.reserve(candidates=1 << 16, contacts=1 << 16)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ds.traverse(sc.pairs)
    moved = sc.pos.copy()
    moved[1] += np.float32(0.25)
    ds.set_poses(sc.quat, moved)  # not refitted: the contacts keep the refit's poses
    ds.contacts()
    assert ds.stats().status == 0
    posed = ds.read_contacts()
    assert len(posed) > 0
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    world = ds.read_vertices()
    ds2 = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds2.set_vertices(world)
    ds2.refit(kd.REFIT_VERTICES)
    ds2.traverse_sync(sc.pairs, contacts=True)
    ref = ds2.read_contacts()
    def rows(c):
        return sorted(np.column_stack([c["p"], c["n"], c["depth"][:, None]]).astype(np.float32).view(np.uint32)
                      .reshape(len(c), -1).tolist())
    assert rows(posed) == rows(ref)
    ds.close()
    ds2.close()


def test_pose_graph_before_its_first_launch(ctx, oracle):
    """A scene whose pose-mode step is captured but not yet launched has no
    posed vertices from a refit: reading them poses the vertices with the
    current poses, and the first launch gives the rows of a plain pose refit."""
    sc = scenes.touching_pair(n=4, seed=3, K=14)
    ref = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ref.reserve(candidates=1 << 16, contacts=1 << 16)
    ref.set_poses(sc.quat, sc.pos)
    ref.refit(kd.REFIT_POSE)
    ref.traverse_sync(sc.pairs, contacts=True)
    want = ref.read_contacts()
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.reserve(candidates=1 << 16, contacts=1 << 16)
    ds.set_poses(sc.quat, sc.pos)
    ds.graph_capture(sc.pairs, refit_mode=kd.REFIT_POSE)
    xw = np.concatenate([oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)])
    assert ds.read_vertices().tobytes() == np.ascontiguousarray(xw, np.float32).tobytes()
    ds.graph_launch()
    assert ds.stats().status == 0
    got = ds.read_contacts()
    def rows(c):
        return sorted(np.column_stack([c["p"], c["n"], c["depth"][:, None]]).astype(np.float32).view(np.uint32)
                      .reshape(len(c), -1).tolist())
    assert len(want) > 0 and rows(got) == rows(want)
    ds.graph_release()
    ds.close()
    ref.close()


def test_pose_graph_capture_after_an_earlier_pose_refit(ctx, oracle):
    """A direct pose refit, then a pose change, then the capture of a pose
    step: before the first launch the vertices read back are posed with the
    current poses (not the earlier refit's), and the first launch gives the
    rows of a plain pose refit at those poses."""
    sc = scenes.touching_pair(n=4, seed=6, K=14)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.reserve(candidates=1 << 16, contacts=1 << 16)
    old = sc.pos.copy()
    old[1] += np.float32(0.3)
    ds.set_poses(sc.quat, old)
    ds.refit(kd.REFIT_POSE)
    ds.set_poses(sc.quat, sc.pos)
    ds.graph_capture(sc.pairs, refit_mode=kd.REFIT_POSE)
    xw = np.concatenate([oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)])
    assert ds.read_vertices().tobytes() == np.ascontiguousarray(xw, np.float32).tobytes()
    ds.graph_launch()
    assert ds.stats().status == 0
    ref = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ref.reserve(candidates=1 << 16, contacts=1 << 16)
    ref.set_poses(sc.quat, sc.pos)
    ref.refit(kd.REFIT_POSE)
    ref.traverse_sync(sc.pairs, contacts=True)
    assert len(ref.read_contacts()) > 0
    assert contact_rows(ds.read_contacts()) == contact_rows(ref.read_contacts())
    ds.graph_release()
    ds.close()
    ref.close()


def test_graph_launch_restores_the_graph_refit_mode(ctx):
    """Capture a pose step, refit other positions directly in vertex mode, then
    launch the graph: the contacts, the vertices read back and the adjoint all
    follow the graph's pose step, as after a plain pose refit."""
    import torch
    sc = scenes.touching_pair(n=4, seed=7, K=14)
    ref = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ref.reserve(candidates=1 << 16, contacts=1 << 16)
    ref.set_poses(sc.quat, sc.pos)
    ref.refit(kd.REFIT_POSE)
    ref.traverse_sync(sc.pairs, contacts=True)
    want = ref.read_contacts()
    assert len(want) > 0
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.reserve(candidates=1 << 16, contacts=1 << 16)
    ds.set_poses(sc.quat, sc.pos)
    ds.graph_capture(sc.pairs, refit_mode=kd.REFIT_POSE)
    other = np.concatenate([m.xyz for m in sc.meshes]) + np.float32(0.05)
    ds.set_vertices(other)
    ds.refit(kd.REFIT_VERTICES)
    ds.graph_launch()
    assert ds.stats().status == 0
    got = ds.read_contacts()
    assert contact_rows(got) == contact_rows(want)
    assert ds.read_vertices().tobytes() == ref.read_vertices().tobytes()

    def grad(scene, rows):
        n = len(rows)
        dd = torch.tensor(2.0 * rows["depth"], device="cuda")
        dn = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        g = torch.zeros((int(scene.v_off[-1]), 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        scene.adjoint(dd, dn, g)
        scene.ctx.synchronize()
        return g.cpu().numpy().astype(np.float64)

    # same rows in the same order (one traversal state each): the gradients
    # differ only by the arrival order of float atomics
    gr, gd = grad(ref, want), grad(ds, got)
    scale = max(np.abs(gr).max(), 1e-30)
    assert np.abs(gr).max() > 0
    assert np.abs(gd - gr).max() <= 1e-5 * scale
    ds.graph_release()
    ds.close()
    ref.close()


def contact_rows(c):
    return sorted(np.column_stack([c["p"], c["n"], c["depth"][:, None]]).astype(np.float32).view(np.uint32)
                  .reshape(len(c), -1).tolist())


def check_against_fp64(oracle, dev_rows, ref64_rows, xa, A, xb, B, pairs):
    """Device FP32 contacts vs the FP64 oracle on the pairs whose discrete
    decisions (overlap, chosen faces, set of generated contact candidates)
    agree between FP32 and FP64.  Edge/face-plane crossing candidates lie on
    their own plane, so the reference's inside test decides them by rounding
    and the two precisions often keep different candidate sets; where they
    keep the same set, depth and normal must agree within 1e-5 relative to
    max(|depth|, one lattice cell)."""
    _, rec32 = oracle.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, pairs, "f")
    _, rec64 = oracle.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, pairs, "d")
    same = ((rec32["face_a"] == rec64["face_a"]) & (rec32["face_b"] == rec64["face_b"])
            & (rec32["overlap"] == rec64["overlap"]) & (rec32["cand_mask"] == rec64["cand_mask"]))
    g32, g64 = {}, {}
    for row in dev_rows:
        g32.setdefault(int(row[7]), []).append(row)
    for row in ref64_rows:
        g64.setdefault(int(row[7]), []).append(row)
    with_contacts = [p for p in g32]
    agree = [p for p in with_contacts if same[p] and p in g64]
    for p in agree:
        a, b = np.array(g32[p], np.float64), np.array(g64[p])
        scale = max(1.0, abs(b[0, 6]))
        assert abs(a[0, 6] - b[0, 6]) <= 1e-5 * scale
        assert np.abs(a[0, 3:6] - b[0, 3:6]).max() <= 1e-5
    # Every contact-producing pair: the FP64 depth and normal evaluated with
    # the FP32 run's discrete decisions (face, extreme candidates) frozen.
    ta, tb = A.tets[pairs[:, 0]], B.tets[pairs[:, 1]]
    for p in with_contacts:
        a12 = xa[ta[p]].astype(np.float64).ravel()
        b12 = xb[tb[p]].astype(np.float64).ravel()
        d64, n64 = oracle.frozen_depth(a12, b12, rec32[p])
        row = np.array(g32[p][0], np.float64)
        assert abs(row[6] - d64) <= 1e-5 * max(1.0, abs(d64)), (p, row[6], d64)
        assert np.abs(row[3:6] - n64).max() <= 1e-5, (p, row[3:6], n64)
    return len(agree), len(with_contacts)


@pytest.mark.parametrize("K", [6, 14, 26])
def test_small_batch_batched_equals_plain_equals_oracle(ctx, oracle, K):
    sc = scenes.small_batch(n_pairs=12, seed=K, K=K)
    worlds = scene_world(oracle, sc)
    ds = kd.DeviceScene(ctx, K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ref_rows, ref_tests = oracle_pairs(oracle, sc, worlds)
    # the reference counts one root test per pair and then tests the root pair
    # again in the recursion; the oracle does the same
    for mode in (kd.TRAVERSE_BATCHED, kd.TRAVERSE_PLAIN):
        st = ds.traverse_sync(sc.pairs, ds.opts(mode=mode))
        assert st.n_tests == ref_tests
        assert np.array_equal(sorted_rows(ds.candidates()), ref_rows)


def test_surface_filter_off_matches_unfiltered_oracle(ctx, oracle):
    sc = scenes.small_batch(n_pairs=6, seed=3)
    worlds = scene_world(oracle, sc)
    ds = kd.DeviceScene(ctx, 14, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    st = ds.traverse_sync(sc.pairs, ds.opts(surface_filter=0))
    ref_rows, _ = oracle_pairs(oracle, sc, worlds, filt=False)
    assert st.n_leaf_overlaps == len(ref_rows) == st.n_candidates
    assert np.array_equal(sorted_rows(ds.candidates()), ref_rows)


@pytest.mark.parametrize("cfg", [dict(block_warps=4, stack_cap=64, donate_min=8, load_group=1),
                                 dict(block_warps=16, stack_cap=1024, init_chunk=4, donate_min=128, load_group=4),
                                 dict(block_warps=2, stack_cap=128, init_chunk=32, donate_min=16, load_group=2),
                                 dict(block_warps=8, stack_cap=256, load_group=4),
                                 dict(wave_pairs=3, smem_carveout=50, load_group=4),
                                 dict(wave_pairs=1, smem_carveout=100, stack_cap=128)])
def test_tuning_knobs_do_not_change_results(ctx, oracle, cfg):
    sc = scenes.small_batch(n_pairs=10, n_lo=3, n_hi=7, seed=21)
    worlds = scene_world(oracle, sc)
    ds = kd.DeviceScene(ctx, 14, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ref_rows, ref_tests = oracle_pairs(oracle, sc, worlds)
    st = ds.traverse_sync(sc.pairs, ds.opts(**cfg))
    assert st.n_tests == ref_tests
    assert np.array_equal(sorted_rows(ds.candidates()), ref_rows)


def test_capacity_overflow_reports_and_retries(ctx, oracle):
    sc = scenes.small_batch(n_pairs=4, seed=9)
    ds = kd.DeviceScene(ctx, 14, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ds.traverse(sc.pairs)
    full = ds.stats()
    assert full.n_candidates > 16
    rows = sorted_rows(ds.candidates())
    # tiny candidate and queue buffers: the call reports the required size
    ds.set_capacity(candidates=8, queue=2)
    ds.traverse(sc.pairs, ds.opts(stack_cap=64, donate_min=8))
    st = ds.stats(check=False)
    assert st.status == kd.lib.ERR_CAPACITY
    assert st.n_candidates == full.n_candidates or st.device_error & 2
    st = ds.traverse_sync(sc.pairs, ds.opts(stack_cap=64, donate_min=8), max_retries=12)
    assert st.n_candidates == full.n_candidates and st.n_tests == full.n_tests
    assert np.array_equal(sorted_rows(ds.candidates()), rows)


def test_contact_capacity_overflow(ctx):
    sc = scenes.touching_pair(n=3, seed=1)
    ds = kd.DeviceScene(ctx, 14, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    ref = ds.read_contacts()
    assert st.n_contacts > 8
    ds.set_capacity(contacts=4)
    ds.traverse(sc.pairs)
    ds.contacts()
    st2 = ds.stats(check=False)
    assert st2.status == kd.lib.ERR_CAPACITY and st2.n_contacts == st.n_contacts
    ds.traverse_sync(sc.pairs, contacts=True)
    got = ds.read_contacts()
    assert len(got) == len(ref)


def test_edge_cases_empty_and_single_tet(ctx, oracle):
    one = scenes.Mesh(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]), np.uint32([[0, 1, 2, 3]]),
                      np.uint8([15]))
    empty = scenes.Mesh(np.zeros((0, 3), np.float32), np.zeros((0, 4), np.uint32), np.zeros(0, np.uint8))
    big = scenes.lattice(2)
    ds = kd.DeviceScene(ctx, 14, [one, empty, big, one])
    xyz = np.concatenate([one.xyz, empty.xyz, big.xyz - 0.5, one.xyz + np.float32([0.25, 0.25, 0.25])])
    ds.set_vertices(xyz)
    ds.refit(kd.REFIT_VERTICES)
    # no pairs at all
    st = ds.traverse_sync(np.zeros((0, 2), np.uint32))
    assert st.n_tests == 0 and st.n_candidates == 0
    # empty mesh pairs do nothing; leaf-leaf roots; leaf vs tree
    pairs = np.uint32([[0, 1], [1, 2], [0, 3], [3, 2], [2, 0]])
    st = ds.traverse_sync(pairs)
    rows = sorted_rows(ds.candidates())
    ref = []
    tests = 0
    meshes = [one, empty, big, one]
    offs = np.cumsum([0] + [m.n_verts for m in meshes])
    for pi, (a, b) in enumerate(pairs):
        A, B = meshes[a], meshes[b]
        if A.n_tets == 0 or B.n_tets == 0:
            continue
        p, t, _ = oracle.run_pair(14, xyz[offs[a]:offs[a + 1]], A.tets, A.surf, xyz[offs[b]:offs[b + 1]], B.tets,
                                  B.surf, restA=A.xyz, restB=B.xyz)
        tests += t
        ref += [(pi, x, y) for x, y in p]
    assert st.n_tests == tests
    assert np.array_equal(rows, sorted_rows(np.array(ref, np.uint32).reshape(-1, 3)))


def test_invalid_arguments_are_errors_not_crashes(ctx):
    m = scenes.lattice(1)
    with pytest.raises(kd.KdopError):
        kd.DeviceScene(ctx, 10, [m])  # unsupported K
    bad = scenes.Mesh(m.xyz, m.tets.copy(), m.surf)
    bad.tets[0, 0] = 999
    with pytest.raises(kd.KdopError):
        kd.DeviceScene(ctx, 14, [bad])
    ds = kd.DeviceScene(ctx, 14, [m, m])
    with pytest.raises(kd.KdopError):
        ds.traverse(np.uint32([[0, 5]]))  # mesh index out of range
    with pytest.raises(kd.KdopError):
        ds.set_vertices(np.zeros((3, 3), np.float32))  # wrong vertex count
    with pytest.raises(kd.KdopError):
        ds.refit(7)
    with pytest.raises(kd.KdopError):
        ds.traverse(np.uint32([[0, 1]]), ds.opts(stack_cap=100))  # not a power of two
