"""Full-size workloads against the CPU oracle (whose pair sets, test counts and
FP32 contacts equal the reference's -- tests/test_oracle.py).

  config 3: 512 uneven pairs (1k-200k tets), k = 14, batched and plain
  config 2: one pair of 64^3-cell jittered lattices (1.57M tets each), k = 26
  config 5: 256 touching pairs of 20^3-cell lattices, contacts bit for bit
  config 4: deforming pairs stepped by a captured CUDA graph, k = 18
"""
import numpy as np
import pytest

import kdop_b200 as kd
from conftest import sorted_rows
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def worlds_of(oracle, sc):
    return [oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]


def device_scene(ctx, sc):
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    return ds


def test_config3_all_pairs(ctx, oracle):
    sc = scenes.config3()
    ds = device_scene(ctx, sc)
    rows, tests_pp, _ = oracle.run_pairs(sc.K, worlds_of(oracle, sc), sc.meshes, sc.pairs)
    want = sorted_rows(rows.astype(np.int64))
    st = ds.traverse_sync(sc.pairs)
    assert st.n_tests == int(tests_pp.sum())
    assert np.array_equal(sorted_rows(ds.candidates().astype(np.int64)), want)
    st_plain = ds.traverse_sync(sc.pairs, ds.opts(mode=kd.TRAVERSE_PLAIN))
    assert st_plain.n_tests == st.n_tests and st_plain.n_candidates == st.n_candidates
    # unfiltered leaf overlaps: the count of every overlapping leaf pair
    st_all = ds.traverse_sync(sc.pairs, ds.opts(surface_filter=0))
    assert st_all.n_candidates == st_all.n_leaf_overlaps >= st.n_candidates


def test_config2_large_pair_k26(ctx, oracle):
    sc = scenes.config2()
    ds = device_scene(ctx, sc)
    w = worlds_of(oracle, sc)
    A, B = sc.meshes
    pairs, tests, leaf_overlaps = oracle.run_pair(26, w[0], A.tets, A.surf, w[1], B.tets, B.surf, restA=A.xyz,
                                                  restB=B.xyz)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    assert st.n_tests == tests and st.n_leaf_overlaps == leaf_overlaps
    got = ds.candidates()
    assert np.array_equal(sorted_rows(got[:, 1:].astype(np.int64)), sorted_rows(pairs.astype(np.int64)))
    # contacts of the candidate set, bit for bit
    ref, _ = oracle.contacts(w[0], A.tets, A.surf, w[1], B.tets, B.surf, got[:, 1:], "f")
    c = ds.read_contacts()
    dev = np.column_stack([c["p"], c["n"], c["depth"][:, None]]).astype(np.float32)
    assert bit_sorted(dev) == bit_sorted(ref[:, :7])


def bit_sorted(a):
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return u[np.lexsort(u.T[::-1])].tobytes()


def test_config5_contacts_bit_exact(ctx, oracle):
    sc = scenes.config5()
    ds = device_scene(ctx, sc)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    cand = ds.candidates()
    c = ds.read_contacts()
    assert st.n_contacts == len(c) > 1000
    w = worlds_of(oracle, sc)
    ref_rows = []
    for p, (a, b) in enumerate(sc.pairs):
        sel = cand[cand[:, 0] == p, 1:]
        A, B = sc.meshes[a], sc.meshes[b]
        r, _ = oracle.contacts(w[a], A.tets, A.surf, w[b], B.tets, B.surf, sel, "f")
        ref_rows.append(r[:, :7])
    ref = np.concatenate(ref_rows)
    dev = np.column_stack([c["p"], c["n"], c["depth"][:, None]]).astype(np.float32)
    assert bit_sorted(dev) == bit_sorted(ref)


def test_config4_graph_steps_match_oracle(ctx, oracle):
    """Deforming pairs advanced by the captured graph (motion + deform refit +
    traversal + contacts): each step's candidates equal the oracle's on the
    device's world positions, and equal an uncaptured step."""
    sc = scenes.config4(n_pairs=6, n=8)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ex = sc.extra
    ds.set_deformation(ex["amp"], float(np.float32(2 * np.pi / ex["L"])), 0.0)
    ds.set_motion(ex["lin_vel"], ex["ang_vel"], ex["phase_rate"])
    ds.refit(kd.REFIT_DEFORM)
    ds.traverse_sync(sc.pairs, contacts=True)
    ds.graph_capture(sc.pairs, refit_mode=kd.REFIT_DEFORM, motion=True)
    v_off = ds.v_off
    for step in range(4):
        ds.graph_launch()
        st = ds.stats()
        got = sorted_rows(ds.candidates().astype(np.int64))
        c_graph = bit_sorted(np.column_stack([ds.read_contacts()[k] for k in ("p", "n")]))
        world = ds.read_vertices()
        rows = []
        tests = 0
        for p, (a, b) in enumerate(sc.pairs):
            A, B = sc.meshes[a], sc.meshes[b]
            pr, t, _ = oracle.run_pair(sc.K, world[v_off[a]:v_off[a + 1]], A.tets, A.surf,
                                       world[v_off[b]:v_off[b + 1]], B.tets, B.surf, restA=A.xyz, restB=B.xyz)
            tests += t
            if len(pr):
                rows.append(np.column_stack([np.full(len(pr), p), pr]))
        want = sorted_rows(np.concatenate(rows).astype(np.int64)) if rows else np.zeros((0, 3), np.int64)
        assert st.n_tests == tests
        assert np.array_equal(got, want)
        # the same state stepped without the graph
        ds.refit(kd.REFIT_DEFORM)
        st2 = ds.traverse_sync(sc.pairs, contacts=True)
        assert st2.n_tests == st.n_tests
        assert np.array_equal(sorted_rows(ds.candidates().astype(np.int64)), got)
        assert bit_sorted(np.column_stack([ds.read_contacts()[k] for k in ("p", "n")])) == c_graph
    ds.graph_release()
