"""Full-size workloads against the reference's own results and the CPU oracle.

The reference's digests (tests/golden/reference_large.json, made by the
compiled reference: node-pair tests, canonical candidate list, canonical FP32
contact rows) pin configs 2, 3 and 5 directly; the oracle (whose results equal
the reference's at these sizes, tests/test_oracle_large.py) checks the states
the reference cannot produce here (config 4's deformed steps).

  config 3: 512 uneven pairs (1k-200k tets), k = 14, batched and plain
  config 2: one pair of 64^3-cell jittered lattices (1.57M tets each), k = 26
  config 5: 256 touching pairs of 20^3-cell lattices, contacts bit for bit
  config 4: 64 deforming pairs of 40^3-cell lattices stepped 200 times by a
            captured CUDA graph, k = 18
"""
import os

import numpy as np
import pytest

import kdop_b200 as kd
from conftest import canonical_candidates, canonical_contacts, digest, sorted_rows
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def worlds_of(oracle, sc):
    return [oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]


def device_scene(ctx, sc):
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    return ds


def device_digests(ds):
    """Canonical candidate and contact digests of the scene's last step."""
    cand = ds.candidates()
    c = ds.read_contacts()
    cc = canonical_candidates(cand[:, 0], cand[:, 1], cand[:, 2])
    ck = canonical_contacts(cand[c["cand"], 0], c["p"], c["n"], c["depth"])
    return cc, ck


def check_reference(ds, st, ref):
    cc, ck = device_digests(ds)
    assert st.n_tests == ref["tests"]
    assert len(cc) == ref["candidates"] and digest(cc) == ref["candidates_sha256"]
    assert len(ck) == ref["contacts"] and digest(ck) == ref["contacts_sha256"]


def test_config3_all_pairs(ctx, oracle, golden_large):
    sc = scenes.config3()
    ds = device_scene(ctx, sc)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    check_reference(ds, st, golden_large["config3"])
    rows, tests_pp, _ = oracle.run_pairs(sc.K, worlds_of(oracle, sc), sc.meshes, sc.pairs,
                                         threads=os.cpu_count() or 1)
    want = sorted_rows(rows.astype(np.int64))
    assert st.n_tests == int(tests_pp.sum())
    assert np.array_equal(sorted_rows(ds.candidates().astype(np.int64)), want)
    st_plain = ds.traverse_sync(sc.pairs, ds.opts(mode=kd.TRAVERSE_PLAIN))
    assert st_plain.n_tests == st.n_tests and st_plain.n_candidates == st.n_candidates
    # unfiltered leaf overlaps: the count of every overlapping leaf pair
    st_all = ds.traverse_sync(sc.pairs, ds.opts(surface_filter=0))
    assert st_all.n_candidates == st_all.n_leaf_overlaps >= st.n_candidates


def test_config2_large_pair_k26(ctx, oracle, golden_large):
    sc = scenes.config2()
    ds = device_scene(ctx, sc)
    w = worlds_of(oracle, sc)
    A, B = sc.meshes
    pairs, tests, leaf_overlaps = oracle.run_pair(26, w[0], A.tets, A.surf, w[1], B.tets, B.surf, restA=A.xyz,
                                                  restB=B.xyz)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    check_reference(ds, st, golden_large["config2"])
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


def test_config5_contacts_bit_exact(ctx, oracle, golden_large):
    sc = scenes.config5()
    ds = device_scene(ctx, sc)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    check_reference(ds, st, golden_large["config5"])
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


def test_config4_meshes_at_rest_poses_k18(ctx, golden_large):
    """Config 4's 64 pairs of 384,000-tet meshes at their initial rigid poses
    (before any deforming step), k = 18: node-pair tests, candidates and
    FP32 contacts equal the reference's own."""
    sc = scenes.config4()
    ds = device_scene(ctx, sc)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    check_reference(ds, st, golden_large["config4"])
    ds.close()


def oracle_step(oracle, sc, world, v_off):
    """Candidates (pair, a, b) and node-pair tests of the oracle on the given
    world positions, trees built on the rest positions."""
    worlds = [world[v_off[i]:v_off[i + 1]] for i in range(len(sc.meshes))]
    rows, tests_pp, _ = oracle.run_pairs(sc.K, worlds, sc.meshes, sc.pairs, threads=os.cpu_count() or 1)
    return sorted_rows(rows.astype(np.int64)), int(tests_pp.sum()), worlds


def test_config4_full_size_200_graph_steps(ctx, oracle):
    """Config 4 at its stated size: 64 pairs of 40^3-cell lattices (384,000
    tets each), k = 18, 200 steps of motion + deformation + refit + traversal
    + contacts, each step one launch of the captured CUDA graph.  At steps 0,
    1, 50, 100 and 199 the candidates and node-pair tests equal the oracle's
    on the device's own world positions (trees built on the rest positions);
    at steps 0 and 199 the FP32 contacts equal the oracle's bit for bit."""
    sc = scenes.config4()
    assert len(sc.pairs) == 64 and all(m.n_tets == 384000 for m in sc.meshes) and sc.K == 18
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ex = sc.extra
    ds.set_deformation(ex["amp"], float(np.float32(2 * np.pi / ex["L"])), 0.0)
    ds.set_motion(ex["lin_vel"], ex["ang_vel"], ex["phase_rate"])
    ds.refit(kd.REFIT_DEFORM)
    st0 = ds.traverse_sync(sc.pairs, contacts=True)
    ds.reserve(candidates=4 * st0.n_candidates + 4096, contacts=4 * st0.n_contacts + 4096,
               queue=max(2 * st0.queue_used, 1 << 20))
    ds.graph_capture(sc.pairs, refit_mode=kd.REFIT_DEFORM, motion=True)
    v_off = ds.v_off
    checks = {0, 1, 50, 100, 199}
    contact_checks = {0, 199}
    checked = 0
    for step in range(200):
        ds.graph_launch()
        if step not in checks:
            continue
        st = ds.stats()
        assert st.status == 0 and st.device_error == 0
        got = sorted_rows(ds.candidates().astype(np.int64))
        world = ds.read_vertices()
        want, tests, worlds = oracle_step(oracle, sc, world, v_off)
        assert st.n_tests == tests, step
        assert np.array_equal(got, want), step
        assert len(got) > 0
        if step in contact_checks:
            cand = ds.candidates()
            c = ds.read_contacts()
            dev = canonical_contacts(cand[c["cand"], 0], c["p"], c["n"], c["depth"])
            parts = []
            for p, (a, b) in enumerate(sc.pairs):
                sel = cand[cand[:, 0] == p, 1:]
                if len(sel) == 0:
                    continue
                A, B = sc.meshes[a], sc.meshes[b]
                r, _ = oracle.contacts(worlds[a], A.tets, A.surf, worlds[b], B.tets, B.surf, sel, "f")
                parts.append(canonical_contacts(np.full(len(r), p), r[:, 0:3], r[:, 3:6], r[:, 6]))
            ref = np.concatenate(parts)
            ref = ref[np.lexsort(ref.T[::-1])]
            assert len(dev) == len(ref) > 0, step
            assert dev.tobytes() == ref.tobytes(), step
        checked += 1
    assert checked == len(checks)
    ds.graph_release()
    ds.close()


def fp64_check_all_rows(oracle, sc, ds, worlds):
    """Every contact row of the scene's last step against the FP64 oracle.

    Frozen decisions: the FP64 depth and normal evaluated with the FP32 run's
    discrete decisions (contact face, extreme candidates) for every row.  The
    error of a depth, a difference of dot products p.n, scales with the
    magnitude of its operands, so it is taken relative to max(|depth|,
    largest |coordinate| of the pair's eight vertices); the normal is a unit
    vector.  Unfrozen: the plain FP64 contacts on the pairs whose discrete
    decisions agree with the FP32 run (edge/face crossings lie on their own
    plane, so the inside test is decided by rounding and the precisions
    often keep different candidate sets); returns (agreeing pairs, pairs with
    contacts, worst frozen depth error, worst frozen normal error)."""
    cand = ds.candidates()
    c = ds.read_contacts()
    worst_d = worst_n = 0.0
    agree = with_c = 0
    n_rows = 0
    for p, (a, b) in enumerate(sc.pairs):
        k = np.nonzero(cand[c["cand"], 0] == p)[0]
        if len(k) == 0:
            continue
        A, B = sc.meshes[a], sc.meshes[b]
        ci = c["cand"][k]
        sel_rows = np.unique(ci)
        sel = cand[sel_rows, 1:]
        _, rec32 = oracle.contacts(worlds[a], A.tets, A.surf, worlds[b], B.tets, B.surf, sel, "f")
        r64, rec64 = oracle.contacts(worlds[a], A.tets, A.surf, worlds[b], B.tets, B.surf, sel, "d")
        local = np.searchsorted(sel_rows, ci)
        a12 = worlds[a][A.tets[sel[local, 0]]].astype(np.float64).reshape(-1, 12)
        b12 = worlds[b][B.tets[sel[local, 1]]].astype(np.float64).reshape(-1, 12)
        d64, n64 = oracle.frozen_batch(a12, b12, rec32[local])
        scale = np.maximum(np.abs(d64), np.maximum(np.abs(a12).max(1), np.abs(b12).max(1)))
        ed = np.abs(c["depth"][k].astype(np.float64) - d64) / scale
        en = np.abs(c["n"][k].astype(np.float64) - n64).max(1)
        worst_d, worst_n = max(worst_d, float(ed.max())), max(worst_n, float(en.max()))
        n_rows += len(k)
        same = ((rec32["face_a"] == rec64["face_a"]) & (rec32["face_b"] == rec64["face_b"])
                & (rec32["overlap"] == rec64["overlap"]) & (rec32["cand_mask"] == rec64["cand_mask"]))
        with_c += len(sel_rows)
        # first row of each candidate on both sides (depth and normal are the
        # same for every row of a candidate)
        j_dev, first_dev = np.unique(local, return_index=True)
        j_64, first_64 = np.unique(r64[:, 7].astype(np.int64), return_index=True)
        both = np.intersect1d(j_dev[same[j_dev]], j_64)
        if len(both):
            gd = k[first_dev[np.searchsorted(j_dev, both)]]
            fd = first_dev[np.searchsorted(j_dev, both)]
            r = r64[first_64[np.searchsorted(j_64, both)]]
            sc_j = np.maximum(np.abs(r[:, 6]), scale[fd])
            assert (np.abs(c["depth"][gd].astype(np.float64) - r[:, 6]) <= 1e-5 * sc_j).all()
            assert (np.abs(c["n"][gd].astype(np.float64) - r[:, 3:6]) <= 1e-5).all()
            agree += len(both)
    assert n_rows == len(c)
    return agree, with_c, worst_d, worst_n


@pytest.mark.parametrize("name", ["config5", "config2"])
def test_contacts_within_1e5_of_fp64_at_full_size(ctx, oracle, name):
    """Every contact row of full config 5 (3.5 M rows) and config 2 within
    1e-5 relative of the FP64 oracle (see fp64_check_all_rows)."""
    sc = scenes.config5() if name == "config5" else scenes.config2()
    ds = device_scene(ctx, sc)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    assert st.n_contacts > 1000
    agree, with_c, worst_d, worst_n = fp64_check_all_rows(oracle, sc, ds, worlds_of(oracle, sc))
    print(f"{name}: {st.n_contacts} rows, frozen FP64 worst depth error {worst_d:.3g}, normal {worst_n:.3g}; "
          f"decisions agree on {agree} of {with_c} pairs with contacts")
    assert worst_d <= 1e-5 and worst_n <= 1e-5
    assert agree > 0
