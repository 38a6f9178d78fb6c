"""kdop_sort_results: the device sort that puts a traversal's results in a
reproducible order (candidates by (pair, tet A, tet B), contacts grouped by
candidate in that order), checked against the unsorted output of the same
run, across repeated runs, and through the adjoint."""
import numpy as np
import pytest

import kdop_b200 as kd
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def run(ctx, sc, contacts=True, sort=True):
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ds.traverse_sync(sc.pairs, contacts=contacts)
    cand0 = ds.candidates().copy()
    rows0 = ds.read_contacts().copy() if contacts else None
    if sort:
        ds.sort_results()
    return ds, cand0, rows0


def row_bits(rows):
    return np.column_stack([rows["p"].view(np.uint32), rows["n"].view(np.uint32),
                            rows["depth"].view(np.uint32)[:, None]])


def check_sorted(ds, cand0, rows0):
    cand = ds.candidates()
    order = np.lexsort((cand0[:, 2], cand0[:, 1], cand0[:, 0]))
    assert np.array_equal(cand, cand0[order]), "candidate rows not in (pair, tet A, tet B) order"
    if rows0 is None:
        return cand, None
    rows = ds.read_contacts()
    assert len(rows) == len(rows0)
    c = rows["cand"].astype(np.int64)
    assert np.all(np.diff(c) >= 0), "contact rows not grouped by candidate in order"
    # rows of sorted candidate k == rows of its original candidate, in order
    new_of_old = np.empty(len(order), np.int64)
    new_of_old[order] = np.arange(len(order))
    c0 = new_of_old[rows0["cand"].astype(np.int64)]
    perm0 = np.argsort(c0, kind="stable")  # original rows, grouped by new index, generation order kept
    assert np.array_equal(c0[perm0], c)
    assert np.array_equal(row_bits(rows0)[perm0], row_bits(rows))
    return cand, rows


def test_sorted_results_contact_rich(ctx):
    sc = scenes.config5(n_pairs=24, n=12, seed=9)
    ds, cand0, rows0 = run(ctx, sc)
    assert len(rows0) > 100
    check_sorted(ds, cand0, rows0)


def test_sorted_candidates_many_tiles(ctx):
    # > 100k candidates: many radix tiles and a two-level scan
    sc = scenes.config3(n_pairs=24, seed=5)
    ds, cand0, rows0 = run(ctx, sc)
    assert len(cand0) > 100_000
    check_sorted(ds, cand0, rows0)


def test_sort_without_contacts(ctx):
    sc = scenes.small_batch(n_pairs=6, seed=3)
    ds, cand0, _ = run(ctx, sc, contacts=False)
    check_sorted(ds, cand0, None)


def test_sorted_results_are_reproducible(ctx):
    sc = scenes.config5(n_pairs=16, n=10, seed=2)
    out = []
    for _ in range(2):
        ds, _, _ = run(ctx, sc)
        out.append((ds.candidates(), row_bits(ds.read_contacts()), ds.read_contacts()["cand"]))
        ds.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_adjoint_unchanged_by_sorting(ctx):
    sc = scenes.config5(n_pairs=8, n=10, seed=6)
    grads = []
    for sort in (False, True):
        ds, _, _ = run(ctx, sc, sort=sort)
        rows = ds.read_contacts()
        dd = np.ascontiguousarray(2.0 * rows["depth"], np.float32)  # L = sum of depth^2
        dn = np.zeros((len(rows), 3), np.float32)
        g = np.zeros((sum(m.n_verts for m in sc.meshes), 3), np.float32)
        ds.adjoint(dd, dn, g)
        grads.append(g)
        ds.close()
    gmax = np.abs(grads[0]).max()
    assert gmax > 0
    # The adjoint adds each contact's contribution to its vertices with float
    # atomics, in whatever order the threads arrive (sorting the rows changes
    # it): a vertex's sum of contributions of opposite sign keeps a rounding
    # error of a few float epsilons of its largest terms, so the absolute
    # tolerance scales with the largest gradient.  A contact attached to the
    # wrong vertices would move entries by about the contributions themselves.
    np.testing.assert_allclose(grads[1], grads[0], rtol=1e-5, atol=1e-5 * gmax)


def test_sort_with_no_candidates(ctx):
    sc = scenes.touching_pair(n=4, seed=1)
    sc.pos = sc.pos.copy()
    sc.pos[1] += np.float32([100.0, 0.0, 0.0])
    ds, cand0, rows0 = run(ctx, sc)
    assert len(cand0) == 0 and len(rows0) == 0
    assert len(ds.candidates()) == 0
