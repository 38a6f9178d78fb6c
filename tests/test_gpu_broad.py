"""kdop_broad_phase against the oracle's restatement of the reference's
broad phase (pinned to the reference by tests/test_oracle.py)."""
import numpy as np
import pytest

import kdop_b200 as kd
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def radii(oracle, meshes):
    return np.array([oracle.mesh_radius(m.xyz) for m in meshes], np.float32)


def test_broad_phase_matches_oracle(ctx, oracle):
    sc = scenes.config3(n_pairs=96, seed=4)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    rng = np.random.default_rng(3)
    r = radii(oracle, sc.meshes)
    for trial in range(3):
        pos = (rng.random((len(sc.meshes), 3)) * 400).astype(np.float32)
        got = ds.broad_phase(pos)
        want = oracle.broad_pairs(pos, r)
        assert len(want) > 0
        assert np.array_equal(got, want)


def test_broad_phase_from_poses_and_touching_boxes(ctx, oracle):
    sc = scenes.small_batch(n_pairs=12, seed=8)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    r = radii(oracle, sc.meshes)
    # boxes that touch exactly along x count as overlapping (strict <)
    pos = np.zeros((len(sc.meshes), 3), np.float32)
    pos[:, 0] = np.cumsum(np.concatenate([[0], r[:-1] + r[1:]])).astype(np.float32)
    want = oracle.broad_pairs(pos, r)
    ds.set_poses(sc.quat, pos)
    got = ds.broad_phase()  # positions of set_poses
    assert np.array_equal(got, want)
    assert np.array_equal(ds.broad_phase(pos), want)


def test_broad_phase_feeds_the_traversal(ctx, oracle):
    sc = scenes.config5(n_pairs=16, n=8, seed=2)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    pairs = ds.broad_phase()
    want = oracle.broad_pairs(sc.pos, radii(oracle, sc.meshes))
    assert np.array_equal(pairs, want)
    st = ds.traverse_sync(pairs, contacts=True)
    assert st.n_contacts > 0
