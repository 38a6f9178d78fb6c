"""Failure detection on the GPU without a GPU fault: every device-side wait of
the traversal is bounded.  The test hook `test_stuck_work` leaves work units
outstanding that no warp will ever complete (a counter nothing brings to
zero), so the waiting warps give up after `timeout_ms`; the call must report
KDOP_ERR_TIMEOUT within a bounded time and the context must stay usable."""
import time

import numpy as np
import pytest

import kdop_b200 as kd
from kdop_b200 import lib, scenes

pytestmark = pytest.mark.gpu


def sorted_cand(ds):
    c = ds.candidates()
    return c[np.lexsort((c[:, 2], c[:, 1], c[:, 0]))]


@pytest.mark.parametrize("mode", [kd.TRAVERSE_BATCHED, kd.TRAVERSE_PLAIN])
def test_stuck_work_times_out_and_context_recovers(ctx, mode):
    sc = scenes.small_batch(n_pairs=6, seed=12)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    good = ds.traverse_sync(sc.pairs, ds.opts(mode=mode))
    want = sorted_cand(ds)

    t0 = time.perf_counter()
    ds.traverse(sc.pairs, ds.opts(mode=mode, test_stuck_work=1, timeout_ms=200))
    st = ds.stats(check=False)
    elapsed = time.perf_counter() - t0
    assert st.status == lib.ERR_TIMEOUT
    assert st.device_error & 1
    # every wait gave up after its limit: bounded, far below a hang
    assert elapsed < 30.0

    # the scene (and the context) keep working: same results as before
    again = ds.traverse_sync(sc.pairs, ds.opts(mode=mode))
    assert again.n_tests == good.n_tests
    assert np.array_equal(sorted_cand(ds), want)


def test_stuck_work_is_rejected_outside_its_range(ctx):
    sc = scenes.small_batch(n_pairs=2, seed=1)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    with pytest.raises(kd.KdopError):
        ds.traverse(sc.pairs, ds.opts(test_stuck_work=-1))
