"""The project's traversal autotuner (kdop_autotune).

Its choice must lie in the documented knob sets, traversing with it must give
the oracle's candidates and node-pair tests (launch shapes change only the
schedule, never the result), and the choice is cached: for the tuned scene
and, on the same context, for another scene of the same K and size class
(floor(log2) of its total tet count), but not for a scene of another class.
"""
import numpy as np
import pytest

import kdop_b200 as kd
from conftest import sorted_rows, world_xyz
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu

KNOBS = {"block_warps": {4, 8, 16}, "stack_cap": {128, 256, 512, 1024}, "load_group": {1, 2, 4, 8},
         "donate_min": {32, 64, 128, 256}, "wave_pairs": {0, 16, 64, 128}, "smem_carveout": {0, 25, 50, 100},
         "init_chunk": {1, 4}}


def shape(o):
    d = o.as_dict()
    return {k: d[k] for k in KNOBS}


def posed_scene(ctx, sc):
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    return ds


def test_autotune_choice_is_valid_cached_and_exact(oracle):
    ctx = kd.Context(0)  # a context of its own: its cache starts empty
    sc = scenes.config3(n_pairs=48, seed=21, max_tets=3e4)
    ds = posed_scene(ctx, sc)
    before = shape(ds.default_opts())
    best = ds.autotune(sc.pairs, repeats=5)
    got = shape(best)
    for k, allowed in KNOBS.items():
        assert got[k] in allowed, (k, got[k])
    # the scene's defaults are now the tuned choice
    assert shape(ds.default_opts()) == got
    # the tuned launch gives the oracle's result
    st = ds.traverse_sync(sc.pairs, ds.default_opts())
    worlds = [world_xyz(oracle, sc, i) for i in range(len(sc.meshes))]
    rows, tests_pp, _ = oracle.run_pairs(sc.K, worlds, sc.meshes, sc.pairs)
    assert st.n_tests == int(tests_pp.sum())
    assert np.array_equal(sorted_rows(ds.candidates().astype(np.int64)), sorted_rows(rows.astype(np.int64)))

    # another scene of the same K and size class picks up the cached choice
    sc2 = scenes.config3(n_pairs=48, seed=21, max_tets=3e4)
    ds2 = kd.DeviceScene(ctx, sc2.K, sc2.meshes)
    assert int(np.log2(sc2.n_tets)) == int(np.log2(sc.n_tets))
    assert shape(ds2.default_opts()) == got
    # a scene of another size class keeps the static defaults
    sc3 = scenes.small_batch(n_pairs=2, seed=5)
    assert int(np.log2(sc3.n_tets)) != int(np.log2(sc.n_tets))
    ds3 = kd.DeviceScene(ctx, sc3.K, sc3.meshes)
    assert shape(ds3.default_opts()) == before
    # and a scene of another K as well
    sc4 = scenes.config3(n_pairs=48, seed=21, max_tets=3e4, K=18)
    ds4 = kd.DeviceScene(ctx, sc4.K, sc4.meshes)
    assert shape(ds4.default_opts()) == before
    for d in (ds, ds2, ds3, ds4):
        d.close()
    ctx.close()
