"""GPU tree build (KDOP_BUILD_DEVICE) against the host build (KDOP_BUILD_HOST,
the reference's std::sort Morton order + index-median make_tree): identical
node records for every mesh, identical traversal results."""
import numpy as np
import pytest

import kdop_b200 as kd
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def trees(ds, n_meshes):
    return [ds.read_tree(m) for m in range(n_meshes)]


def assert_same_trees(ctx, K, meshes, expect_host_orders=None):
    dd = kd.DeviceScene(ctx, K, meshes, build=kd.BUILD_DEVICE)
    dh = kd.DeviceScene(ctx, K, meshes, build=kd.BUILD_HOST)
    idd, idh = dd.info(), dh.info()
    assert idd["build"] == kd.BUILD_DEVICE and idh["build"] == kd.BUILD_HOST
    for k in ("n_nodes", "depth", "n_tets"):
        assert idd[k] == idh[k], k
    if expect_host_orders is not None:
        assert idd["host_orders"] == expect_host_orders
    for m, ((vd, td), (vh, th)) in enumerate(zip(trees(dd, len(meshes)), trees(dh, len(meshes)))):
        assert np.array_equal(td, th), f"mesh {m}: leaf tets differ"
        assert np.array_equal(vd.view(np.uint32), vh.view(np.uint32)), f"mesh {m}: volumes differ"
    return dd, dh


def truncated(m, k):
    """First k tets of a lattice mesh (the tree topology depends on the count only)."""
    t = m.tets[:k]
    return scenes.Mesh(m.xyz, t, scenes.surface_map(t) if k else np.zeros(0, np.uint8))


def test_every_small_tet_count(ctx):
    rng = np.random.default_rng(0)
    base = scenes.lattice(4, 0.15, rng)  # 384 tets
    counts = list(range(1, 70)) + [127, 128, 129, 255, 256, 257, 383, 384]
    meshes = [truncated(base, k) for k in counts]
    assert_same_trees(ctx, 14, meshes, expect_host_orders=0)


def test_odd_root_count_and_empty_meshes(ctx):
    rng = np.random.default_rng(1)
    base = scenes.lattice(3, 0.1, rng)
    meshes = [truncated(base, 5), truncated(base, 0), truncated(base, 17), truncated(base, 1), truncated(base, 0),
              truncated(base, 33), truncated(base, 2)]
    assert_same_trees(ctx, 8, meshes)


@pytest.mark.parametrize("K", scenes.SUPPORTED_K)
def test_batch_all_K(ctx, K):
    sc = scenes.small_batch(n_pairs=6, seed=K, K=K)
    dd, dh = assert_same_trees(ctx, K, sc.meshes, expect_host_orders=0)
    for ds in (dd, dh):
        ds.set_poses(sc.quat, sc.pos)
        ds.refit(kd.REFIT_POSE)
    sd = dd.traverse_sync(sc.pairs, contacts=True)
    sh = dh.traverse_sync(sc.pairs, contacts=True)
    assert sd.n_tests == sh.n_tests and sd.n_candidates == sh.n_candidates and sd.n_contacts == sh.n_contacts
    dd.sort_results()
    dh.sort_results()
    assert np.array_equal(dd.candidates(), dh.candidates())


def test_config3_subset(ctx):
    sc = scenes.config3(n_pairs=64, seed=8)
    assert_same_trees(ctx, sc.K, sc.meshes, expect_host_orders=0)


def test_equal_codes_take_the_host_order(ctx):
    rng = np.random.default_rng(3)
    m = scenes.lattice(3, 0.1, rng)
    # the same tet twice: equal centroids, equal Morton codes
    t = np.concatenate([m.tets, m.tets[:5]])
    dup = scenes.Mesh(m.xyz, t, scenes.surface_map(t))
    assert_same_trees(ctx, 14, [m, dup, m], expect_host_orders=1)


def test_given_leaf_order(ctx):
    rng = np.random.default_rng(4)
    m = scenes.lattice(3, 0.1, rng)
    m2 = scenes.Mesh(m.xyz, m.tets, m.surf)
    m2.leaf_order = rng.permutation(m.n_tets).astype(np.uint32)
    assert_same_trees(ctx, 14, [m, m2], expect_host_orders=1)
