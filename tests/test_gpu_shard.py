"""kdop_traverse_shard: a traversal split into shards from a breadth-first
frontier (one huge pair over several ranks or GPUs).  The shards together
must give exactly the unsharded traversal: every candidate tet pair on one
shard, test counts summing to the total, contacts to the same rows."""
import numpy as np
import pytest

import kdop_b200 as kd
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def rows_sorted(c):
    return c[np.lexsort((c[:, 2], c[:, 1], c[:, 0]))] if len(c) else c


def contact_bits(rows):
    b = np.column_stack([rows["p"].view(np.uint32), rows["n"].view(np.uint32), rows["depth"].view(np.uint32)[:, None]])
    return b[np.lexsort(b.T[::-1])] if len(b) else b


def scene(ctx, sc):
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ds.reserve(candidates=4 << 20, contacts=4 << 20, queue=4 << 20)
    return ds


@pytest.mark.parametrize("case", ["one_pair", "batch"])
@pytest.mark.parametrize("n_ranks,frontier_min", [(1, 4096), (2, 256), (3, 4096), (4, 64)])
def test_shards_add_up_to_the_traversal(ctx, case, n_ranks, frontier_min):
    sc = scenes.config2(n=16) if case == "one_pair" else scenes.small_batch(n_pairs=10, n_lo=3, n_hi=7, seed=21)
    ds = scene(ctx, sc)
    full = ds.traverse_sync(sc.pairs, contacts=True)
    want = rows_sorted(ds.candidates())
    want_contacts = contact_bits(ds.read_contacts())
    got, got_contacts, tests = [], [], 0
    for r in range(n_ranks):
        ds.traverse_shard(sc.pairs, r, n_ranks, frontier_min)
        ds.contacts()
        st = ds.stats()
        tests += st.n_tests
        got.append(ds.candidates())
        got_contacts.append(ds.read_contacts())
    got = rows_sorted(np.concatenate(got))
    assert tests == full.n_tests
    assert len(got) == len(want)  # no candidate on two shards
    assert np.array_equal(got, want)
    gc = np.concatenate(got_contacts)
    assert np.array_equal(contact_bits(gc), want_contacts)


def test_shard_arguments_are_checked(ctx):
    sc = scenes.small_batch(n_pairs=2, seed=3)
    ds = scene(ctx, sc)
    for rank, n_ranks, fmin in ((2, 2, 64), (-1, 2, 64), (0, 0, 64), (0, 1, 0)):
        with pytest.raises(kd.KdopError):
            ds.traverse_shard(sc.pairs, rank, n_ranks, fmin)
