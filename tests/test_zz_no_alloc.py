"""kdop_traverse_noalloc: the traversal entry point that allocates no device
memory, for callers that cannot call cudaMalloc while they run (a plugin whose
host application's allocator owns all device memory, a simulator with a fixed
device-memory budget reserved at start-up, a real-time step that must not
risk an allocation failure).

The caller owns every buffer (here torch allocates them, in the test, before
the call); the entry point keeps its scratch in a static device array.  Its
output must equal the allocating entry point's (kdop_traverse) exactly --
candidate pairs are integer results -- on two calls in a row, which also
shows that each call starts from cleared scratch.  This file is collected
last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

import kdop_b200 as kd
from conftest import sorted_rows
from kdop_b200 import scenes

pytestmark = pytest.mark.gpu


def _global_to_local(rows_a, rows_b, rows_p, pairs, t_off):
    ma = pairs[rows_p, 0]
    mb = pairs[rows_p, 1]
    return np.column_stack([rows_p, rows_a - t_off[ma], rows_b - t_off[mb]]).astype(np.int64)


def test_noalloc_traversal_matches_allocating_entry_point(ctx):
    import torch

    sc = scenes.small_batch(n_pairs=12, n_lo=3, n_hi=7, seed=31)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    st = ds.traverse_sync(sc.pairs)
    want = sorted_rows(ds.candidates().astype(np.int64))
    assert len(want) > 0

    lib = ds.lib
    lib.kdop_traverse_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    lib.kdop_traverse_noalloc.restype = ctypes.c_int

    # caller-owned device buffers, allocated before the calls
    n = len(sc.pairs)
    cap = int(st.n_candidates) + 64
    pairs_d = torch.tensor(sc.pairs.astype(np.int32), device="cuda")
    cand_d = torch.empty(3 * cap, dtype=torch.int32, device="cuda")
    cnt_d = torch.empty(4, dtype=torch.int64, device="cuda")
    t_off = ds.t_off

    for call in range(2):
        cand_d.fill_(-1)
        cnt_d.fill_(-1)
        torch.cuda.synchronize()
        rc = lib.kdop_traverse_noalloc(ds.h, n, pairs_d.data_ptr(), cand_d.data_ptr(), cap, cnt_d.data_ptr(), None)
        assert rc == 0, rc
        ctx.synchronize()
        counts = cnt_d.cpu().numpy()
        assert counts[3] == 0, f"device error bits {counts[3]} on call {call}"
        assert counts[0] == st.n_candidates and counts[1] == st.n_tests and counts[2] == st.n_leaf_overlaps
        c = cand_d.cpu().numpy().view(np.uint32).astype(np.int64)
        k = int(counts[0])
        got = _global_to_local(c[:k], c[cap:cap + k], c[2 * cap:2 * cap + k], sc.pairs.astype(np.int64), t_off)
        assert np.array_equal(sorted_rows(got), want), f"call {call} differs"


def test_noalloc_rejects_oversized_requests(ctx):
    import torch

    sc = scenes.small_batch(n_pairs=2, seed=3)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    lib = ds.lib
    lib.kdop_traverse_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    assert lib.kdop_traverse_noalloc(ds.h, 1, buf.data_ptr(), buf.data_ptr(), 1 << 33, buf.data_ptr(), None) == \
        kd.lib.ERR_CAPACITY
    assert lib.kdop_traverse_noalloc(ds.h, 1 << 31, buf.data_ptr(), buf.data_ptr(), 8, buf.data_ptr(), None) == \
        kd.lib.ERR_CAPACITY
    assert lib.kdop_traverse_noalloc(ds.h, 1, None, buf.data_ptr(), 8, buf.data_ptr(), None) == kd.lib.ERR_INVALID


def test_noalloc_queue_exhaustion_is_reported_and_the_next_call_is_clean(ctx):
    """A run that needs more than the static array's 65,536 queue entries sets
    error bit 2 (queue full) in counters[3] and still returns: entries that
    found no room are dropped and never counted as outstanding work, so the
    waiting warps see the work count reach zero.  The next call (a scene
    whose traversal fits the static queue) starts from a cleared array and
    gives the allocating entry point's result again."""
    import torch

    def noalloc(ds, pairs_d, n, cand_d, cap, cnt_d, opts):
        fn = ds.lib.kdop_traverse_noalloc
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                       ctypes.c_void_p, ctypes.c_void_p]
        fn.restype = ctypes.c_int
        torch.cuda.synchronize()
        rc = fn(ds.h, n, pairs_d.data_ptr(), cand_d.data_ptr(), cap, cnt_d.data_ptr(),
                ctypes.byref(opts) if opts is not None else None)
        assert rc == 0, rc
        ctx.synchronize()
        return cnt_d.cpu().numpy()

    # the exhausting run: smallest deques and eager donation, so that most
    # node pairs pass through the queue
    sc = scenes.config3(n_pairs=24, seed=5, min_tets=2e4, max_tets=6e4)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    hungry = ds.opts(stack_cap=64, donate_min=1, init_chunk=1)
    st = ds.traverse_sync(sc.pairs, hungry)
    assert st.queue_used > 65536, f"case too small to exhaust the static queue ({st.queue_used} entries)"
    cap = int(st.n_candidates) + 64
    pairs_d = torch.tensor(sc.pairs.astype(np.int32), device="cuda")
    cand_d = torch.empty(3 * cap, dtype=torch.int32, device="cuda")
    cnt_d = torch.empty(4, dtype=torch.int64, device="cuda")
    counts = noalloc(ds, pairs_d, len(sc.pairs), cand_d, cap, cnt_d, hungry)
    assert counts[3] & 2, f"queue exhaustion not reported (error bits {counts[3]})"
    assert not counts[3] & 1, "the run gave up waiting instead of ending"

    # the next call, on a scene whose default traversal fits the queue
    sm = scenes.small_batch(n_pairs=12, n_lo=3, n_hi=7, seed=31)
    ds2 = kd.DeviceScene(ctx, sm.K, sm.meshes)
    ds2.set_poses(sm.quat, sm.pos)
    ds2.refit(kd.REFIT_POSE)
    base = ds2.traverse_sync(sm.pairs)
    assert base.queue_used <= 65536
    want = sorted_rows(ds2.candidates().astype(np.int64))
    cap2 = int(base.n_candidates) + 64
    pairs2 = torch.tensor(sm.pairs.astype(np.int32), device="cuda")
    cand2 = torch.empty(3 * cap2, dtype=torch.int32, device="cuda")
    counts = noalloc(ds2, pairs2, len(sm.pairs), cand2, cap2, cnt_d, None)
    assert counts[3] == 0, f"error bits {counts[3]} after the exhausted run"
    assert counts[0] == base.n_candidates and counts[1] == base.n_tests
    c = cand2.cpu().numpy().view(np.uint32).astype(np.int64)
    k = int(counts[0])
    got = _global_to_local(c[:k], c[cap2:cap2 + k], c[2 * cap2:2 * cap2 + k], sm.pairs.astype(np.int64), ds2.t_off)
    assert np.array_equal(sorted_rows(got), want)
    ds.close()
    ds2.close()
