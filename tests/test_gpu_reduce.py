"""Contact point reduction on the device (kdop_reduce_contact_rows,
kdop_reduce_contacts) against the reference's own std::sort + std::unique
over prox::ContactPoint (golden fixture) and the oracle's restatement."""
import os
import sys

import numpy as np
import pytest

import kdop_b200 as kd
from kdop_b200 import scenes

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import reduction_rows  # noqa: E402

pytestmark = pytest.mark.gpu


def as_contacts(rows7, cand=None):
    c = np.zeros(len(rows7), kd.CONTACT_DTYPE)
    c["p"], c["n"], c["depth"] = rows7[:, 0:3], rows7[:, 3:6], rows7[:, 6]
    c["cand"] = np.arange(len(rows7)) if cand is None else cand
    return c


def as_rows7(c):
    return np.column_stack([c["p"], c["n"], c["depth"][:, None]]).astype(np.float32)


def test_reduce_rows_matches_reference_golden(ctx, golden):
    rows, bodies = golden["reduce_rows"], golden["reduce_bodies"]
    out, ob = ctx.reduce_contact_rows(as_contacts(rows), bodies)
    assert np.array_equal(ob, golden["reduce_out_bodies"])
    assert np.all(as_rows7(out) == golden["reduce_out_rows"])  # float ==: -0 == +0
    # `cand` names the input row each kept row came from
    assert np.all(as_rows7(as_contacts(rows)[out["cand"]]) == as_rows7(out))


@pytest.mark.parametrize("seed,n_base,nb", [(11, 1, 1), (12, 7, 2), (13, 5000, 3), (14, 40000, 1), (15, 200000, 64)])
def test_reduce_rows_matches_oracle(ctx, oracle, seed, n_base, nb):
    rows, bodies = reduction_rows(np.random.default_rng(seed), n_base=n_base, n_bodies=nb)
    want_r, want_b, want_src = oracle.reduce_contacts(rows, bodies)
    out, ob = ctx.reduce_contact_rows(as_contacts(rows), bodies)
    assert np.array_equal(ob, want_b)
    assert np.all(as_rows7(out) == want_r)
    assert np.array_equal(out["cand"], want_src)  # stable among fully equal keys, like the oracle


def test_reduce_rows_long_segments(ctx, oracle):
    # every row on one p.y value: a single segment walked by one thread
    rng = np.random.default_rng(5)
    rows = rng.uniform(-1, 1, (4000, 7)).astype(np.float32)
    rows[:, 1] = np.float32(0.5)
    rows[2000:] = rows[:2000] + np.float32(2e-7)  # within the tolerance in every field
    rows[2000:, 1] = np.float32(0.5)  # same p.y: each copy sorts next to its original (by p.x)
    bodies = np.zeros((4000, 2), np.uint32)
    want_r, want_b, _ = oracle.reduce_contacts(rows, bodies)
    out, ob = ctx.reduce_contact_rows(as_contacts(rows), bodies)
    assert len(out) == len(want_r) == 2000
    assert np.all(as_rows7(out) == want_r)


def test_reduce_rows_edge_cases(ctx):
    out, ob = ctx.reduce_contact_rows(np.zeros(0, kd.CONTACT_DTYPE), np.zeros((0, 2), np.uint32))
    assert len(out) == 0
    one = as_contacts(np.ones((1, 7), np.float32))
    out, ob = ctx.reduce_contact_rows(one, np.array([[3, 4]], np.uint32))
    assert len(out) == 1 and ob.tolist() == [[3, 4]]
    # capacity: reports the rows needed, writes nothing
    lib = kd.load_library()
    import ctypes as C
    rows, bodies = reduction_rows(np.random.default_rng(3), n_base=50, n_bodies=2)
    c = as_contacts(rows)
    dst = np.zeros(4, kd.CONTACT_DTYPE)
    n = C.c_int64()
    rc = lib.kdop_reduce_contact_rows(ctx.h, c.ctypes.data_as(C.c_void_p), bodies.ctypes.data_as(C.c_void_p),
                                      len(c), dst.ctypes.data_as(C.c_void_p), None, 4, C.byref(n))
    assert rc == kd.lib.ERR_CAPACITY and n.value > 4
    assert not dst.view(np.uint8).any()


def test_reduce_scratch_reused_across_sizes(oracle):
    """The sort scratch lives in the context: a fresh context reduces sets that
    grow, shrink and grow again, each equal to the oracle's result."""
    c = kd.Context(0)
    try:
        for seed, n_base, nb in [(21, 20000, 4), (22, 3, 1), (23, 60000, 9), (24, 500, 2), (25, 60000, 9)]:
            rows, bodies = reduction_rows(np.random.default_rng(seed), n_base=n_base, n_bodies=nb)
            want_r, want_b, want_src = oracle.reduce_contacts(rows, bodies)
            out, ob = c.reduce_contact_rows(as_contacts(rows), bodies)
            assert np.array_equal(ob, want_b), seed
            assert np.all(as_rows7(out) == want_r), seed
            assert np.array_equal(out["cand"], want_src), seed
    finally:
        c.close()


def test_reduce_rows_device_buffers(ctx, oracle):
    torch = pytest.importorskip("torch")
    rows, bodies = reduction_rows(np.random.default_rng(8), n_base=3000, n_bodies=5)
    c = as_contacts(rows)
    d_rows = torch.from_numpy(c.view(np.uint8).copy()).cuda()
    d_bodies = torch.from_numpy(bodies.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(len(c) * 32, dtype=torch.uint8, device="cuda")
    d_ob = torch.zeros(len(c) * 8, dtype=torch.uint8, device="cuda")
    import ctypes as C
    n = C.c_int64()
    rc = ctx.lib.kdop_reduce_contact_rows(ctx.h, C.c_void_p(d_rows.data_ptr()), C.c_void_p(d_bodies.data_ptr()),
                                          len(c), C.c_void_p(d_out.data_ptr()), C.c_void_p(d_ob.data_ptr()), len(c),
                                          C.byref(n))
    assert rc == 0
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(kd.CONTACT_DTYPE)[:n.value]
    ob = d_ob.cpu().numpy().view(np.uint32).reshape(-1, 2)[:n.value]
    want_r, want_b, _ = oracle.reduce_contacts(rows, bodies)
    assert np.all(as_rows7(out) == want_r) and np.array_equal(ob, want_b)


def test_reduce_scene_contacts(ctx, oracle):
    sc = scenes.config5(n_pairs=6, n=6)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    ds.reserve(candidates=1 << 20, contacts=1 << 20)
    ds.traverse_sync(sc.pairs, contacts=True)
    rows = ds.read_contacts()
    assert len(rows) > 100
    cand = ds.candidates()  # (pair, tet A, tet B) per candidate row
    bodies = sc.pairs[cand[rows["cand"], 0]].astype(np.uint32)
    want_r, want_b, want_src = oracle.reduce_contacts(as_rows7(rows), bodies)
    out, ob = ds.reduce_contacts()
    assert np.array_equal(ob, want_b)
    assert np.all(as_rows7(out) == want_r)
    assert np.array_equal(out["cand"], rows["cand"][want_src])
    # the scene's own contacts and records are untouched (the adjoint still reads them)
    assert np.array_equal(ds.read_contacts().view(np.uint8), rows.view(np.uint8))


def test_reduce_arguments_and_state_are_checked(ctx):
    import ctypes as C
    lib = kd.load_library()
    n = C.c_int64()
    rows = as_contacts(np.ones((3, 7), np.float32))
    bodies = np.zeros((3, 2), np.uint32)
    rp, bp = rows.ctypes.data_as(C.c_void_p), bodies.ctypes.data_as(C.c_void_p)
    assert lib.kdop_reduce_contact_rows(None, rp, bp, 3, rp, None, 3, C.byref(n)) == kd.lib.ERR_INVALID
    assert lib.kdop_reduce_contact_rows(ctx.h, rp, bp, -1, rp, None, 3, C.byref(n)) == kd.lib.ERR_INVALID
    assert lib.kdop_reduce_contact_rows(ctx.h, None, bp, 3, rp, None, 3, C.byref(n)) == kd.lib.ERR_INVALID
    assert lib.kdop_reduce_contact_rows(ctx.h, rp, bp, 3, rp, None, 3, None) == kd.lib.ERR_INVALID
    sc = scenes.small_batch(n_pairs=2, seed=3)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    with pytest.raises(kd.KdopError):
        ds.reduce_contacts()  # before kdop_contacts
