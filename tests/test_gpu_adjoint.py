"""Hand-written adjoint of contact generation, through torch.autograd.

Loss = sum of squared penetration depths over all contacts, the candidate pair
set and every discrete choice fixed by the forward pass.  The FP32 gradient of
the CUDA adjoint is checked against (1) the FP64 oracle gradient
(or_depth_grad_d with the forward's decisions) on every vertex and (2) FP64
central finite differences (h = 1e-6) of the frozen-decision loss on up to
1000 random vertices; both within 1e-3 relative.
"""
import numpy as np
import pytest
import torch

import kdop_b200 as kd
from kdop_b200 import scenes
from kdop_b200.autograd import contact_geometry

pytestmark = pytest.mark.gpu

H = 1e-6
RTOL = 1e-3


def oracle_rec_dtype():
    from oracle.pyoracle import OR_RECORD_DTYPE
    return OR_RECORD_DTYPE


def run_case(ctx, oracle, sc, n_fd=1000, seed=0, w=None):
    """Loss = sum(depth^2) (+ sum(normal . w) when w is given)."""
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    world = np.concatenate([oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)])
    x = torch.tensor(world, device="cuda", requires_grad=True)
    depth, normal = contact_geometry(x, ds, sc.pairs)
    loss = (depth.double() ** 2).sum()
    wv = np.zeros(3) if w is None else np.asarray(w, np.float64)
    if w is not None:
        loss = loss + (normal.double() @ torch.tensor(wv, device="cuda")).sum()
    loss.backward()
    g_gpu = x.grad.detach().cpu().numpy().astype(np.float64)
    assert depth.numel() > 0

    # decisions of the forward pass, from the FP32 oracle (bit-identical to the device)
    cand = ds.candidates()
    rows = ds.read_contacts()
    n_per_cand = np.bincount(rows["cand"], minlength=len(cand))
    v_off = ds.v_off
    live = np.nonzero(n_per_cand > 0)[0]
    va = np.zeros((len(live), 4), np.int64)
    vb = np.zeros((len(live), 4), np.int64)
    recs = np.zeros(len(live), oracle_rec_dtype())
    for p in np.unique(cand[live, 0]):
        a, b = sc.pairs[p]
        k = np.nonzero(cand[live, 0] == p)[0]
        tp = cand[live[k], 1:]
        A, B = sc.meshes[a], sc.meshes[b]
        xa, xb = world[v_off[a]:v_off[a + 1]], world[v_off[b]:v_off[b + 1]]
        _, rec = oracle.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, tp, "f")
        recs[k] = rec
        va[k] = A.tets[tp[:, 0]].astype(np.int64) + v_off[a]
        vb[k] = B.tets[tp[:, 1]].astype(np.int64) + v_off[b]
    nc = n_per_cand[live].astype(np.float64)
    assert np.array_equal(recs["ncontacts"], n_per_cand[live])

    X = world.astype(np.float64)

    # (1) FP64 oracle gradient on every vertex
    d, _ = oracle.frozen_batch(X[va].reshape(-1, 12), X[vb].reshape(-1, 12), recs)
    g24 = oracle.depth_grad_batch(X[va].reshape(-1, 12), X[vb].reshape(-1, 12), recs, 2.0 * d * nc,
                                  nc[:, None] * wv[None, :])
    g_ref = np.zeros_like(X)
    np.add.at(g_ref, va.ravel(), g24[:, :12].reshape(-1, 3))
    np.add.at(g_ref, vb.ravel(), g24[:, 12:].reshape(-1, 3))
    scale = np.abs(g_ref).max()
    err = np.abs(g_gpu - g_ref)
    bound = RTOL * np.maximum(np.abs(g_ref), 1e-2 * scale)
    bad = err > bound
    assert not bad.any(), (bad.sum(), err[bad][:5], g_ref[bad][:5])

    # (2) FP64 central differences of the frozen-decision loss
    owner = np.concatenate([np.repeat(np.arange(len(live)), 4), np.repeat(np.arange(len(live)), 4)])
    verts = np.concatenate([va.ravel(), vb.ravel()])
    order = np.argsort(verts, kind="stable")
    verts_s, owner_s = verts[order], owner[order]
    uniq, start = np.unique(verts_s, return_index=True)
    end = np.append(start[1:], len(verts_s))
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(uniq), size=min(n_fd, len(uniq)), replace=False)
    worst = 0.0
    for u in pick:
        v = uniq[u]
        ks = np.unique(owner_s[start[u]:end[u]])
        for c in range(3):
            ls = []
            for sgn in (1.0, -1.0):
                a_loc, b_loc = X[va[ks]], X[vb[ks]]
                a_loc[va[ks] == v, c] += sgn * H
                b_loc[vb[ks] == v, c] += sgn * H
                dd, nn = oracle.frozen_batch(a_loc.reshape(-1, 12), b_loc.reshape(-1, 12), recs[ks])
                ls.append(float((nc[ks] * (dd * dd + nn @ wv)).sum()))
            fd = (ls[0] - ls[1]) / (2 * H)
            e = abs(g_gpu[v, c] - fd) / max(abs(fd), 1e-2 * scale)
            worst = max(worst, e)
            assert e <= RTOL, (v, c, g_gpu[v, c], fd)
    recs_n = len(live)
    ds.close()
    return recs_n, len(pick), worst


def test_adjoint_small_touching_batch(ctx, oracle):
    rng_sc = scenes.config5(n_pairs=6, n=5, seed=4)
    n_pairs, n_fd, worst = run_case(ctx, oracle, rng_sc, n_fd=200)
    assert n_pairs > 10


def test_adjoint_config5_full(ctx, oracle):
    """256 pairs of 20^3-cell lattices (48k tets each), 1000 FD vertices."""
    sc = scenes.config5()
    n_pairs, n_fd, worst = run_case(ctx, oracle, sc, n_fd=1000)
    assert n_fd == 1000


def test_adjoint_depth_and_normal_gradients(ctx, oracle):
    """dL/dn flows through the adjoint too: L = sum(d^2) + sum(n . w)."""
    sc = scenes.config5(n_pairs=4, n=4, seed=9)
    n_pairs, n_fd, worst = run_case(ctx, oracle, sc, n_fd=200, w=[0.3, -0.2, 0.7])
    assert n_pairs > 5
