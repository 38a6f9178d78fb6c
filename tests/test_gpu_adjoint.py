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
    t_all = [m.tets.astype(np.int64) + v_off[i] for i, m in enumerate(sc.meshes)]
    recs = {}
    for p in np.unique(cand[n_per_cand > 0, 0]):
        a, b = sc.pairs[p]
        sel = np.nonzero((cand[:, 0] == p) & (n_per_cand > 0))[0]
        tp = cand[sel, 1:]
        A, B = sc.meshes[a], sc.meshes[b]
        xa, xb = world[v_off[a]:v_off[a + 1]], world[v_off[b]:v_off[b + 1]]
        _, rec = oracle.contacts(xa, A.tets, A.surf, xb, B.tets, B.surf, tp, "f")
        for k, ci in enumerate(sel):
            recs[ci] = (t_all[a][cand[ci, 1]], t_all[b][cand[ci, 2]], rec[k])
    assert all(int(r[2]["ncontacts"]) == n_per_cand[ci] for ci, r in recs.items())

    X = world.astype(np.float64)

    def pair_loss(va, vb, rec, ncont, Xv):
        d, n = oracle.frozen_depth(Xv[va].ravel(), Xv[vb].ravel(), rec)
        return ncont * (d * d + float(n @ wv))

    # (1) FP64 oracle gradient on every vertex
    g_ref = np.zeros_like(X)
    touching = {}
    for ci, (va, vb, rec) in recs.items():
        nc = n_per_cand[ci]
        d, _ = oracle.frozen_depth(X[va].ravel(), X[vb].ravel(), rec)
        g24 = oracle.depth_grad(X[va].ravel(), X[vb].ravel(), rec, 2.0 * d * nc, nc * wv)
        g_ref[va] += g24[:12].reshape(4, 3)
        g_ref[vb] += g24[12:].reshape(4, 3)
        for v in list(va) + list(vb):
            touching.setdefault(int(v), []).append(ci)
    scale = np.abs(g_ref).max()
    err = np.abs(g_gpu - g_ref)
    bound = RTOL * np.maximum(np.abs(g_ref), 1e-2 * scale)
    bad = err > bound
    assert not bad.any(), (bad.sum(), err[bad][:5], g_ref[bad][:5])

    # (2) FP64 central differences of the frozen-decision loss
    rng = np.random.default_rng(seed)
    verts = np.array(sorted(touching))
    pick = rng.choice(verts, size=min(n_fd, len(verts)), replace=False)
    worst = 0.0
    for v in pick:
        for c in range(3):
            lp = lm = 0.0
            Xp = X.copy()
            Xm = X.copy()
            Xp[v, c] += H
            Xm[v, c] -= H
            for ci in touching[int(v)]:
                va, vb, rec = recs[ci]
                nc = n_per_cand[ci]
                lp += pair_loss(va, vb, rec, nc, Xp)
                lm += pair_loss(va, vb, rec, nc, Xm)
            fd = (lp - lm) / (2 * H)
            e = abs(g_gpu[v, c] - fd) / max(abs(fd), 1e-2 * scale)
            worst = max(worst, e)
            assert e <= RTOL, (v, c, g_gpu[v, c], fd)
    ds.close()
    return len(recs), len(pick), worst


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
