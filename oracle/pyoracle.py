"""ctypes access to the CPU oracle and to the reference's compiled CPU path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference leg of bench.py.  The product library never uses it.

  Oracle     -> oracle/_build/libkdop_oracle.so  (the project's C restatement)
  Reference  -> oracle/_ref/libkdop_ref_record.so (reference code + counting)
  RefTimer   -> oracle/_ref/libkdop_ref_time.so   (unmodified reference code)
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libkdop_oracle.so")
REF_RECORD_SO = os.path.join(HERE, "_ref", "libkdop_ref_record.so")
REF_TIME_SO = os.path.join(HERE, "_ref", "libkdop_ref_time.so")

_i64 = C.c_int64
_p = C.c_void_p


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class OrRecord(C.Structure):
    _fields_ = [("face_a", C.c_int32), ("face_b", C.c_int32), ("imin", C.c_int32), ("imax", C.c_int32),
                ("ncontacts", C.c_int32), ("overlap", C.c_int32), ("cand_mask", C.c_uint64)]


OR_RECORD_DTYPE = np.dtype([("face_a", np.int32), ("face_b", np.int32), ("imin", np.int32),
                            ("imax", np.int32), ("ncontacts", np.int32), ("overlap", np.int32),
                            ("cand_mask", np.uint64)])


def available() -> bool:
    return os.path.exists(ORACLE_SO)


def reference_available() -> bool:
    return os.path.exists(REF_RECORD_SO) and os.path.exists(REF_TIME_SO)


class Oracle:
    """The project's C restatement (kdop_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        self.lib = C.CDLL(path)
        L = self.lib
        L.or_dirs_f.argtypes = [C.c_int, _p]
        L.or_leaf_dops_f.argtypes = [C.c_int, _p, _i64, _p, _p]
        L.or_morton_order.argtypes = [_p, _i64, _i64, _p, _p]
        L.or_build_tree.argtypes = [_i64, _p, _p, _p, _p]
        L.or_build_tree.restype = _i64
        L.or_refit_f.argtypes = [C.c_int, _p, _p, _i64, _p, _p, _p, _p]
        L.or_run_pair_f.argtypes = [C.c_int, _i64, _p, _p, _i64, _p, _p, _i64, _p, _p, _i64, _p, _p, _i64, _p, _p,
                                    _p, _p]
        L.or_run_pairs_f.argtypes = [C.c_int, C.c_int, _p, _p, _p, _p, _p, _p, _i64, _p, C.c_int, _i64, _p, _p, _p,
                                     _p]
        L.or_surface_map.argtypes = [_i64, _i64, _p, _p]
        for nm in ("or_contacts_f", "or_contacts_d", "or_contacts_dd"):
            getattr(L, nm).argtypes = [_p, _p, _p, _p, _p, _p, _i64, _p, _i64, _p, _p, _p]
        L.or_frozen_depth_d.argtypes = [_p, _p, _p, _p]
        L.or_frozen_depth_d.restype = C.c_double
        L.or_depth_grad_d.argtypes = [_p, _p, _p, C.c_double, _p, _p]
        L.or_frozen_batch_d.argtypes = [_i64, _p, _p, _p, _p, _p]
        L.or_depth_grad_batch_d.argtypes = [_i64, _p, _p, _p, _p, _p, _p]
        L.or_rotate_f.argtypes = [_p, _p, _i64, _p, _p]
        L.or_sin_f.argtypes = [C.c_float]
        L.or_sin_f.restype = C.c_float
        L.or_deform_f.argtypes = [C.c_float, C.c_float, C.c_float, _i64, _p, _p]

    def dirs(self, K: int) -> np.ndarray:
        out = np.zeros((13, 3), np.float32)
        n = self.lib.or_dirs_f(K, _ptr(out))
        if n < 0:
            raise ValueError(f"unsupported K={K}")
        return out[:n].copy()

    def leaf_dops(self, K, xyz, tets) -> np.ndarray:
        xyz, tets = _c(xyz, np.float32), _c(tets, np.uint32)
        out = np.zeros((tets.shape[0], K), np.float32)
        self.lib.or_leaf_dops_f(K, _ptr(xyz), tets.shape[0], _ptr(tets), _ptr(out))
        return out

    def morton_order(self, xyz, tets) -> np.ndarray:
        xyz, tets = _c(xyz, np.float32), _c(tets, np.uint32)
        perm = np.zeros(tets.shape[0], np.uint32)
        self.lib.or_morton_order(_ptr(xyz), xyz.shape[0], tets.shape[0], _ptr(tets), _ptr(perm))
        return perm

    def build_tree(self, perm):
        perm = _c(perm, np.uint32)
        nt = perm.shape[0]
        nn = max(2 * nt - 1, 0)
        left = np.zeros(nn, np.int64)
        right = np.zeros(nn, np.int64)
        tet = np.zeros(nn, np.int64)
        n = self.lib.or_build_tree(nt, _ptr(perm), _ptr(left), _ptr(right), _ptr(tet))
        assert n == nn
        return left, right, tet

    def refit(self, K, xyz, tets, left, right, tet) -> np.ndarray:
        xyz, tets = _c(xyz, np.float32), _c(tets, np.uint32)
        vol = np.zeros((left.shape[0], K), np.float32)
        self.lib.or_refit_f(K, _ptr(xyz), _ptr(tets), left.shape[0], _ptr(_c(left, np.int64)),
                            _ptr(_c(right, np.int64)), _ptr(_c(tet, np.int64)), _ptr(vol))
        return vol

    def run_pair(self, K, xyzA, tetsA, surfA, xyzB, tetsB, surfB, restA=None, restB=None):
        """Pairs (n,2) in traversal order, node-pair tests, leaf overlaps.
        Trees are built on restA/restB (default: the world positions)."""
        xyzA, tetsA, surfA = _c(xyzA, np.float32), _c(tetsA, np.uint32), _c(surfA, np.uint8)
        xyzB, tetsB, surfB = _c(xyzB, np.float32), _c(tetsB, np.uint32), _c(surfB, np.uint8)
        restA = None if restA is None else _c(restA, np.float32)
        restB = None if restB is None else _c(restB, np.float32)
        cap = 1 << 16
        while True:
            out = np.zeros((cap, 2), np.uint32)
            np_, tests, lo = _i64(), _i64(), _i64()
            rc = self.lib.or_run_pair_f(K, xyzA.shape[0], _ptr(xyzA), _ptr(restA), tetsA.shape[0], _ptr(tetsA),
                                        _ptr(surfA), xyzB.shape[0], _ptr(xyzB), _ptr(restB), tetsB.shape[0],
                                        _ptr(tetsB), _ptr(surfB), cap, _ptr(out), C.byref(np_), C.byref(tests),
                                        C.byref(lo))
            if rc == -1:
                cap = np_.value + 16
                continue
            if rc != 0:
                raise RuntimeError(f"or_run_pair_f failed: {rc}")
            return out[:np_.value].copy(), tests.value, lo.value

    def run_pairs(self, K, meshes_xyz_world, meshes, pairs, threads=0, rest=True):
        """Many pairs; meshes_xyz_world[i] are mesh i's world vertices, trees
        are built on the meshes' rest positions (rest=True) or on the world
        positions.  Returns (rows (n,3) = pair, a, b; tests per pair; pairs
        per pair)."""
        n = len(meshes)
        v_off = np.zeros(n + 1, np.int64)
        t_off = np.zeros(n + 1, np.int64)
        for i, m in enumerate(meshes):
            v_off[i + 1] = v_off[i] + m.n_verts
            t_off[i + 1] = t_off[i] + m.n_tets
        xyz = _c(np.concatenate(meshes_xyz_world, axis=0), np.float32)
        rxyz = _c(np.concatenate([m.xyz for m in meshes], axis=0), np.float32) if rest else None
        tets = _c(np.concatenate([m.tets for m in meshes], axis=0), np.uint32)
        surf = _c(np.concatenate([m.surf for m in meshes], axis=0), np.uint8)
        pairs = _c(pairs, np.uint32)
        npairs = pairs.shape[0]
        tpp = np.zeros(npairs, np.int64)
        ppp = np.zeros(npairs, np.int64)
        cap = 1 << 20
        while True:
            out = np.zeros((cap, 3), np.uint32)
            nout = _i64()
            rc = self.lib.or_run_pairs_f(K, n, _ptr(v_off), _ptr(xyz), _ptr(rxyz), _ptr(t_off), _ptr(tets), _ptr(surf),
                                         npairs,
                                         _ptr(pairs), threads, cap, _ptr(out), C.byref(nout), _ptr(tpp), _ptr(ppp))
            if rc == -1:
                cap = nout.value + 16
                continue
            if rc != 0:
                raise RuntimeError(f"or_run_pairs_f failed: {rc}")
            return out[:nout.value].copy(), tpp, ppp

    def surface_map(self, n_verts, tets) -> np.ndarray:
        tets = _c(tets, np.uint32)
        surf = np.zeros(tets.shape[0], np.uint8)
        self.lib.or_surface_map(n_verts, tets.shape[0], _ptr(tets), _ptr(surf))
        return surf

    def contacts(self, xyzA, tetsA, surfA, xyzB, tetsB, surfB, pairs, precision="f"):
        """Contacts of explicit tet pairs: (rows (n,8) p3 n3 d pair, records)."""
        tetsA, surfA = _c(tetsA, np.uint32), _c(surfA, np.uint8)
        tetsB, surfB = _c(tetsB, np.uint32), _c(surfB, np.uint8)
        pairs = _c(pairs, np.uint32).reshape(-1, 2)
        if precision == "dd":
            xyzA, xyzB = _c(xyzA, np.float64), _c(xyzB, np.float64)
            fn, dt = self.lib.or_contacts_dd, np.float64
        else:
            xyzA, xyzB = _c(xyzA, np.float32), _c(xyzB, np.float32)
            fn, dt = (self.lib.or_contacts_f, np.float32) if precision == "f" else (self.lib.or_contacts_d,
                                                                                   np.float64)
        rec = np.zeros(pairs.shape[0], OR_RECORD_DTYPE)
        cap = max(64, 8 * pairs.shape[0])
        while True:
            out = np.zeros((cap, 8), dt)
            n = _i64()
            rc = fn(_ptr(xyzA), _ptr(tetsA), _ptr(surfA), _ptr(xyzB), _ptr(tetsB), _ptr(surfB), pairs.shape[0],
                    _ptr(pairs), cap, _ptr(out), C.byref(n), _ptr(rec))
            if rc == -1:
                cap = n.value + 16
                continue
            return out[:n.value].copy(), rec

    def frozen_depth(self, a12, b12, rec):
        a12, b12 = _c(a12, np.float64), _c(b12, np.float64)
        r = OrRecord(*[int(rec[k]) for k in OR_RECORD_DTYPE.names])
        n = np.zeros(3, np.float64)
        d = self.lib.or_frozen_depth_d(_ptr(a12), _ptr(b12), C.byref(r), _ptr(n))
        return d, n

    def depth_grad(self, a12, b12, rec, gd, gn):
        a12, b12 = _c(a12, np.float64), _c(b12, np.float64)
        r = OrRecord(*[int(rec[k]) for k in OR_RECORD_DTYPE.names])
        gn = _c(gn, np.float64)
        g = np.zeros(24, np.float64)
        self.lib.or_depth_grad_d(_ptr(a12), _ptr(b12), C.byref(r), float(gd), _ptr(gn), _ptr(g))
        return g

    def frozen_batch(self, a12, b12, rec):
        """Frozen-decision depth (n,) and normal (n,3) of n pairs, double."""
        a12, b12 = _c(a12, np.float64).reshape(-1, 12), _c(b12, np.float64).reshape(-1, 12)
        rec = np.ascontiguousarray(rec, OR_RECORD_DTYPE)
        n = a12.shape[0]
        d = np.zeros(n, np.float64)
        nrm = np.zeros((n, 3), np.float64)
        self.lib.or_frozen_batch_d(n, _ptr(a12), _ptr(b12), _ptr(rec), _ptr(d), _ptr(nrm))
        return d, nrm

    def depth_grad_batch(self, a12, b12, rec, gd, gn):
        """Gradient (n,24) of gd*depth + gn.normal per pair, double."""
        a12, b12 = _c(a12, np.float64).reshape(-1, 12), _c(b12, np.float64).reshape(-1, 12)
        rec = np.ascontiguousarray(rec, OR_RECORD_DTYPE)
        n = a12.shape[0]
        gd = _c(gd, np.float64).reshape(n)
        gn = _c(gn, np.float64).reshape(n, 3)
        g = np.zeros((n, 24), np.float64)
        self.lib.or_depth_grad_batch_d(n, _ptr(a12), _ptr(b12), _ptr(rec), _ptr(gd), _ptr(gn), _ptr(g))
        return g

    def rotate(self, q, p, xyz) -> np.ndarray:
        q, p, xyz = _c(q, np.float32), _c(p, np.float32), _c(xyz, np.float32)
        out = np.zeros_like(xyz)
        self.lib.or_rotate_f(_ptr(q), _ptr(p), xyz.shape[0], _ptr(xyz), _ptr(out))
        return out

    def sin(self, x: float) -> float:
        return float(self.lib.or_sin_f(C.c_float(x)))

    @staticmethod
    def mesh_radius(xyz) -> np.float32:
        """Bounding radius of a mesh: max |r0| over its rest vertices, norm as
        sqrt(((x*x) + (y*y)) + (z*z)) in float (narrow_shape_types.h:189-206)."""
        x = _c(xyz, np.float32)
        if len(x) == 0:
            return np.float32(0)
        d = (x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1]) + x[:, 2] * x[:, 2]
        return np.float32(np.sqrt(d.astype(np.float32)).max())

    @staticmethod
    def broad_pairs(pos, radius) -> np.ndarray:
        """All-pair broad phase (broad_find_overlaps.h:44-125): boxes
        pos +- radius (prox_rigid_body.h:159-172) in float; (i, j), i < j,
        overlapping unless a max is strictly below a min; sorted."""
        p = _c(pos, np.float32)
        r = _c(radius, np.float32)
        lo = p - r[:, None]
        hi = p + r[:, None]
        n = len(p)
        out = []
        for i in range(n - 1):
            sep = (hi[i + 1:] < lo[i]) | (hi[i] < lo[i + 1:])
            js = np.nonzero(~sep.any(axis=1))[0] + i + 1
            out += [(i, int(j)) for j in js]
        return np.array(out, np.uint32).reshape(-1, 2)

    @staticmethod
    def reduce_contacts(rows, bodies):
        """PROX contact point reduction (prox_collision_detection.h:341-350):
        sort by ContactPoint::operator< (prox_contact_point.h:135-194: body i,
        body j, p.y, p.x, p.z, n.y, n.x, n.z, depth, each by float `<`), then
        std::unique with ContactPoint::operator== (:91-133: same bodies and
        every component |new - kept| not above working_precision<float>() =
        10 FLT_EPSILON, tiny_precision.h:21-24), which drops a row equal to the
        last row kept.  rows: (n, 7) float32 (p, n, depth); bodies: (n, 2).
        Returns (rows, bodies, source index) of the kept rows in sorted order
        (stable among rows whose keys all compare equal)."""
        r = _c(rows, np.float32).reshape(-1, 7)
        b = _c(bodies, np.uint32).reshape(-1, 2)
        n = len(r)
        if n == 0:
            return r.copy(), b.copy(), np.zeros(0, np.int64)
        # lexsort: last key most significant; float keys compare by value (-0 == +0)
        order = np.lexsort((r[:, 6], r[:, 5], r[:, 3], r[:, 4], r[:, 2], r[:, 0], r[:, 1], b[:, 1], b[:, 0]))
        rs, bs = r[order], b[order]
        eps = np.float32(np.float32(np.finfo(np.float32).eps) * np.float32(10))
        keep = np.ones(n, bool)
        # a row whose p.y differs from its predecessor's by more than eps (or
        # whose bodies differ) cannot equal any earlier row: segments between
        # such rows are independent; walk each longer one sequentially
        dy = np.abs(rs[1:, 1] - rs[:-1, 1])
        brk = np.ones(n, bool)
        brk[1:] = (dy > eps) | (bs[1:, 0] != bs[:-1, 0]) | (bs[1:, 1] != bs[:-1, 1])
        starts = np.nonzero(brk)[0]
        ends = np.append(starts[1:], n)
        for s0, e0 in zip(starts, ends):
            if e0 - s0 < 2:
                continue
            last = s0
            for j in range(s0 + 1, e0):
                d = np.abs(rs[j] - rs[last])
                if (d > eps).any():  # a NaN difference is not "above" eps
                    last = j
                else:
                    keep[j] = False
        return rs[keep], bs[keep], order[keep]

    def deform(self, amp, w, phase, xyz) -> np.ndarray:
        xyz = _c(xyz, np.float32)
        out = np.zeros_like(xyz)
        self.lib.or_deform_f(C.c_float(amp), C.c_float(w), C.c_float(phase), xyz.shape[0], _ptr(xyz), _ptr(out))
        return out


class Reference:
    """The reference's own CPU path, compiled from its sources (ref_harness.cpp)."""

    def __init__(self, path: str = REF_RECORD_SO):
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_surface_map.argtypes = [C.c_int, _p, C.c_int, _p, _p]
        L.ref_mesh_reorder.argtypes = [C.c_int, _p, C.c_int, _p, _p, _p]
        L.ref_rotate.argtypes = [_p, _p, C.c_int, _p, _p]
        L.ref_direction_table.argtypes = [C.c_int, _p]
        L.ref_contacts_pairs.argtypes = [C.c_int, _p, _p, _p, _p, _p, _p, C.c_longlong, _p, C.c_longlong, _p, _p]
        if hasattr(L, "ref_broad_pairs"):
            L.ref_broad_pairs.argtypes = [C.c_int, _p, _p, C.c_int, _p, C.c_longlong, _p]
            L.ref_mesh_radius.argtypes = [C.c_int, _p]
            L.ref_mesh_radius.restype = C.c_float
        if hasattr(L, "ref_reduce_contacts"):
            L.ref_reduce_contacts.argtypes = [C.c_longlong, _p, _p, C.c_int, _p, _p, _p]
        if hasattr(L, "ref_traverse"):
            L.ref_traverse.argtypes = [C.c_int, C.c_ulonglong, C.c_int, C.c_int, _p, _p, _p, C.c_int, _p,
                                       C.c_int, _p, _p, _p, C.c_int, _p, C.c_longlong, _p, _p, C.c_longlong, _p,
                                       _p, _p, C.c_longlong, _p, _p, _p]

    def surface_map(self, xyz, tets) -> np.ndarray:
        xyz, tets = _c(xyz, np.float32), _c(tets, np.uint32)
        out = np.zeros(tets.shape[0], np.uint8)
        self.lib.ref_surface_map(xyz.shape[0], _ptr(xyz), tets.shape[0], _ptr(tets), _ptr(out))
        return out

    def broad_pairs(self, pos, radius, algorithm: int = 0) -> np.ndarray:
        """broad::find_overlaps over boxes pos +- radius: 0 all-pair, 1 grid."""
        pos, radius = _c(pos, np.float32), _c(radius, np.float32)
        n = len(pos)
        cap = max(n * (n - 1) // 2, 1)
        out = np.zeros((cap, 2), np.uint32)
        cnt = C.c_longlong()
        rc = self.lib.ref_broad_pairs(n, _ptr(pos), _ptr(radius), algorithm, _ptr(out), cap, C.byref(cnt))
        if rc != 0:
            raise RuntimeError(f"ref_broad_pairs failed: {rc}")
        return out[:cnt.value]

    def mesh_radius(self, xyz) -> np.float32:
        xyz = _c(xyz, np.float32)
        return np.float32(self.lib.ref_mesh_radius(len(xyz), _ptr(xyz)))

    def reduce_contacts(self, rows, bodies):
        """PROX's std::sort + std::unique over ContactPoints (the reference's
        own comparisons); returns the kept (rows, bodies) in order."""
        r = _c(rows, np.float32).reshape(-1, 7)
        b = _c(bodies, np.uint32).reshape(-1, 2)
        n = len(r)
        out_r = np.zeros((max(n, 1), 7), np.float32)
        out_b = np.zeros((max(n, 1), 2), np.uint32)
        cnt = C.c_longlong()
        nb = int(b.max()) + 1 if n else 1
        rc = self.lib.ref_reduce_contacts(n, _ptr(r), _ptr(b), nb, _ptr(out_r), _ptr(out_b), C.byref(cnt))
        if rc != 0:
            raise RuntimeError(f"ref_reduce_contacts failed: {rc}")
        return out_r[:cnt.value], out_b[:cnt.value]

    def mesh_reorder(self, xyz, tets):
        xyz, tets = _c(xyz, np.float32), _c(tets, np.uint32)
        ox = np.zeros_like(xyz)
        ot = np.zeros_like(tets)
        rc = self.lib.ref_mesh_reorder(xyz.shape[0], _ptr(xyz), tets.shape[0], _ptr(tets), _ptr(ox), _ptr(ot))
        if rc != 0:
            raise RuntimeError("ref_mesh_reorder failed")
        return ox, ot

    def rotate(self, q, p, xyz) -> np.ndarray:
        q, p, xyz = _c(q, np.float32), _c(p, np.float32), _c(xyz, np.float32)
        out = np.zeros_like(xyz)
        self.lib.ref_rotate(_ptr(q), _ptr(p), xyz.shape[0], _ptr(xyz), _ptr(out))
        return out

    def direction_table(self, K) -> np.ndarray:
        out = np.zeros((13, 3), np.float32)
        n = self.lib.ref_direction_table(K, _ptr(out))
        if n < 0:
            raise ValueError(K)
        return out[:n].copy()

    def contacts(self, xyzA, tetsA, surfA, xyzB, tetsB, surfB, pairs, fp64=False):
        xyzA, tetsA, surfA = _c(xyzA, np.float32), _c(tetsA, np.uint32), _c(surfA, np.uint8)
        xyzB, tetsB, surfB = _c(xyzB, np.float32), _c(tetsB, np.uint32), _c(surfB, np.uint8)
        pairs = _c(pairs, np.uint32).reshape(-1, 2)
        cap = max(64, 8 * pairs.shape[0])
        while True:
            out = np.zeros((cap, 8), np.float64)
            n = C.c_longlong()
            self.lib.ref_contacts_pairs(1 if fp64 else 0, _ptr(xyzA), _ptr(tetsA), _ptr(surfA), _ptr(xyzB),
                                        _ptr(tetsB), _ptr(surfB), pairs.shape[0], _ptr(pairs), cap, _ptr(out),
                                        C.byref(n))
            if n.value > cap:
                cap = n.value + 16
                continue
            return out[:n.value].copy()

    def traverse(self, K, restA, qA, pA, tetsA, restB, qB, pB, tetsB, mem_bytes=(1 << 64) - 1, reorder=True,
                 want_volumes=False):
        """One pair through the reference pipeline: reorder + tree on the rest
        positions, pose (q, p), refit, tandem traversal.  Returns dict with
        pairs (n,2) in the caller's tet numbering (traversal order), contacts
        (m,8) rows p3 n3 d pair-row, tests, and optionally the preorder node
        volumes / leaf tets of tree A (one-chunk trees only)."""
        xyzA, tetsA = _c(restA, np.float32), _c(tetsA, np.uint32)
        xyzB, tetsB = _c(restB, np.float32), _c(tetsB, np.uint32)
        qA, pA, qB, pB = _c(qA, np.float32), _c(pA, np.float32), _c(qB, np.float32), _c(pB, np.float32)
        capp, capc = 1 << 16, 1 << 17
        nn = 2 * tetsA.shape[0] - 1
        while True:
            pairs = np.zeros((capp, 2), np.uint32)
            cont = np.zeros((capc, 8), np.float32)
            vols = np.zeros((nn, K), np.float32) if want_volumes else None
            leaf = np.zeros(nn, np.int64) if want_volumes else None
            npairs, ncont, tests, nnodes = C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_longlong()
            rc = self.lib.ref_traverse(K, C.c_ulonglong(mem_bytes), 1 if reorder else 0, xyzA.shape[0], _ptr(xyzA),
                                       _ptr(qA), _ptr(pA), tetsA.shape[0], _ptr(tetsA), xyzB.shape[0], _ptr(xyzB),
                                       _ptr(qB), _ptr(pB), tetsB.shape[0], _ptr(tetsB), capp, _ptr(pairs),
                                       C.byref(npairs), capc, _ptr(cont),
                                       C.byref(ncont), C.byref(tests), nn if want_volumes else 0, _ptr(vols),
                                       _ptr(leaf), C.byref(nnodes))
            if rc != 0:
                raise RuntimeError(f"ref_traverse failed: {rc}")
            if npairs.value > capp or ncont.value > capc:
                capp, capc = max(capp, npairs.value + 16), max(capc, ncont.value + 16)
                continue
            res = {"pairs": pairs[:npairs.value].copy(), "contacts": cont[:ncont.value].copy(),
                   "tests": tests.value}
            if want_volumes:
                res["volumes"] = vols
                res["leaf"] = leaf
            return res


class RefTimer:
    """Times the unmodified reference refit + tandem traversal over mesh pairs."""

    def __init__(self, path: str = REF_TIME_SO):
        self.lib = C.CDLL(path)
        self.lib.ref_time_pairs.argtypes = [C.c_int, C.c_ulonglong, C.c_int, _p, _p, _p, _p, _p, _p, C.c_longlong,
                                            _p, C.c_int, C.c_int, _p, _p]

    def time_pairs(self, K, meshes, quat, pos, pairs, threads=1, mem_bytes=(1 << 64) - 1, repeats=1):
        """Seconds for simulation steps of the reference over `pairs`: per
        pair, pose + refit of both meshes and the tandem traversal with
        contact generation (trees set up once, untimed, on the rest
        positions).  Returns (seconds of one step, contacts) for repeats == 1,
        else (list of per-step seconds, contacts of the last step)."""
        n = len(meshes)
        v_off = np.zeros(n + 1, np.int64)
        t_off = np.zeros(n + 1, np.int64)
        for i, m in enumerate(meshes):
            v_off[i + 1] = v_off[i] + m.n_verts
            t_off[i + 1] = t_off[i] + m.n_tets
        xyz = _c(np.concatenate([m.xyz for m in meshes], axis=0), np.float32)
        tets = _c(np.concatenate([m.tets for m in meshes], axis=0), np.uint32)
        quat, pos = _c(quat, np.float32), _c(pos, np.float32)
        pairs = _c(pairs, np.uint32)
        sec = np.zeros(max(int(repeats), 1), np.float64)
        cont = C.c_longlong()
        rc = self.lib.ref_time_pairs(K, C.c_ulonglong(mem_bytes), n, _ptr(v_off), _ptr(xyz), _ptr(quat), _ptr(pos),
                                     _ptr(t_off), _ptr(tets), pairs.shape[0], _ptr(pairs), threads, len(sec),
                                     _ptr(sec), C.byref(cont))
        if rc != 0:
            raise RuntimeError(f"ref_time_pairs failed: {rc}")
        return (float(sec[0]) if repeats == 1 else [float(x) for x in sec]), cont.value
