"""ctypes binding of libkdop_cuda.so (C ABI: include/kdop_cuda.h).

Mirrors the reference's kDOP interface for one simulation step
(SIMULATION/KDOP/KDOP/include): a DeviceScene replaces mesh_reorder +
make_tree for a set of meshes, refit() replaces refit_tree (with the rigid
transform of narrow_update_kdop_bvh.h done on the device), traverse() replaces
tandem_traversal over a pool of TestPairs, and contacts() returns what the
reference reports through ContactsCallback (point, normal, depth).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

HOST, DEVICE = 0, 1
REFIT_VERTICES, REFIT_POSE, REFIT_DEFORM = 0, 1, 2
TRAVERSE_BATCHED, TRAVERSE_PLAIN = 0, 1
BUILD_DEVICE, BUILD_HOST = 0, 1

_STATUS = {0: "ok", -1: "invalid argument", -2: "capacity exceeded", -3: "CUDA error",
           -4: "device wait timed out", -5: "out of memory", -6: "call out of order"}
ERR_INVALID, ERR_CAPACITY, ERR_CUDA, ERR_TIMEOUT, ERR_NOMEM, ERR_STATE = -1, -2, -3, -4, -5, -6

CONTACT_DTYPE = np.dtype([("p", np.float32, 3), ("n", np.float32, 3), ("depth", np.float32),
                          ("cand", np.uint32)])


class KdopError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"kdop: {_STATUS.get(status, status)}" + (f": {msg}" if msg else ""))
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [("n_verts", C.c_int64), ("xyz", C.c_void_p), ("n_tets", C.c_int64), ("tets", C.c_void_p),
                ("surface", C.c_void_p), ("leaf_order", C.c_void_p)]


class SceneInfo(C.Structure):
    _fields_ = [("K", C.c_int32), ("n_meshes", C.c_int32), ("n_verts", C.c_int64), ("n_tets", C.c_int64),
                ("n_nodes", C.c_int64), ("depth", C.c_int32), ("node_bytes", C.c_int32),
                ("device_bytes", C.c_int64), ("build", C.c_int32), ("host_orders", C.c_int32)]


class TraverseOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("surface_filter", C.c_int32), ("block_warps", C.c_int32),
                ("stack_cap", C.c_int32), ("init_chunk", C.c_int32), ("donate_min", C.c_int32),
                ("timeout_ms", C.c_int32), ("load_group", C.c_int32), ("wave_pairs", C.c_int32),
                ("smem_carveout", C.c_int32), ("test_stuck_work", C.c_int32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


class Stats(C.Structure):
    _fields_ = [("n_pairs", C.c_int64), ("n_tests", C.c_int64), ("n_leaf_overlaps", C.c_int64),
                ("n_candidates", C.c_int64), ("n_contacts", C.c_int64), ("candidate_capacity", C.c_int64),
                ("contact_capacity", C.c_int64), ("queue_capacity", C.c_int64), ("queue_used", C.c_int64),
                ("device_error", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


_LIB = None


def library_path() -> str:
    return os.environ.get("KDOP_CUDA_LIB", os.path.join(HERE, "libkdop_cuda.so"))


def load_library():
    """Load libkdop_cuda.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise KdopError(ERR_STATE, f"{path} is missing: build it with `make -C bvh-tvcg18_b200` "
                                   f"or __graft_entry__.build()")
    L = C.CDLL(path)
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
    sig = {
        "kdop_api_version": ([], i32),
        "kdop_status_string": ([i32], C.c_char_p),
        "kdop_last_error": ([vp], C.c_char_p),
        "kdop_ctx_create": ([i32, C.POINTER(vp)], i32),
        "kdop_ctx_destroy": ([vp], i32),
        "kdop_ctx_set_stream": ([vp, vp], i32),
        "kdop_ctx_stream": ([vp], vp),
        "kdop_ctx_synchronize": ([vp], i32),
        "kdop_ctx_launch_count": ([vp], i64),
        "kdop_scene_create": ([vp, i32, i32, C.POINTER(MeshDesc), C.POINTER(vp)], i32),
        "kdop_scene_create_ex": ([vp, i32, i32, C.POINTER(MeshDesc), i32, C.POINTER(vp)], i32),
        "kdop_scene_destroy": ([vp], i32),
        "kdop_scene_get_info": ([vp, C.POINTER(SceneInfo)], i32),
        "kdop_read_tree": ([vp, i32, i64, vp, vp, C.POINTER(i64)], i32),
        "kdop_set_vertices": ([vp, vp, i64, i32], i32),
        "kdop_set_poses": ([vp, vp, vp, i32], i32),
        "kdop_set_deformation": ([vp, C.c_float, C.c_float, C.c_float], i32),
        "kdop_refit": ([vp, i32], i32),
        "kdop_read_vertices": ([vp, vp, i64], i32),
        "kdop_traverse_opts_default": ([vp, C.POINTER(TraverseOpts)], i32),
        "kdop_traverse": ([vp, i64, vp, i32, C.POINTER(TraverseOpts)], i32),
        "kdop_get_stats": ([vp, C.POINTER(Stats)], i32),
        "kdop_reserve": ([vp, i64, i64, i64], i32),
        "kdop_set_capacity": ([vp, i64, i64, i64], i32),
        "kdop_read_candidates": ([vp, vp, i64, C.POINTER(i64)], i32),
        "kdop_contacts": ([vp], i32),
        "kdop_sort_results": ([vp], i32),
        "kdop_broad_phase": ([vp, vp, i32, vp, i64, C.POINTER(i64)], i32),
        "kdop_traverse_shard": ([vp, i64, vp, i32, C.POINTER(TraverseOpts), i32, i32, i64], i32),
        "kdop_read_contacts": ([vp, vp, i64, C.POINTER(i64)], i32),
        "kdop_reduce_contacts": ([vp, vp, vp, i64, C.POINTER(i64)], i32),
        "kdop_reduce_contact_rows": ([vp, vp, vp, i64, vp, vp, i64, C.POINTER(i64)], i32),
        "kdop_contacts_adjoint": ([vp, vp, vp, vp, i32], i32),
        "kdop_set_motion": ([vp, vp, vp, C.c_float, i32], i32),
        "kdop_graph_capture": ([vp, i32, i64, vp, i32, C.POINTER(TraverseOpts), i32], i32),
        "kdop_graph_launch": ([vp], i32),
        "kdop_graph_release": ([vp], i32),
        "kdop_autotune": ([vp, i64, vp, i32, i32, C.POINTER(TraverseOpts)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    if hasattr(a, "data_ptr"):  # torch tensor
        return C.c_void_p(a.data_ptr())
    raise TypeError(type(a))


def _mem(a) -> int:
    if hasattr(a, "is_cuda") and a.is_cuda:
        return DEVICE
    return HOST


def _host(a, dtype):
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a, dtype=dtype)


def _arg(a, dtype):
    """Host numpy array or a contiguous CUDA tensor of the right dtype."""
    if hasattr(a, "is_cuda") and a.is_cuda:
        import torch
        tdt = {np.float32: torch.float32, np.uint32: torch.int32}[dtype]
        if a.dtype != tdt:
            a = a.to(tdt)
        return a.contiguous()
    return _host(a, dtype)


class Context:
    """One CUDA device and stream (kdop_ctx)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.kdop_ctx_create(device, C.byref(h))
        if rc != 0:
            raise KdopError(rc, f"kdop_ctx_create(device={device})")
        self.h = h
        self.device = device
        if stream is not None:
            self._check(self.lib.kdop_ctx_set_stream(self.h, C.c_void_p(stream)))

    def _check(self, rc: int, what: str = ""):
        if rc != 0:
            msg = self.lib.kdop_last_error(self.h)
            raise KdopError(rc, (msg.decode() if msg else "") or what)
        return rc

    def reduce_contact_rows(self, rows, bodies):
        """PROX contact reduction of any rows (CONTACT_DTYPE) with their bodies
        ((n, 2) uint32) via kdop_reduce_contact_rows: (kept rows, bodies)."""
        rows = np.ascontiguousarray(rows, CONTACT_DTYPE)
        bodies = np.ascontiguousarray(bodies, np.uint32).reshape(-1, 2)
        n = len(rows)
        out = np.zeros(max(n, 1), CONTACT_DTYPE)
        ob = np.zeros((max(n, 1), 2), np.uint32)
        nr = C.c_int64()
        self._check(self.lib.kdop_reduce_contact_rows(self.h, _ptr(rows), _ptr(bodies), n, _ptr(out), _ptr(ob), n,
                                                      C.byref(nr)), "kdop_reduce_contact_rows")
        return out[:nr.value], ob[:nr.value]

    @property
    def stream(self) -> int:
        return int(self.lib.kdop_ctx_stream(self.h) or 0)

    def synchronize(self):
        self._check(self.lib.kdop_ctx_synchronize(self.h))

    @property
    def launches(self) -> int:
        return int(self.lib.kdop_ctx_launch_count(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.kdop_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceScene:
    """Meshes and their kDOP trees on the device (kdop_scene)."""

    def __init__(self, ctx: Context, K: int, meshes: Sequence, surface: bool = True, build: int = 0):
        """build: BUILD_DEVICE (trees built on the GPU) or BUILD_HOST."""
        self.ctx = ctx
        self.lib = ctx.lib
        self.K = K
        descs = (MeshDesc * max(len(meshes), 1))()
        self._keep = []
        self.v_off = np.zeros(len(meshes) + 1, np.int64)
        self.t_off = np.zeros(len(meshes) + 1, np.int64)
        for i, m in enumerate(meshes):
            xyz = np.ascontiguousarray(m.xyz, np.float32)
            tets = np.ascontiguousarray(m.tets, np.uint32)
            surf = np.ascontiguousarray(m.surf, np.uint8) if (surface and m.surf is not None) else None
            self._keep += [xyz, tets, surf]
            order = getattr(m, "leaf_order", None)
            order = None if order is None else np.ascontiguousarray(order, np.uint32)
            self._keep.append(order)
            descs[i] = MeshDesc(xyz.shape[0], _ptr(xyz), tets.shape[0], _ptr(tets), _ptr(surf), _ptr(order))
            self.v_off[i + 1] = self.v_off[i] + xyz.shape[0]
            self.t_off[i + 1] = self.t_off[i] + tets.shape[0]
        h = C.c_void_p()
        ctx._check(self.lib.kdop_scene_create_ex(ctx.h, K, len(meshes), descs, build, C.byref(h)),
                   "kdop_scene_create")
        self._keep = []
        self.h = h
        self.n_meshes = len(meshes)
        self.pairs = None

    # ---- info ----
    def info(self) -> dict:
        inf = SceneInfo()
        self.ctx._check(self.lib.kdop_scene_get_info(self.h, C.byref(inf)))
        return {k: int(getattr(inf, k)) for k, _ in inf._fields_}

    def read_tree(self, mesh: int):
        nt = int(self.t_off[mesh + 1] - self.t_off[mesh])
        nn = max(2 * nt - 1, 0)
        vol = np.zeros((max(nn, 1), self.K), np.float32)
        tet = np.zeros(max(nn, 1), np.int64)
        n = C.c_int64()
        self.ctx._check(self.lib.kdop_read_tree(self.h, mesh, nn, _ptr(vol), _ptr(tet), C.byref(n)))
        return vol[:n.value], tet[:n.value]

    # ---- positions / refit ----
    def set_vertices(self, xyz):
        a = _arg(xyz, np.float32)
        n = a.shape[0] if a.ndim == 2 else a.size // 3
        self.ctx._check(self.lib.kdop_set_vertices(self.h, _ptr(a), n, _mem(a)), "kdop_set_vertices")

    def set_poses(self, quat, pos):
        q, p = _arg(quat, np.float32), _arg(pos, np.float32)
        self.ctx._check(self.lib.kdop_set_poses(self.h, _ptr(q), _ptr(p), _mem(q)), "kdop_set_poses")

    def set_deformation(self, amp: float, w: float, phase: float):
        self.ctx._check(self.lib.kdop_set_deformation(self.h, amp, w, phase))

    def set_motion(self, lin_vel, ang_vel, phase_rate: float):
        l, a = _arg(lin_vel, np.float32), _arg(ang_vel, np.float32)
        self.ctx._check(self.lib.kdop_set_motion(self.h, _ptr(l), _ptr(a), phase_rate, _mem(l)))

    def refit(self, mode: int = REFIT_VERTICES):
        self.ctx._check(self.lib.kdop_refit(self.h, mode), "kdop_refit")

    def read_vertices(self) -> np.ndarray:
        n = int(self.v_off[-1])
        out = np.zeros((max(n, 1), 3), np.float32)
        self.ctx._check(self.lib.kdop_read_vertices(self.h, _ptr(out), n))
        return out[:n]

    # ---- traversal ----
    def default_opts(self) -> TraverseOpts:
        o = TraverseOpts()
        self.lib.kdop_traverse_opts_default(self.h, C.byref(o))
        return o

    def opts(self, **kw) -> TraverseOpts:
        o = self.default_opts()
        for k, v in kw.items():
            setattr(o, k, int(v))
        return o

    def traverse(self, pairs, opts: Optional[TraverseOpts] = None):
        p = _arg(pairs, np.uint32)
        n = p.shape[0] if p.ndim == 2 else p.size // 2
        self.pairs = p
        self.ctx._check(self.lib.kdop_traverse(self.h, n, _ptr(p), _mem(p), C.byref(opts) if opts else None),
                        "kdop_traverse")

    def broad_phase(self, positions=None) -> np.ndarray:
        """(n, 2) uint32 mesh pairs whose bounding boxes overlap (i < j, sorted);
        positions: (n_meshes, 3) or None for the poses of set_poses."""
        pos = None if positions is None else _arg(positions, np.float32)
        n = C.c_int64()
        cap = 1 << 16
        while True:
            out = np.zeros((cap, 2), np.uint32)
            rc = self.lib.kdop_broad_phase(self.h, _ptr(pos), _mem(pos) if pos is not None else HOST, _ptr(out), cap,
                                           C.byref(n))
            if rc == ERR_CAPACITY and n.value > cap:
                cap = n.value
                continue
            self.ctx._check(rc, "kdop_broad_phase")
            return out[:n.value]

    def traverse_shard(self, pairs, rank: int, n_ranks: int, frontier_min: int = 16384,
                       opts: Optional[TraverseOpts] = None):
        """Shard `rank` of `n_ranks` of the traversal (frontier-seeded): the
        shards' candidates and test counts together equal traverse()'s."""
        p = _arg(pairs, np.uint32)
        n = p.shape[0] if p.ndim == 2 else p.size // 2
        self.pairs = p
        self.ctx._check(self.lib.kdop_traverse_shard(self.h, n, _ptr(p), _mem(p), C.byref(opts) if opts else None,
                                                     int(rank), int(n_ranks), int(frontier_min)),
                        "kdop_traverse_shard")

    def stats(self, check: bool = True) -> Stats:
        st = Stats()
        rc = self.lib.kdop_get_stats(self.h, C.byref(st))
        if check:
            self.ctx._check(rc, "kdop_get_stats")
        st.status = rc
        return st

    def reserve(self, candidates: int = 0, contacts: int = 0, queue: int = 0):
        self.ctx._check(self.lib.kdop_reserve(self.h, int(candidates), int(contacts), int(queue)))

    def set_capacity(self, candidates: int = 0, contacts: int = 0, queue: int = 0):
        self.ctx._check(self.lib.kdop_set_capacity(self.h, int(candidates), int(contacts), int(queue)))

    def traverse_sync(self, pairs, opts: Optional[TraverseOpts] = None, contacts: bool = False,
                      max_retries: int = 6) -> Stats:
        """Traverse (and optionally generate contacts), growing buffers and
        retrying on KDOP_ERR_CAPACITY."""
        for _ in range(max_retries):
            self.traverse(pairs, opts)
            if contacts:
                self.contacts()
            st = self.stats(check=False)
            if st.status == 0:
                return st
            if st.status != ERR_CAPACITY:
                self.ctx._check(st.status, "traversal")
            grow_c = st.n_candidates > st.candidate_capacity
            grow_k = st.n_contacts > st.contact_capacity
            grow_q = bool(st.device_error & 2)
            self.reserve(candidates=int(st.n_candidates * 1.25) + 1024 if grow_c else 0,
                         contacts=int(st.n_contacts * 1.25) + 1024 if grow_k else 0,
                         queue=max(2 * st.queue_capacity, int(st.queue_used * 1.25) + 1024) if grow_q else 0)
        raise KdopError(ERR_CAPACITY, "buffers still too small after retries")

    def candidates(self) -> np.ndarray:
        """(n, 3) uint32 rows: pair index, tet of A, tet of B (mesh-local)."""
        st = self.stats(check=False)
        n = min(st.n_candidates, st.candidate_capacity)
        rows = np.zeros((max(n, 1), 3), np.uint32)
        nr = C.c_int64()
        self.ctx._check(self.lib.kdop_read_candidates(self.h, _ptr(rows), n, C.byref(nr)))
        return rows[:nr.value]

    # ---- contacts ----
    def contacts(self):
        self.ctx._check(self.lib.kdop_contacts(self.h), "kdop_contacts")

    def sort_results(self):
        """Reproducible order of the last traversal's results (device sort):
        candidates by (pair, tet A, tet B), contacts grouped to match."""
        self.ctx._check(self.lib.kdop_sort_results(self.h), "kdop_sort_results")

    def read_contacts(self) -> np.ndarray:
        st = self.stats(check=False)
        n = min(st.n_contacts, st.contact_capacity)
        rows = np.zeros(max(n, 1), CONTACT_DTYPE)
        nr = C.c_int64()
        self.ctx._check(self.lib.kdop_read_contacts(self.h, _ptr(rows), n, C.byref(nr)))
        return rows[:nr.value]

    def reduce_contacts(self):
        """PROX contact reduction of the last kdop_contacts (kdop_reduce_contacts):
        (kept rows, their bodies (n, 2) = the meshes of the rows' pairs)."""
        st = self.stats(check=False)
        n = min(st.n_contacts, st.contact_capacity)
        rows = np.zeros(max(n, 1), CONTACT_DTYPE)
        bodies = np.zeros((max(n, 1), 2), np.uint32)
        nr = C.c_int64()
        self.ctx._check(self.lib.kdop_reduce_contacts(self.h, _ptr(rows), _ptr(bodies), n, C.byref(nr)),
                        "kdop_reduce_contacts")
        return rows[:nr.value], bodies[:nr.value]

    def read_contacts_into(self, buf) -> int:
        """Contact rows into `buf` (host array or CUDA tensor of at least
        32 bytes per row); returns the number of rows."""
        st = self.stats(check=False)
        n = min(st.n_contacts, st.contact_capacity)
        nr = C.c_int64()
        self.ctx._check(self.lib.kdop_read_contacts(self.h, _ptr(buf), n, C.byref(nr)))
        return nr.value

    def adjoint(self, d_depth, d_normal, grad):
        """grad += dL/d(world vertex positions); arrays host numpy or CUDA tensors."""
        self.ctx._check(self.lib.kdop_contacts_adjoint(self.h, _ptr(d_depth), _ptr(d_normal), _ptr(grad),
                                                       _mem(grad)), "kdop_contacts_adjoint")

    # ---- graph / tuning ----
    def graph_capture(self, pairs, refit_mode: int = REFIT_POSE, opts: Optional[TraverseOpts] = None,
                      motion: bool = False):
        p = _arg(pairs, np.uint32)
        n = p.shape[0] if p.ndim == 2 else p.size // 2
        self.pairs = p
        self.ctx._check(self.lib.kdop_graph_capture(self.h, refit_mode, n, _ptr(p), _mem(p),
                                                    C.byref(opts) if opts else None, 1 if motion else 0),
                        "kdop_graph_capture")

    def graph_launch(self):
        self.ctx._check(self.lib.kdop_graph_launch(self.h), "kdop_graph_launch")

    def graph_release(self):
        self.lib.kdop_graph_release(self.h)

    def autotune(self, pairs, repeats: int = 2) -> TraverseOpts:
        p = _arg(pairs, np.uint32)
        n = p.shape[0] if p.ndim == 2 else p.size // 2
        best = TraverseOpts()
        self.ctx._check(self.lib.kdop_autotune(self.h, n, _ptr(p), _mem(p), repeats, C.byref(best)),
                        "kdop_autotune")
        return best

    def close(self):
        if getattr(self, "h", None):
            self.lib.kdop_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
