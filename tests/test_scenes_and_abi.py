"""Synthetic scenes and the C ABI surface (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from kdop_b200 import scenes


def signed_volumes(m):
    p = m.xyz.astype(np.float64)[m.tets.astype(np.int64)]
    return np.einsum("ij,ij->i", p[:, 3] - p[:, 0], np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])) / 6.0


@pytest.mark.parametrize("n,jit", [(1, 0.0), (3, 0.0), (5, 0.2)])
def test_lattice_orientation_and_counts(n, jit):
    m = scenes.lattice(n, jit, np.random.default_rng(0))
    assert m.n_tets == 6 * n ** 3 and m.n_verts == (n + 1) ** 3
    assert np.all(signed_volumes(m) > 0)
    # a tet is interior iff none of its faces is on the boundary
    surf_faces = int(sum(bin(int(s)).count("1") for s in m.surf))
    assert surf_faces == 2 * 6 * n * n  # two triangles per boundary square


def test_config_shapes():
    sc = scenes.config3(n_pairs=16, seed=2)
    assert len(sc.meshes) == 32 and sc.pairs.shape == (16, 2) and sc.K == 14
    for m in sc.meshes:
        n = round((m.n_tets / 6) ** (1 / 3))
        assert 6 <= n <= 32
    c5 = scenes.config5(n_pairs=2, n=3)
    assert c5.K == 14 and len(c5.meshes) == 4


def header_symbols():
    src = open(os.path.join(ROOT, "include", "kdop_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kdop_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(cuda_library_path):
    lib = ctypes.CDLL(cuda_library_path)
    names = header_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_status_strings_without_gpu(cuda_library_path):
    lib = ctypes.CDLL(cuda_library_path)
    lib.kdop_status_string.restype = ctypes.c_char_p
    assert lib.kdop_api_version() == 1
    assert lib.kdop_status_string(-2) == b"capacity exceeded"
    # null handles are rejected, not dereferenced
    assert lib.kdop_scene_destroy(None) == -1
    assert lib.kdop_ctx_destroy(None) == -1


def test_python_binding_fails_loudly_without_library(monkeypatch, tmp_path):
    from kdop_b200 import lib
    monkeypatch.setenv("KDOP_CUDA_LIB", str(tmp_path / "missing.so"))
    monkeypatch.setattr(lib, "_LIB", None)
    with pytest.raises(lib.KdopError):
        lib.load_library()
