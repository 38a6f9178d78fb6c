"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
a CPU-only machine.  The CPU oracle and the CUDA library are built on demand
(make) when their shared objects are missing."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bvh-tvcg18_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_golden.npz")
GOLDEN_LARGE = os.path.join(ROOT, "tests", "golden", "reference_large.json")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from make_golden_large import canonical_candidates, canonical_contacts, digest  # noqa: E402,F401


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _make(args):
    subprocess.run(["make", "-s"] + args, cwd=ROOT, check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    if not pyoracle.available():
        _make(["-C", "oracle", "oracle"])
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference's own CPU code (only where it has been compiled)."""
    from oracle import pyoracle
    if not pyoracle.reference_available():
        pytest.skip("reference harness not built (oracle/_ref)")
    return pyoracle.Reference()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def golden_large():
    """Digests of the reference's own results on the full-size workloads."""
    import json
    with open(GOLDEN_LARGE) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def cuda_library_path():
    from kdop_b200 import lib
    path = lib.library_path()
    if not os.path.exists(path):
        _make(["-C", "bvh-tvcg18_b200"])
    return path


@pytest.fixture(scope="session")
def ctx(cuda_library_path):
    import kdop_b200
    return kdop_b200.Context(0)


def world_xyz(oracle, scene, i):
    """World positions of mesh i of a scene (the oracle's rotate + translate)."""
    m = scene.meshes[i]
    return oracle.rotate(scene.quat[i], scene.pos[i], m.xyz)


def sorted_rows(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a)
    if a.size == 0:
        return a.reshape(0, a.shape[1] if a.ndim == 2 else 2)
    keys = tuple(a[:, k] for k in reversed(range(a.shape[1])))
    return a[np.lexsort(keys)]
