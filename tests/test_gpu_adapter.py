"""The C++ drop-in binding (include/kdop_cuda_tag.hpp) driven by the
reference's own narrow-phase calls: oracle/_ref/adapter_check runs
make_tree / refit_tree / tandem_traversal once with kdop::sequential and once
with the kdop::cuda tag on the same meshes, over several simulation steps
(the tag's device scenes persist between them), for one-chunk trees (K = 8,
14, 26) and the narrow phase's default 8000-byte chunked trees (K = 8, 14;
branches and a super-chunk level), and for pools whose mesh sets change
between steps (one body shared by two pairs; a cached scene reused), and
exits 0 when every node volume of every chunk level and the root kDOP are
bit-identical and the callbacks received the same contacts."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "adapter_check")


@pytest.mark.gpu
def test_reference_calls_through_the_cuda_tag():
    if not os.path.exists(BIN):
        pytest.skip("adapter_check not built (make -C oracle adapter needs the reference headers)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


@pytest.mark.gpu
def test_cuda_tag_loop_timing():
    """100 narrow-phase steps (pose, refit_tree of both bodies, tandem_traversal
    with contacts) through the kdop::cuda tag with the default 8000-byte
    chunked trees, beside the same loop through kdop::sequential; the tag
    keeps its device scenes between steps.  Prints milliseconds per step."""
    if not os.path.exists(BIN):
        pytest.skip("adapter_check not built (make -C oracle adapter needs the reference headers)")
    r = subprocess.run([BIN, "--time", "100", "16"], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "loop K=8" in r.stdout
