"""The C++ drop-in binding (include/kdop_cuda_tag.hpp) driven by the
reference's own narrow-phase calls: oracle/_ref/adapter_check runs
make_tree / refit_tree / tandem_traversal once with kdop::sequential and once
with the kdop::cuda tag on the same meshes and exits 0 when node volumes are
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
