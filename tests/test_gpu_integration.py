"""The drop-in check on a GPU: the reference engine, built from its own sources, renders through the
`cuda` backend adapter (optical-pathtracer_b200/owe_adapter/cuda_backend.cpp) and libowec.so, and
matches the white-furnace answer and its own cpu backend (oracle/integration_main.cpp)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "owe_cuda_integration")


def test_reference_engine_renders_through_the_cuda_backend():
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/owe_cuda_integration was not built (the reference sources were absent)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
