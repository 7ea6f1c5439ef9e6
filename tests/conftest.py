import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "optical-pathtracer_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def save_artifact(name, **arrays):
    """Writes arrays to $OWEC_TEST_ARTIFACTS/<name>.npz when that directory is set (diagnostics of a
    failed comparison); does nothing otherwise."""
    import numpy as np
    out = os.environ.get("OWEC_TEST_ARTIFACTS")
    if out:
        os.makedirs(out, exist_ok=True)
        np.savez_compressed(os.path.join(out, name + ".npz"), **arrays)
