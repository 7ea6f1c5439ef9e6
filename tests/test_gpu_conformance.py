"""The reference's own backend conformance suite (tests/test_backends.cpp and tests/test_references.cpp
of the reference, compiled from its sources with its harness) run with the `cuda` backend in its
registry (oracle/Makefile, target conformance): every check the suite makes of every backend it
finds, analytic known answers and statistical agreement with the reference's CPU transport, now also
made of this backend through the adapter, exactly as the reference's tests would after the
registry line is added.

The harness prints `[backend]` before each backend's part of a test and one line per failed CHECK;
this test attributes those lines to the backend they follow."""
import os
import re
import subprocess

import pytest

from conftest import save_artifact

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DIR = os.path.join(ROOT, "oracle", "_ref", "conformance")
BIN = os.path.join(DIR, "owe_conformance")

# Cases that cannot run here on any backend, with the reason: their scene files name model files
# that the reference ships as Git LFS pointers, absent from its checkout (the_lens.owe's table, the
# telescope's ground relief), so loading the scene throws before any backend renders.
MISSING_DATA = {"backends_reset_observer_matches_fresh_render",
                "backends_agree_with_reference_through_instruments_and_cameras"}


def parse(text):
    """{test: {"status": "OK"|"FAIL", "backends": [names run], "failures": {backend: [lines]}}}"""
    out, cur, backend = {}, None, None
    for line in text.splitlines():
        m = re.match(r"\[ RUN  \] (\S+)", line)
        if m:
            cur, backend = m.group(1), None
            out[cur] = {"status": None, "backends": [], "failures": {}}
            continue
        if cur is None:
            continue
        m = re.match(r"\[ ( OK |FAIL) \] (\S+)", line)
        if m:
            out[cur]["status"] = m.group(1).strip()
            cur = None
            continue
        m = re.match(r"    \[(\w+)\](\s|$)", line)
        if m:
            backend = m.group(1)
            out[cur]["backends"].append(backend)
            continue
        if "cannot open" in line:
            out[cur]["failures"].setdefault("(data)", []).append(line.strip())
        elif "CHECK" in line or "expected" in line or "exception" in line:
            out[cur]["failures"].setdefault(backend or "(before any backend)", []).append(line.strip())
    return out


def test_reference_conformance_suite_passes_on_cuda():
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/conformance/owe_conformance is not built (the reference sources were absent)")
    r = subprocess.run([BIN, "backends_", "reference_"], cwd=DIR, capture_output=True, text=True, timeout=1500)
    text = r.stdout + r.stderr
    save_artifact("conformance_log", log=text)
    res = parse(text)
    assert res, text[-2000:]
    ran_on_cuda = [t for t, v in res.items() if "cuda" in v["backends"]]
    # a missing model file met while a listed case runs a backend's turn is the data's failure, not
    # the backend's
    data_error = ("OBJ file has no faces", "cannot read image", "cannot open")
    cuda_failures = {t: v["failures"]["cuda"] for t, v in res.items() if "cuda" in v["failures"]
                     and not (t in MISSING_DATA and all(any(e in l for e in data_error) for l in v["failures"]["cuda"]))}
    other = {t: v["failures"] for t, v in res.items() if v["status"] == "FAIL" and t not in MISSING_DATA
             and "cuda" not in v["failures"]}
    assert not cuda_failures, cuda_failures
    assert not other, other
    # every backend test the reference could run reached the cuda backend, and so did the known
    # answers it checks on every light-tracing backend (its ripple-caustic check names the "gpu"
    # backend alone; tests/test_gpu_waves.py runs that known answer on cuda)
    backend_tests = [t for t in res if t.startswith("backends_") and t not in MISSING_DATA]
    light_tests = ["reference_lens_focuses_sunlight_with_its_fresnel_losses",
                   "reference_water_surface_transmits_the_fresnel_share", "reference_concave_mirror_concentrates_sunlight"]
    missing = sorted(set(backend_tests + light_tests) - set(ran_on_cuda))
    assert not missing, missing
