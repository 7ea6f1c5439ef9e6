"""The reference's own scene files on `cuda`: every file in its scenes/ and benchmarks/ folders (the
`owe bench` suites of benchmarks/suites.json among them), loaded by the reference engine's loader
and rendered on its `cpu` backend and on `cuda` through the registry, compared by the reference's
compareRenderers statistics at a reduced film size, every detector of each scene
(oracle/scene_suite_main.cpp, built by oracle/Makefile into oracle/_ref/conformance)."""
import glob
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.join(ROOT, "oracle", "_ref", "conformance")
BIN = os.path.join(HERE, "owe_scene_suite")
# what this checkout of the reference lacks: its image assets, and model files stored as Git LFS
# pointers; the reference cannot load those scenes either
MISSING_DATA = ("cannot read image", "OBJ file has no faces", "cannot open")


def test_reference_scene_files_render_alike_on_cuda():
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/conformance/owe_scene_suite was not built (the reference sources were absent)")
    files = sorted(os.path.relpath(p, HERE) for pattern in ("scenes/*.owe", "scenes/*/*.owe", "benchmarks/*.owe",
                                                              "benchmarks/*/*.owe")
                   for p in glob.glob(os.path.join(HERE, pattern)))
    r = subprocess.run([BIN, "--all-detectors", "--spp", "16", "--runs", "8"] + files, cwd=HERE, capture_output=True, text=True, timeout=1500)
    print(r.stdout)
    lines = r.stdout.splitlines()
    fails = [l for l in lines if l.startswith("FAIL")]
    refused = [l for l in lines if l.startswith("REFUSED")]
    unloadable = [l for l in lines if l.startswith("LOAD-FAILED") and not any(m in l for m in MISSING_DATA)]
    ok = [l for l in lines if l.startswith("ok")]
    # Scenes whose light reaches the film only along rare paths (a sunbeam through a pinhole and
    # glass onto a screen, which next-event estimation cannot reach through the glass) give
    # heavy-tailed runs, and eight of them can fail the block test by chance: each such scene is
    # compared once more with four times the runs and samples, which a real bias fails more clearly.
    retried = []
    for line in fails:
        name = line.split()[1]
        r2 = subprocess.run([BIN, "--all-detectors", "--spp", "64", "--runs", "32", name], cwd=HERE, capture_output=True,
                            text=True, timeout=1500)
        print(r2.stdout)
        retried.append((name, [l for l in r2.stdout.splitlines() if l.startswith("FAIL")]))
    assert all(not f for _, f in retried), retried
    assert not refused, refused
    assert not unloadable, unloadable
    assert len(ok) + len(fails) >= 30, r.stdout + r.stderr
    assert r.returncode == 0 or fails
