"""CPU checks of the boundary: the CUDA library loads and exports every function include/owec.h
declares, the ctypes mirror matches the C struct layouts, and the procedural workloads are what
they claim to be. No GPU calls."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import owec_abi as A
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = A.load_library()
    declared = A.declared_symbols()
    assert len(declared) >= 17
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/owec.h but not exported"
    assert lib.owec_abi_version() == A.ABI_VERSION


def test_library_is_built_for_sm_100a_only():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", A.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_struct_layouts_match_the_header():
    # Sizes the C compiler gives include/owec.h's structs (x86-64 SysV), checked with a tiny probe.
    src = r'''
    #include <stdio.h>
    #include "owec.h"
    int main(void) {
      printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(owec_spectrum), sizeof(owec_medium),
        sizeof(owec_optics), sizeof(owec_emission), sizeof(owec_boundary), sizeof(owec_mesh),
        sizeof(owec_environment), sizeof(owec_detector), sizeof(owec_scene_desc), sizeof(owec_settings),
        sizeof(owec_stats));
      return 0; }
    '''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "probe")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        sizes = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    mine = [ctypes.sizeof(t) for t in (A.Spectrum, A.Medium, A.Optics, A.Emission, A.Boundary, A.Mesh,
                                        A.Environment, A.Detector, A.SceneDesc, A.Settings, A.Stats)]
    assert sizes == mine


def test_uv_sphere_has_two_to_the_twenty_triangles_and_closes():
    v, t = scenes.uv_sphere(1024, 512)
    assert len(t) == 1 << 20
    # closed and consistently oriented: every edge appears once in each direction
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]).astype(np.int64)
    key = e[:, 0] * len(v) + e[:, 1]
    rkey = e[:, 1] * len(v) + e[:, 0]
    assert len(np.unique(key)) == len(key)
    assert np.array_equal(np.sort(key), np.sort(rkey))
    r = np.linalg.norm(v, axis=1)
    assert r.min() >= 0.95 - 1e-12 and r.max() <= 1.05 + 1e-12
    # outward: the signed volume is positive
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    assert np.einsum("ij,ij->i", a, np.cross(b, c)).sum() > 0


def test_gradient_noise_is_seeded_and_bounded():
    p = np.random.default_rng(0).uniform(-3, 3, (10000, 3))
    a = scenes.gradient_noise3(p, 7)
    b = scenes.gradient_noise3(p, 7)
    c = scenes.gradient_noise3(p, 8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(a).max() < 1.5 and a.std() > 0.1


def test_scene_descriptions_are_well_formed():
    for sb in (scenes.glass_sphere_on_floor(8, 8), scenes.bvh_stress_room(8, 8, 64, 32), scenes.furnace_sphere(0.5),
               scenes.invisible_sphere()):
        d = sb.desc()
        assert d.abi_version == A.ABI_VERSION and d.n_regions >= 1
        for i in range(d.n_boundaries):
            b = d.boundaries[i]
            assert b.front < d.n_regions and b.back < d.n_regions and b.optics < d.n_optics
            R = np.array(b.to_world[:]).reshape(3, 4)[:, :3]
            assert np.allclose(R @ R.T, np.eye(3), atol=1e-12)
