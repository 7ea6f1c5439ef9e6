"""The restatement (oracle/owe_oracle.cpp) pinned against the reference engine (oracle/_ref) and
the reference's known answers. CPU only."""
import numpy as np
import pytest

import owec_abi as A
import scenes
from oracle_ref import PortEngine, ReferenceEngine


def test_port_cast_rays_equal_world_intersect():
    desc = scenes.bvh_stress_room(8, 8, n_lon=128, n_lat=64).desc()
    o, d = scenes.random_rays(20000, 5, (-2.8, -2.8, 0.1), (2.8, 2.8, 3.9), (-1.1, -1.1, 0.1), (1.1, 1.1, 2.3))
    rb, rp, rt = ReferenceEngine(desc).cast_rays(o, d)
    pb, pp, pt = PortEngine(desc).cast_rays(o, d)
    assert np.array_equal(rb, pb) and np.array_equal(rp, pp)
    hit = rb != A.KNONE
    assert np.max(np.abs(rt[hit] - pt[hit]) / rt[hit]) < 1e-12


def test_port_light_table_equals_reference():
    desc = scenes.bvh_stress_room(8, 8, n_lon=32, n_lat=16).desc()
    assert np.allclose(PortEngine(desc).light_pdfs(), ReferenceEngine(desc).info()["light_pdfs"], rtol=1e-12)
    desc = scenes.glass_sphere_on_floor(8, 8).desc()
    assert np.allclose(PortEngine(desc).light_pdfs(), ReferenceEngine(desc).info()["light_pdfs"], rtol=1e-12)


@pytest.mark.parametrize("mode", [A.WAVELENGTHS_UNIFORM1, A.WAVELENGTHS_HERO4])
def test_port_paths_equal_reference_paths(mode):
    """Both are IEEE double with the same draw order: one-sample passes agree pixel for pixel
    (apart from rare contact-order differences)."""
    desc = scenes.glass_sphere_on_floor(48, 48).desc()
    s = A.make_settings(seed=9, max_depth=16, rr_depth=4, wavelength_mode=mode)
    a, sa = ReferenceEngine(desc).render(s, 1, passes=2)
    b, sb = PortEngine(desc).render(s, 1, passes=2)
    close = np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), 1e-12)
    assert close.mean() > 0.999
    assert sa["paths"] == sb["paths"]
    assert abs(sa["segments"] - sb["segments"]) <= 0.001 * sa["segments"]


def test_port_matches_reference_on_the_area_lit_room():
    desc = scenes.bvh_stress_room(32, 24, n_lon=128, n_lat=64).desc()
    s = A.make_settings(seed=4, max_depth=12, rr_depth=6)
    a, _ = ReferenceEngine(desc).render(s, 2)
    b, _ = PortEngine(desc).render(s, 2)
    close = np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), 1e-12)
    assert close.mean() > 0.99


@pytest.mark.parametrize("rho", [0.0, 0.8])
def test_port_white_furnace(rho):
    img, st = PortEngine(scenes.furnace_sphere(rho, 8, 8).desc()).render(A.make_settings(seed=1), 1024)
    assert abs(img[:, :, 1].mean() - 1 / (1 - rho)) < 0.01 / (1 - rho)
    assert st["leaks"] == 0 and st["inconsistencies"] == 0


def test_port_invisible_sphere():
    img, _ = PortEngine(scenes.invisible_sphere().desc()).render(A.make_settings(seed=1), 512)
    assert abs(img[:, :, 1].mean() - 1.0) < 0.006
