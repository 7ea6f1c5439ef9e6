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


@pytest.mark.parametrize("mode", [A.WALK_PRIMARY_TRANSMISSION, A.WALK_STOCHASTIC])
def test_port_walks_equal_reference_walks(mode):
    """Tracer::walk restated: the achromat imaging a point source, every walk the reference's."""
    sb, info = scenes.achromat_scene(film=32, half_size=2.5e-4)
    desc = sb.desc()
    w = scenes.achromat_walk(info, seed=5, mode=mode)
    a, sa = ReferenceEngine(desc).walk(w, 0, 50_000)
    b, sb_ = PortEngine(desc).walk(w, 0, 50_000)
    assert sa == sb_
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12 * a.max())


def test_port_slab_walks_equal_reference_walks():
    h = 1e-4 * np.sin(np.linspace(0, 5, 24))[None, :] * np.cos(np.linspace(0, 4, 24))[:, None]
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = 0
    sb, info = scenes.caustic_slab_scene(n=24, heights=h, wall_bins=32)
    desc = sb.desc()
    w = scenes.caustic_walk(info, seed=2)
    a, sa = ReferenceEngine(desc).walk(w, 0, 40_000)
    b, sb_ = PortEngine(desc).walk(w, 0, 40_000)
    assert sa == sb_
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12 * a.max())


def test_port_rough_glass_and_metal_equal_reference():
    """GGX dielectric and conductor lobes (optics.hpp:104-246) on camera paths."""
    sb = scenes.SceneBuilder()
    sb.uniform_sky(1.0)
    bk7 = sb.medium_sellmeier(*scenes.NBK7, rel_air=True)
    sb.sphere_body(0.5, (-0.6, 0, 0.5), bk7, sb.dielectric(0.3))
    gold_n = sb.spectrum_tabulated([400, 500, 600, 700], [1.47, 0.97, 0.25, 0.16])
    gold_k = sb.spectrum_tabulated([400, 500, 600, 700], [1.95, 1.87, 3.0, 3.95])
    metal = sb.optics_(A.SURF_CONDUCTOR, roughness=0.2, cond_n=gold_n, cond_k=gold_k)
    opaque = sb.medium_opaque()
    sb.sphere_body(0.5, (0.6, 0, 0.5), opaque, metal)
    sb.sheet(5, 5, scenes.pose(), sb.diffuse(0.5))
    sb.observer(24, 16, (0, -3, 1.2), (0, 0, 0.4), fov_y_deg=40)
    desc = sb.desc()
    s = A.make_settings(seed=3, max_depth=8, rr_depth=4)
    a, _ = ReferenceEngine(desc).render(s, 2)
    b, _ = PortEngine(desc).render(s, 2)
    close = np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), 1e-12)
    assert close.mean() > 0.99


def test_port_fog_room_equals_reference():
    """Participating medium (free flight, HG scattering, medium NEE) with a PMMA heightfield panel:
    every one-sample path of the restatement is the reference's."""
    desc = scenes.fog_room(32, 24).desc()
    s = A.make_settings(seed=2, max_depth=24, rr_depth=6)
    a, sa = ReferenceEngine(desc).render(s, 1, passes=4)
    b, sb_ = PortEngine(desc).render(s, 1, passes=4)
    assert sa == sb_
    close = np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), 1e-12)
    assert close.mean() > 0.999
