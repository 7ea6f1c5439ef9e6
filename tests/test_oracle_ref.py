"""The oracle itself (CPU): the reference engine built from its own sources drives the same scene
descriptions the CUDA backend takes, and reproduces the reference's own known answers. These pin
the harness before it checks the GPU."""
import math

import numpy as np
import pytest

import owec_abi as A
import scenes
from oracle_ref import ReferenceEngine


def test_driver_pass_equals_the_reference_cpu_backend_bit_for_bit():
    """ref_driver.cpp's pass loop (hero-4 wavelengths) is CpuRenderer::pass: identical films."""
    desc = scenes.glass_sphere_on_floor(24, 24).desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=3, max_depth=16, rr_depth=4)
    a, sa = ref.render(s, 8, passes=2)
    b, sb, _ = ref.render_backend(s, 8, passes=2)
    assert np.array_equal(a, b)
    assert sa["paths"] == sb["paths"] == 24 * 24 * 16


@pytest.mark.parametrize("rho", [0.0, 0.5])
def test_reference_white_furnace(rho):
    desc = scenes.furnace_sphere(rho, 8, 8).desc()
    img, st = ReferenceEngine(desc).render(A.make_settings(seed=1), 1024)
    assert abs(img[:, :, 1].mean() - 1 / (1 - rho)) < 0.01 / (1 - rho)
    assert st["leaks"] == 0 and st["inconsistencies"] == 0


def test_reference_glass_catalog_index():
    """N-BK7's n_d = 1.5168 (Schott), as the reference's catalog test pins (tests/test_optics.cpp:94)."""
    sb = scenes.glass_sphere_on_floor(8, 8)
    ref = ReferenceEngine(sb.desc())
    n_glass = ref.index(1, 587.5618)
    n_air = ref.index(0, 587.5618)
    assert abs(n_glass / n_air - 1.5168) < 2e-4


def test_reference_ray_cast_on_the_displaced_sphere():
    sb = scenes.bvh_stress_room(8, 8, n_lon=64, n_lat=32)
    ref = ReferenceEngine(sb.desc())
    o = np.array([[0.0, -2.5, 1.2], [0.0, 0.0, 3.5]])
    d = np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    b, p, t = ref.cast_rays(o, d)
    assert b[0] == 0 and 1.2 < t[0] < 1.6  # the sphere (boundary 0), radius 1 +- 5 %, at y = 0
    assert b[1] == 7 and abs(t[1] - 0.48) < 1e-12  # the lamp sheet just under the ceiling, z = 3.98


def test_single_wavelength_mode_is_the_uniform_estimator():
    """One wavelength uniform in [380, 780]: a white Lambertian furnace still gives L = 1/(1 - rho)
    in Y (the estimator integrates cmf over 380-780 only, so Y is (int_380^780 ybar) / int ybar)."""
    desc = scenes.furnace_sphere(0.5, 8, 8).desc()
    s = A.make_settings(seed=2, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    img, _ = ReferenceEngine(desc).render(s, 2048)
    lam = np.linspace(380, 780, 40001)

    def lobe(x, mu, s1, s2):
        t = (x - mu) / np.where(x < mu, s1, s2)
        return np.exp(-0.5 * t * t)

    ybar = lambda l: 0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1)  # noqa: E731
    full = np.linspace(360, 830, 40001)
    frac = np.trapezoid(ybar(lam), lam) / np.trapezoid(ybar(full), full)
    assert abs(img[:, :, 1].mean() - 2 * frac) < 0.03
