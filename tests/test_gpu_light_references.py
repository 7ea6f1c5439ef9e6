"""The reference's known answers for light-capable backends (tests/test_references.cpp:77-210), run
with the light integrator: sunlight through a water layer, into a concave mirror's focus, and through
a biconvex N-BK7 lens, each against its closed form within 1 %. (The ripple-caustic answer of the
same file is in test_gpu_waves.py.)"""
import math

import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes

pytestmark = pytest.mark.gpu

LAMBDA_D = 587.5618
WATER = ((5.684027565e-1, 1.726177391e-1, 2.086189578e-2, 1.130748688e-1),
         (5.101829712e-3, 1.821153936e-2, 2.620722293e-2, 1.069792721e1))
WATER_ABSORPTION = ([380, 400, 450, 500, 550, 600, 650, 700, 750, 800],
                    [0.0114, 0.00663, 0.0092, 0.0204, 0.0565, 0.2224, 0.34, 0.65, 2.47, 2.07])


def _y_weighted(f):
    """The mean of f(lambda) weighted by the CIE y-bar over 360-830 nm in 0.5 nm steps: what a
    detector's Y channel reports for a spectral factor f (yWeighted, test_references.cpp:38-47)."""
    lams = np.arange(360.0, 830.0 + 0.25, 0.5)
    w = scenes._cie_y(lams)
    return float(np.sum(np.array([f(l) for l in lams]) * w) / np.sum(w))


def _fresnel(n1, n2, ci):
    st2 = (n1 / n2) ** 2 * (1 - ci * ci)
    if st2 >= 1:
        return 1.0
    ct = math.sqrt(1 - st2)
    rs = (n1 * ci - n2 * ct) / (n1 * ci + n2 * ct)
    rp = (n2 * ci - n1 * ct) / (n2 * ci + n1 * ct)
    return 0.5 * (rs * rs + rp * rp)


def _render_light(sb, particles_per_pixel, seed=5):
    with owe_cuda.Context() as c:
        c.upload(sb.desc())
        c.build_bvh()
        c.set_settings(A.make_settings(seed=seed, integrator="light"))
        c.run_pass(particles_per_pixel)
        img = c.resolve()[0]
        st = c.stats()
    assert st["device_faults"] == 0, st
    return img


def _sun_irradiance(sb):
    return math.pi * math.sin(sb.env.sun_angular_radius) ** 2


def _sensor(sb, width, height, half_x, half_y, xf):
    b = sb.sheet(half_x, half_y, xf, sb.optics_(A.SURF_DETECTOR))
    sb.sensor(width, height, b, half_x, half_y)


def test_water_layer_transmits_the_fresnel_share():
    """Sun at 40 degrees elevation over a 10 cm layer of water; a sensor under it receives
    E = E_sun cos(ti) T(ti) T(tt) exp(-sigma_a d / cos(tt))."""
    sb = scenes.SceneBuilder()
    el = math.radians(40)
    sb.sun((math.cos(el), 0.0, math.sin(el)), 1.0)
    v, t = scenes.box_mesh((-0.6, -0.6, 0.25), (0.6, 0.6, 0.35))
    sb.mesh_body(v, t, sb.medium_water(), sb.dielectric())
    _sensor(sb, 16, 16, 0.1, 0.1, scenes.pose())
    img = _render_light(sb, 64000)
    ci = math.cos(math.radians(50))

    def share(l):
        n = scenes.sellmeier_index(WATER, l, rel_air=False) / scenes.ciddor_air(l)
        ct = math.sqrt(1 - (1 - ci * ci) / (n * n))
        return ci * (1 - _fresnel(1, n, ci)) * (1 - _fresnel(n, 1, ct)) * math.exp(-np.interp(l, *WATER_ABSORPTION) * 0.1 / ct)

    expected = _sun_irradiance(sb) * _y_weighted(share)
    e = img[:, :, 1].mean()
    assert abs(e / expected - 1) < 0.01, (e, expected)


def test_concave_mirror_concentrates_sunlight():
    """A spherical mirror (R = 0.4 m, 0.1 m aperture, reflectance 0.9) under an overhead sun and a
    1 cm sensor at its focus facing it, which shades 1 cm^2 of the mirror:
    P = E_sun (pi 0.05^2 - 0.01^2) 0.9."""
    sb = scenes.SceneBuilder()
    sb.sun((0.0, 0.0, 1.0), 1.0)
    coating = sb.optics_(A.SURF_MIRROR, sb.spectrum_constant(0.9), back_absorbs=True)
    sb.boundary(A.SHAPE_SAG, [1 / 0.4, 0.0, 0.05, 0.0], scenes.pose(), 0, 0, coating)
    _sensor(sb, 20, 20, 0.005, 0.005, scenes.pose(scenes.align_z((0, 0, -1)), (0.0, 0.0, 0.199)))
    img = _render_light(sb, 8000)
    power = img[:, :, 1].sum() * (0.01 / 20) ** 2
    e0 = _sun_irradiance(sb)
    expected = e0 * (math.pi * 0.05 ** 2 - 0.01 ** 2) * 0.9
    assert abs(power / expected - 1) < 0.01, (power, expected)
    assert img[:, :, 1].max() > 100 * e0  # the sun's image, concentrated


def test_lens_focuses_sunlight_with_its_fresnel_losses():
    """Overhead sun, an f = 100 mm biconvex N-BK7 lens of 40 mm clear aperture (radii from the lens
    maker's equation with its 8 mm thickness, designSimpleLens) with a black rim, and a sensor near its
    focus: every watt through the aperture arrives except what the two surfaces reflect."""
    f, t = 0.1, 0.008
    n_d = scenes.sellmeier_index(scenes.NBK7, LAMBDA_D, rel_air=False)
    R = (n_d - 1) * f * (1 + math.sqrt(1 - t / (n_d * f)))
    sb = scenes.SceneBuilder()
    sb.sun((0.0, 0.0, 1.0), 1.0)
    bk7 = sb.medium_sellmeier(*scenes.NBK7, rel_air=True)
    scenes.lens_body(sb, [(R, 0.02), (-R, 0.02)], [bk7], [t], z0=0.1, rim="black")
    _sensor(sb, 48, 48, 0.012, 0.012, scenes.translate(0.0, 0.0, -0.0015))
    img = _render_light(sb, 400 * 16)

    def transmitted(l):
        n = scenes.sellmeier_index(scenes.NBK7, l, rel_air=False)
        a, b = 2 * (n_d - 1), -(n_d - 1) ** 2 * t / n_d
        Rl = (a * f + math.sqrt((a * f) ** 2 + 4 * b * f)) / 2
        s = w = 0.0
        for i in range(400):
            h = 0.02 * (i + 0.5) / 400
            c1 = math.sqrt(1 - (h / Rl) ** 2)
            th1 = math.asin(math.sqrt(1 - c1 * c1))
            th2 = math.asin(math.sqrt(1 - c1 * c1) / n)
            tilt = th1 - th2
            h2 = h - t * math.tan(tilt)
            c3 = math.cos(math.asin(h2 / Rl) + tilt)
            s += h * (1 - _fresnel(1, n, c1)) * (1 - _fresnel(n, 1, c3))
            w += h
        return s / w

    e0 = _sun_irradiance(sb)
    expected = e0 * math.pi * 0.02 ** 2 * _y_weighted(transmitted)
    power = img[:, :, 1].sum() * (0.024 / 48) ** 2
    assert abs(power / expected - 1) < 0.01, (power, expected)
    assert img[:, :, 1].max() > 150 * e0, img[:, :, 1].max() / e0
