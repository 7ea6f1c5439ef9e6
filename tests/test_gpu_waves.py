"""Liquid wave surfaces on a GPU (WaveSurface, src/owe/scene/geometry.cpp:190-344): analytic sums of
plane waves and sums sampled as bicubic Hermite splines, against the reference engine's
World::intersect and path tracer, and the light integrator against the reference's known answer for
ripple caustics (tests/test_references.cpp:322-403)."""
import math

import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from conftest import save_artifact
from oracle_ref import ReferenceEngine, block_z_test

pytestmark = pytest.mark.gpu


def _ctx(desc, settings=None):
    c = owe_cuda.Context()
    c.upload(desc)
    c.build_bvh()
    if settings is not None:
        c.set_settings(settings)
    return c


@pytest.mark.parametrize("sampled", [False, True])
def test_wave_casts_match_world_intersect(sampled):
    """Rays from the air above the pool and from inside the water: the same boundaries as
    World::intersect, and the same distances."""
    desc = scenes.wave_pool(sampled=sampled).desc()
    above = scenes.random_rays(100_000, 31, (-0.2, -0.2, 0.01), (0.2, 0.2, 0.12), (-0.14, -0.14, -0.01), (0.14, 0.14, 0.0))
    below = scenes.random_rays(100_000, 32, (-0.13, -0.13, -0.07), (0.13, 0.13, -0.01), (-0.15, -0.15, -0.08), (0.15, 0.15, 0.02))
    o = np.concatenate([above[0], below[0]])
    d = np.concatenate([above[1], below[1]])
    rb, _, rt = ReferenceEngine(desc).cast_rays(o, d)
    with _ctx(desc) as c:
        gb, _, gt = c.cast_rays(o, d)
    surface = rb == 0
    assert surface.sum() > 100_000, surface.sum()
    diff = gb != rb
    assert np.mean(diff) < 2e-4, (np.mean(diff), np.bincount(rb[diff & (rb != A.KNONE)], minlength=desc.n_boundaries))
    hit = (gb == rb) & (rb != A.KNONE)
    rel = np.abs(gt[hit] - rt[hit]) / np.maximum(rt[hit], 1e-9)
    # the distances come back as FP32
    assert np.median(rel) < 1e-7 and np.quantile(rel, 0.999) < 1e-5, (np.median(rel), np.quantile(rel, 0.999))


def test_wave_one_sample_paths_follow_the_reference():
    """One-sample passes through the analytic pool: refraction at the waves' exact normals, the
    water's dispersion and absorption make the same paths as on the CPU."""
    desc = scenes.wave_pool(64, 48).desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=7, max_depth=12, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    img_ref, _ = ref.render(s, 1, passes=1)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        img_gpu = c.resolve()[0]
        st = c.stats()
    a, b = img_ref[:, :, 1].ravel(), img_gpu[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.97, f"only {close.mean():.3f} of paths agree"
    assert st["device_faults"] == 0 and st["leaks"] == 0, st


@pytest.mark.parametrize("sampled", [False, True])
def test_wave_pool_renders_like_the_reference(sampled):
    desc = scenes.wave_pool(sampled=sampled).desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    ref_incons = 0
    with _ctx(desc) as c:
        for k in range(8):
            img, rs, _ = ref.render_backend(A.make_settings(seed=40 + k, max_depth=16), 64)
            ref_incons += rs["inconsistencies"] + rs["leaks"]
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=50 + k, max_depth=16))
            c.reset_film()
            c.run_pass(64)
            runs_gpu.append(c.resolve()[0])
        st = c.stats()
    save_artifact(f"wave_pool_{'sampled' if sampled else 'analytic'}", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    assert st["device_faults"] == 0, st
    assert st["inconsistencies"] + st["leaks"] <= max(2 * ref_incons, 1e-4 * st["paths"]), (st, ref_incons)
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


def _refract(d, n, eta):
    """Snell refraction of unit rows d at unit normals n (flipped against d) with n1 / n2 = eta;
    NaN rows where the light is totally reflected."""
    s = np.where(np.sum(d * n, axis=1, keepdims=True) > 0, -1.0, 1.0)
    n = n * s
    ci = -np.sum(d * n, axis=1, keepdims=True)
    k = 1 - eta * eta * (1 - ci * ci)
    out = d * eta + n * (eta * ci - np.sqrt(np.where(k < 0, np.nan, k)))
    return out / np.linalg.norm(out, axis=1, keepdims=True)


def _fresnel(n1, n2, ci):
    """Unpolarised Fresnel reflectance from n1 into n2 at incidence cosine ci."""
    st2 = (n1 / n2) ** 2 * (1 - ci * ci)
    ct = np.sqrt(np.clip(1 - st2, 0, None))
    rs = (n1 * ci - n2 * ct) / (n1 * ci + n2 * ct)
    rp = (n2 * ci - n1 * ct) / (n2 * ci + n1 * ct)
    return np.where(st2 >= 1, 1.0, 0.5 * (rs * rs + rp * rp))


def _ripple_irradiance(a, lam_w, depth, gap, theta_s, n_samples=4_000_000, seed=99):
    """The irradiance profile on the sensor under a rippled water layer, from the surface-to-sensor
    ray map traced analytically and histogrammed into 160 bins over |u| < 0.02 (the reference's
    tests/test_references.cpp:346-381): entry points over a window holding every preimage, sun
    directions within its disc, wavelengths drawn with the CIE y-bar weight, Snell and Fresnel at the
    wave and the flat bottom, Beer-Lambert in the water."""
    k = 2 * math.pi / lam_w
    rng = np.random.default_rng(seed)
    lams = np.arange(360.0, 830.0 + 0.25, 0.5)
    cdf = np.cumsum(scenes._cie_y(lams))
    X, Y = 0.03, 0.012
    absorption = ([380, 400, 450, 500, 550, 600, 650, 700, 750, 800],
                  [0.0114, 0.00663, 0.0092, 0.0204, 0.0565, 0.2224, 0.34, 0.65, 2.47, 2.07])
    water = ((5.684027565e-1, 1.726177391e-1, 2.086189578e-2, 1.130748688e-1),
             (5.101829712e-3, 1.821153936e-2, 2.620722293e-2, 1.069792721e1))
    cone = 2 * math.pi * (1 - math.cos(theta_s))
    hist = np.zeros(160)
    chunk = 1_000_000
    for start in range(0, n_samples, chunk):
        m = min(chunk, n_samples - start)
        x = (2 * rng.random(m) - 1) * X
        y = (2 * rng.random(m) - 1) * Y
        li = np.minimum(np.searchsorted(cdf, rng.random(m) * cdf[-1], side="right"), len(lams) - 1)
        lam = lams[li]
        u1, u2 = rng.random(m), rng.random(m)
        cos_t = (1 - u1) + u1 * math.cos(theta_s)
        sin_t = np.sqrt(np.clip(1 - cos_t * cos_t, 0, None))
        phi = 2 * math.pi * u2
        d0 = np.stack([np.cos(phi) * sin_t, np.sin(phi) * sin_t, -cos_t], axis=1)
        n_rel = np.array([scenes.sellmeier_index(water, l, rel_air=False) / scenes.ciddor_air(l) for l in lams])[li]
        h = a * np.sin(k * x)
        normal = np.stack([-a * k * np.cos(k * x), np.zeros(m), np.ones(m)], axis=1)
        normal /= np.linalg.norm(normal, axis=1, keepdims=True)
        d1 = _refract(d0, normal, 1 / n_rel[:, None])
        d2 = _refract(d1, np.tile([0.0, 0.0, 1.0], (m, 1)), n_rel[:, None])
        ok = np.isfinite(d1).all(axis=1) & np.isfinite(d2).all(axis=1)
        c1 = np.abs(np.sum(d0 * normal, axis=1))
        c2 = np.abs(d1[:, 2])
        t1 = (-depth - h) / d1[:, 2]
        qx = x + d1[:, 0] * t1
        qy = y + d1[:, 1] * t1
        t2 = -gap / d2[:, 2]
        u = qx + d2[:, 0] * t2
        v = qy + d2[:, 1] * t2
        ok &= (np.abs(v) < 0.01) & (np.abs(u) < 0.02)
        w = (np.abs(d0[:, 2]) * cone * (2 * X) * (2 * Y) / n_samples * (1 - _fresnel(1.0, n_rel, c1)) *
             (1 - _fresnel(n_rel, 1.0, c2)) * np.exp(-np.interp(lam, *absorption) * t1))
        bins = ((u[ok] + 0.02) / 0.04 * 160).astype(int)
        np.add.at(hist, np.minimum(bins, 159), w[ok])
    return hist / ((0.04 / 160) * 0.02)


def test_ripple_caustics_follow_the_ray_map_jacobian():
    """The light integrator's particles through a rippled water surface land on the sensor as the
    analytic ray map's pushforward does: the same mean irradiance (1 %), the same profile (L1 within
    6 %), the fold caustic at the same bin (or its twin a wave away), concentrating the sunlight more
    than threefold -- the reference's own acceptance test for light-capable backends."""
    a, lam_w, depth, gap = 0.0005, 0.02, 0.08, 0.001
    sb = scenes.ripple_caustics(a, lam_w, depth, gap)
    desc = sb.desc()
    with _ctx(desc, A.make_settings(seed=11, integrator="light")) as c:
        c.run_pass(60000)
        img = c.resolve()[0]
        st = c.stats()
    assert st["device_faults"] == 0, st
    rendered = img[:, :, 1].mean(axis=0)
    theta_s = sb.env.sun_angular_radius
    analytic = _ripple_irradiance(a, lam_w, depth, gap, theta_s)
    save_artifact("ripple_caustics", rendered=rendered, analytic=analytic)
    e0 = math.pi * math.sin(theta_s) ** 2
    sum_a, sum_r = analytic.sum(), rendered.sum()
    l1 = np.abs(analytic - rendered).sum()
    arg_a, arg_r = int(np.argmax(analytic)), int(np.argmax(rendered))
    rep = (sum_r / sum_a, l1 / sum_a, arg_a, arg_r, analytic.max() / e0, rendered.max() / e0)
    assert abs(sum_r / sum_a - 1) < 0.01, rep
    assert l1 / sum_a < 0.06, rep
    assert abs(arg_a - arg_r) <= 1 or abs(abs(arg_a - arg_r) - 80) <= 1, rep
    assert analytic.max() > 3 * e0, rep
