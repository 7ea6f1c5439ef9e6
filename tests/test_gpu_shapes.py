"""The trimmed and lathe shapes and the even aspheres on a GPU, against the reference engine.

Cones, torus patches, round walls with openings, domes with a slit, disks with a hole and
numerically crossed aspheric sags: their closest hits against World::intersect on seeded rays, and
rendered images against the reference's own path tracer (compareRenderers' block z-test).
"""
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


def _compare_casts(desc, o, d, min_per_boundary=50):
    rb, rp, rt = ReferenceEngine(desc).cast_rays(o, d)
    with _ctx(desc) as c:
        gb, gp, gt = c.cast_rays(o, d)
    same = gb == rb
    # every boundary is hit often enough for the comparison to mean something
    counts = np.bincount(rb[rb != A.KNONE], minlength=desc.n_boundaries)
    assert counts.min() >= min_per_boundary, counts
    diff = ~same
    both = diff & (rb != A.KNONE) & (gb != A.KNONE)
    # a disagreement is a near-tie (two boundaries at one distance) or a trim edge met within rounding
    assert np.mean(diff) < 2e-4, (np.mean(diff), np.bincount(rb[diff & (rb != A.KNONE)], minlength=desc.n_boundaries))
    hit = same & (rb != A.KNONE)
    rel = np.abs(gt[hit] - rt[hit]) / np.maximum(rt[hit], 1e-9)
    return rel, counts


def test_shape_gallery_casts_match_world_intersect():
    """Closest hits on the cone, torus patch, round wall, dome, holed disk and asphere: the same
    boundaries as World::intersect, distances refined or bisected in FP64."""
    desc = scenes.shape_gallery().desc()
    o, d = scenes.random_rays(200_000, 77, (-2.5, -2.5, 0.05), (2.5, 2.5, 2.5), (-1.5, -1.5, 0.0), (1.5, 1.5, 1.2))
    rel, counts = _compare_casts(desc, o, d)
    assert np.median(rel) < 1e-7 and np.quantile(rel, 0.999) < 1e-5, (np.median(rel), np.quantile(rel, 0.999))


def test_asphere_lens_casts_match_world_intersect():
    desc = scenes.asphere_lens().desc()
    o, d = scenes.random_rays(200_000, 78, (-0.6, -0.6, 1.3), (0.6, 0.6, 2.0), (-0.35, -0.35, 0.8), (0.35, 0.35, 1.0))
    rel, counts = _compare_casts(desc, o, d, min_per_boundary=0)
    assert counts[0] > 10000 and counts[2] > 100
    assert np.median(rel) < 1e-7 and np.quantile(rel, 0.999) < 1e-5, (np.median(rel), np.quantile(rel, 0.999))


@pytest.mark.parametrize("name", ["shape_gallery", "asphere_lens"])
def test_shapes_render_like_the_reference(name):
    """Images of the gallery (sun and sky on Lambertian shapes) and of the aspheric lens (refraction
    through two numerically crossed faces) agree with the reference's path tracer."""
    desc = getattr(scenes, name)().desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(8):
            img, st, _ = ref.render_backend(A.make_settings(seed=600 + k, max_depth=16, rr_depth=5), 48)
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=700 + k, max_depth=16, rr_depth=5))
            c.reset_film()
            c.run_pass(48)
            runs_gpu.append(c.resolve()[0])
        st = c.stats()
    save_artifact(f"shapes_{name}_runs", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    assert st["device_faults"] == 0 and st["leaks"] == 0, st
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


def test_textures_follow_the_reference_paths():
    """Procedural albedos (checker, noise, rings, terrain, bands, radial, marble): with one-sample
    passes the device paths read the CPU paths' albedos at the same points (the same lattice hash
    and FP64 noise) and make the same decisions."""
    desc = scenes.texture_gallery().desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=9, max_depth=8, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    img_ref, _ = ref.render(s, 1, passes=1)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        img_gpu = c.resolve()[0]
    a, b = img_ref[:, :, 1].ravel(), img_gpu[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.97, f"only {close.mean():.3f} of paths agree"


@pytest.mark.parametrize("integrator", ["path", "light"])
def test_textures_render_like_the_reference(integrator):
    desc = scenes.texture_gallery(48, 30).desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(12):
            img, _, _ = ref.render_backend(A.make_settings(seed=300 + k), 64)
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=400 + k, integrator=integrator))
            c.reset_film()
            c.run_pass(64 if integrator == "path" else 512)
            runs_gpu.append(c.resolve()[0])
        assert c.stats()["device_faults"] == 0
    save_artifact(f"textures_{integrator}", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


def test_gradient_sky_follows_the_reference_paths():
    """Environment::sky's gradient (ground, horizon, zenith about a tilted up axis): one-sample
    device paths return the CPU paths' values, and the image agrees statistically."""
    desc = scenes.gradient_sky_scene().desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=4, max_depth=12, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    img_ref, _ = ref.render(s, 1, passes=1)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        img_gpu = c.resolve()[0]
    a, b = img_ref[:, :, 1].ravel(), img_gpu[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.97, f"only {close.mean():.3f} of paths agree"
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(8):
            img, _, _ = ref.render_backend(A.make_settings(seed=50 + k), 64)
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=60 + k))
            c.reset_film()
            c.run_pass(64)
            runs_gpu.append(c.resolve()[0])
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep
