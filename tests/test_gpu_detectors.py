"""Thin-lens observers (with and without a pupil guide) and aimed, flipped surface sensors on a GPU,
against the reference engine's own detectors (IdealObserver::generate, SurfaceSensor::generate,
src/owe/scene/detector.cpp:61-148)."""
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


def _thin_lens_scene(width=48, height=36, guide=None):
    """The lamp-over-floor scene seen through a 60 mm pupil focused at 2.6 m
    (tests/test_backends.cpp:597-614's second observer)."""
    sb = scenes.lamp_over_floor(width, height)
    sb.observer(width, height, (0.0, -2.2, 1.4), (0.0, 0.0, 0.0), fov_y_deg=40.0, pupil=0.03, focus=2.6, guide=guide)
    return sb


def _runs(desc, ref, settings_ref, settings_gpu, spp, n):
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(n):
            img, st, _ = ref.render_backend(settings_ref(k), spp)
            runs_ref.append(img)
            c.set_settings(settings_gpu(k))
            c.reset_film()
            c.run_pass(spp)
            runs_gpu.append(c.resolve()[0])
        assert c.stats()["device_faults"] == 0
    return runs_ref, runs_gpu


@pytest.mark.parametrize("guide", [None, ((0.0, -2.1, 1.33), 0.01, 0.9)])
def test_thin_lens_one_sample_paths_follow_the_reference(guide):
    """With one-sample passes the device draws the pupil point from the same stream as the CPU:
    the thin lens (and the guided pupil mixture) makes the same rays."""
    desc = _thin_lens_scene(64, 48, guide).desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=5, max_depth=8, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    img_ref, _ = ref.render(s, 1, passes=1)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        img_gpu = c.resolve()[0]
    a, b = img_ref[:, :, 1].ravel(), img_gpu[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.97, f"only {close.mean():.3f} of paths agree"


@pytest.mark.parametrize("integrator", ["path", "light"])
def test_thin_lens_renders_like_the_reference(integrator):
    """A thin lens focused at 2.6 m: the path and the light integrator against the reference's path
    tracer (tests/test_backends.cpp:597-614 checks light tracing through a lens pupil the same way)."""
    desc = _thin_lens_scene().desc()
    ref = ReferenceEngine(desc)
    spp = 256 if integrator == "path" else 1024
    # sixteen runs: a particle image's pixels are heavy-tailed (rare connections with large
    # weights), and few runs give their z-scores Student-t tails
    runs_ref, runs_gpu = _runs(desc, ref, lambda k: A.make_settings(seed=800 + k),
                               lambda k: A.make_settings(seed=900 + k, integrator=integrator), spp, 16)
    save_artifact(f"thin_lens_{integrator}", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


def _aimed_sensor_scene(flip=(False, False), screen=False):
    """A Lambertian disk over a 4 x 4-pixel sensor whose directions are aimed at the disk (with a
    smaller focus disk and, on a screen, a cosine share kept), read out flipped."""
    sb = scenes.disk_irradiance(screen=screen)
    b = len(sb.boundaries) - 1
    sb.sensor(4, 4, b, 0.15, 0.15, flip=flip, aim=((0, 0, 0.5), (0, 0, 1), 0.3, 0.9 if screen else 1.0),
              focus=((0.05, 0, 0.5), 0.1, 0.3))
    return sb


@pytest.mark.parametrize("screen", [False, True])
def test_aimed_sensor_renders_like_the_reference(screen):
    desc = _aimed_sensor_scene(screen=screen).desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = _runs(desc, ref, lambda k: A.make_settings(seed=100 + k),
                               lambda k: A.make_settings(seed=200 + k), 4096, 8)
    ok, rep = block_z_test(runs_ref, runs_gpu, block=1)
    assert ok, rep
    expected = scenes.disk_irradiance_mean(2.0, 0.3, 0.5, 0.15)
    y = np.mean([r[:, :, 1].mean() for r in runs_gpu])
    assert abs(y - expected) < 0.01 * expected, (y, expected)


def test_flipped_sensor_mirrors_the_readout():
    """flipX / flipY relabel pixels only: the flipped image is the plain one mirrored, for both
    integrators (one-sample streams of the path integrator differ per pixel, so compare the light
    integrator's film, whose particles do not depend on the labels)."""
    plain = _aimed_sensor_scene().desc()
    flipped = _aimed_sensor_scene(flip=(True, True)).desc()
    imgs = []
    for desc in (plain, flipped):
        with _ctx(desc, A.make_settings(seed=3, integrator="light")) as c:
            c.run_pass(20000)
            imgs.append(c.resolve()[0])
    assert np.array_equal(imgs[1], imgs[0][::-1, ::-1])
