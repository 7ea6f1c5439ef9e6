"""Aim guides of Lambertian surfaces on a GPU (SurfaceOptics::sampleAim*, the diffuse mixture of
sampleScatter and evalScatter, src/owe/transport/scattering.cpp:111-137, 168-175): a scene's indirect
guide toward its lamp (Scene::build, src/owe/scene/scene.hpp:121-140) and a measurement screen's
guide toward its aim disk (Loader::sensor, src/owe/loader/loader_detectors.cpp:237-249), against the
reference engine."""
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


def _guided_lamp(width=48, height=36):
    """The lamp over the floor with the floor's scattering half guided toward the lamp sphere, as an
    `indirect_guide` naming the lamp sets it: the sphere's centre, a normal toward the origin, its
    radius times 1.001, share 0.5."""
    sb = scenes.lamp_over_floor(width, height)
    center = np.array([0.4, -0.2, 1.2])
    sb.aim_guide(sb.boundaries[0].optics, center, -center / np.linalg.norm(center), 0.25 * 1.001, 0.5)
    return sb


def test_guided_one_sample_paths_follow_the_reference():
    desc = _guided_lamp(64, 48).desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=3, max_depth=8, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    img_ref, _ = ref.render(s, 1, passes=1)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        img_gpu = c.resolve()[0]
    a, b = img_ref[:, :, 1].ravel(), img_gpu[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.97, f"only {close.mean():.3f} of paths agree"


def test_guided_floor_renders_like_the_reference_and_the_unguided_floor():
    """The guide changes the sampling, not the image: the guided render agrees with the reference's
    guided render and with the unguided one."""
    guided = _guided_lamp().desc()
    plain = scenes.lamp_over_floor(48, 36).desc()
    ref = ReferenceEngine(guided)
    runs_ref, runs_gpu, runs_plain = [], [], []
    with _ctx(guided) as c, _ctx(plain) as cp:
        for k in range(8):
            img, _, _ = ref.render_backend(A.make_settings(seed=70 + k), 64)
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=80 + k))
            c.reset_film()
            c.run_pass(64)
            runs_gpu.append(c.resolve()[0])
            cp.set_settings(A.make_settings(seed=90 + k))
            cp.reset_film()
            cp.run_pass(64)
            runs_plain.append(cp.resolve()[0])
        assert c.stats()["device_faults"] == 0
    save_artifact("guided_lamp", ref=np.array(runs_ref), gpu=np.array(runs_gpu), plain=np.array(runs_plain))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep
    ok, rep = block_z_test(runs_plain, runs_gpu)
    assert ok, rep


def test_guided_screen_renders_like_the_reference():
    """A diffuse screen whose sensor aims at a Lambertian disk: the loader gives the screen's own
    scattering the sensor's aim with share 0.95; the irradiance it records is the disk's."""
    sb = scenes.disk_irradiance(screen=True)
    b = len(sb.boundaries) - 1
    aim = ((0.0, 0.0, 0.5), (0.0, 0.0, 1.0), 0.3)
    sb.sensor(4, 4, b, 0.15, 0.15, aim=aim + (0.9,))
    sb.aim_guide(sb.boundaries[b].optics, aim[0], aim[1], aim[2], 0.95)
    desc = sb.desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(8):
            img, _, _ = ref.render_backend(A.make_settings(seed=110 + k), 4096)
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=120 + k))
            c.reset_film()
            c.run_pass(4096)
            runs_gpu.append(c.resolve()[0])
        assert c.stats()["device_faults"] == 0
    ok, rep = block_z_test(runs_ref, runs_gpu, block=1)
    assert ok, rep
    expected = scenes.disk_irradiance_mean(2.0, 0.3, 0.5, 0.15)
    y = np.mean([r[:, :, 1].mean() for r in runs_gpu])
    assert abs(y - expected) < 0.01 * expected, (y, expected)
