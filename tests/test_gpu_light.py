"""The light integrator (particle tracing) on a GPU.

The reference's CPU backend has no light integrator: its conformance suite checks one on a backend
against analytic answers (the white furnace, a disk's irradiance on a sensor and on a diffuse
screen) and against the reference's own path tracer on the same scene (compareRenderers' block
z-test through a pinhole). These tests do the same: the oracle is the analytic answer, or the
reference engine's path-traced image (oracle/_ref).
"""
import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from conftest import save_artifact
from oracle_ref import ReferenceEngine, block_z_test

pytestmark = pytest.mark.gpu


def _light(seed=1, **kw):
    return A.make_settings(seed=seed, integrator="light", **kw)


@pytest.mark.parametrize("rho", [0.0, 0.5])
def test_light_white_furnace(rho):
    """Inside a closed emitting diffuse sphere L = Le / (1 - rho): particles reach the eye through
    the emitter's own connections and those of every diffuse vertex (tests/test_backends.cpp:540-574)."""
    desc = scenes.furnace_sphere(rho, 8, 8).desc()
    r = owe_cuda.CudaBackend().create_renderer(desc, _light())
    assert r.integrator == "light" and "particles" in r.backend()
    r.run_pass(4096)
    y = r.resolve()[:, :, 1].mean()
    st = r.stats()
    r.close()
    assert abs(y - 1 / (1 - rho)) < 0.02 / (1 - rho), y
    assert st["paths"] == 8 * 8 * 4096 and st["shadow_rays"] > 0
    assert st["leaks"] == 0 and st["device_faults"] == 0, st


@pytest.mark.parametrize("screen,tol", [(False, 0.01), (True, 0.02)])
def test_light_measures_disk_irradiance_on_a_sensor(screen, tol):
    """A Lambertian disk over a sensor: the particles reaching the sensor's front face, divided by
    the pixel area, give the analytic irradiance; a diffuse screen records the same before it
    scatters (tests/test_backends.cpp:521-538)."""
    expected = scenes.disk_irradiance_mean(2.0, 0.3, 0.5, 0.15)
    desc = scenes.disk_irradiance(screen=screen).desc()
    r = owe_cuda.CudaBackend().create_renderer(desc, _light(seed=3))
    r.run_pass(400000)
    y = r.resolve()[:, :, 1].mean()
    st = r.stats()
    r.close()
    assert abs(y - expected) < tol * expected, (y, expected)
    assert st["device_faults"] == 0, st
    # the path integrator on the same sensor agrees with the same answer
    p = owe_cuda.CudaBackend().create_renderer(desc, A.make_settings(seed=4), "path")
    p.run_pass(40000)
    yp = p.resolve()[:, :, 1].mean()
    p.close()
    assert abs(yp - expected) < 0.01 * expected, (yp, expected)


def test_light_tracing_agrees_with_reference_path_tracing():
    """A lamp over a floor through a pinhole: the particle image against the reference engine's own
    path tracer (its unchanged cpu backend), block z-test over independent seeds
    (tests/test_backends.cpp:597-614, compareRenderers)."""
    desc = scenes.lamp_over_floor().desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        for k in range(10):
            img, st, _ = ref.render_backend(A.make_settings(seed=100 + k), 256)
            assert st["leaks"] == 0
            runs_ref.append(img)
            c.set_settings(_light(seed=200 + k))
            c.reset_film()
            c.run_pass(1024)
            runs_gpu.append(c.resolve()[0])
        assert c.stats()["device_faults"] == 0
    save_artifact("light_vs_path_lamp_floor", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep
    assert np.array(runs_gpu)[:, :, :, 1].mean() > 0


def test_light_film_is_bitwise_reproducible():
    """Splats are exact fixed-point sums: the same pass gives the same film bit for bit whatever
    order the threads added in, and the film resolves to the splats over the particles."""
    desc = scenes.lamp_over_floor(32, 24).desc()
    s = _light(seed=9)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(s)
        c.run_pass(64)
        a, n = c.resolve()
        sums, samples = c.read_film()
        c.reset_film()
        c.run_pass(64)
        b, _ = c.resolve()
    assert np.array_equal(a, b)
    assert np.all(n == 64) and np.all(samples == 64)
    assert np.allclose(sums / samples[:, :, None], a, rtol=1e-14, atol=0)


def test_light_fp64_instantiation_agrees_with_mixed():
    """The all-FP64 instantiation of the particle kernel renders the same image within the noise."""
    desc = scenes.lamp_over_floor().desc()
    runs = {A.PRECISION_MIXED: [], A.PRECISION_FP64: []}
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        for mode in runs:
            for k in range(6):
                c.set_settings(_light(seed=50 + k + 10 * mode, precision=mode))
                c.reset_film()
                c.run_pass(512)
                runs[mode].append(c.resolve()[0])
    ok, rep = block_z_test(runs[A.PRECISION_FP64], runs[A.PRECISION_MIXED])
    assert ok, rep
