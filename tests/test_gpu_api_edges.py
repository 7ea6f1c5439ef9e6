"""The C ABI at its edges on a GPU: calls out of order, settings out of range, empty and degenerate
inputs (no samples, no rays, no boundaries, no emitters, a one-pixel film), rays that meet nothing,
and a context whose scene is replaced. Where the reference renders the case, the device's film is
checked against the reference engine's on the same sample streams."""
import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from oracle_ref import ReferenceEngine

pytestmark = pytest.mark.gpu


def _same_streams(desc, settings, spp):
    ref, _ = ReferenceEngine(desc).render(settings, 1, passes=spp)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(settings)
        c.run_pass(spp)
        img, n = c.resolve()
        st = c.stats()
    assert n.min() == spp and st["device_faults"] == 0 and st["leaks"] == 0
    return ref, img


def test_calls_before_a_scene_are_refused():
    with owe_cuda.Context() as c:
        with pytest.raises(RuntimeError, match="no scene"):
            c.run_pass(1)
        with pytest.raises(RuntimeError, match="no scene"):
            c.resolve()


def test_settings_out_of_range_are_refused_and_change_nothing():
    desc = scenes.lamp_over_floor(8, 6).desc()
    good = A.make_settings(seed=4)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(good)
        c.run_pass(4)
        before, _ = c.resolve()
        for bad in (A.make_settings(seed=4, max_depth=-1), A.make_settings(seed=4, max_depth=4097),
                    A.make_settings(seed=4, wavelength_mode=7), A.make_settings(seed=4, precision=9),
                    A.make_settings(seed=4, integrator=5)):
            with pytest.raises(RuntimeError):
                c.set_settings(bad)
        after, n = c.resolve()
        assert np.array_equal(before, after) and n.max() == 4
        c.set_settings(A.make_settings(seed=4, max_depth=4096))  # the deepest accepted


def test_no_samples_and_no_rays_are_no_ops():
    desc = scenes.lamp_over_floor(8, 6).desc()
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.run_pass(0)
        img, n = c.resolve()
        assert not img.any() and not n.any()
        b, p, t = c.cast_rays(np.zeros((0, 3)), np.zeros((0, 3)))
        assert len(b) == len(p) == len(t) == 0


def test_rays_that_meet_nothing():
    """Rays far above the scene pointing away from it: no boundary (0xFFFFFFFE, the reference's
    kNone), infinite distance."""
    desc = scenes.lamp_over_floor(8, 6).desc()
    rng = np.random.default_rng(3)
    o = rng.uniform(-1, 1, size=(1000, 3)) + np.array([0.0, 0.0, 50.0])
    d = np.tile([0.0, 0.0, 1.0], (1000, 1))
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        b, p, t = c.cast_rays(o, d)
    assert np.all(b == 0xFFFFFFFE) and np.all(np.isinf(t))


def test_one_pixel_film():
    desc = scenes.lamp_over_floor(1, 1).desc()
    ref, img = _same_streams(desc, A.make_settings(seed=8), 256)
    assert img.shape == (1, 1, 3) and np.isfinite(img).all()
    # the same 256 paths: equal but for a path whose FP32 decision turned the other way
    assert abs(img[0, 0, 1] - ref[0, 0, 1]) <= 2e-2 * abs(ref[0, 0, 1]) + 1e-12


def test_a_scene_without_boundaries_sees_its_sky():
    """No boundaries at all (the device builds no tree): every camera path escapes to the uniform
    sky, as the reference's do."""
    sb = scenes.SceneBuilder()
    sb.uniform_sky(0.7)
    sb.observer(8, 6, (0, 0, 0), (1, 0, 0), fov_y_deg=40.0)
    desc = sb.desc()
    for precision in (A.PRECISION_MIXED, A.PRECISION_FP64):
        ref, img = _same_streams(desc, A.make_settings(seed=1, precision=precision), 16)
        assert np.allclose(img, ref, rtol=1e-6, atol=1e-12)


def test_a_scene_without_emitters_is_black():
    sb = scenes.SceneBuilder()
    sb.sheet(2.0, 2.0, scenes.pose(), sb.diffuse(0.8))
    sb.observer(8, 6, (0.0, -2.0, 1.0), (0.0, 0.0, 0.0), fov_y_deg=40.0)
    ref, img = _same_streams(sb.desc(), A.make_settings(seed=2), 8)
    assert not img.any() and not ref.any()


def test_a_replaced_scene_renders_as_in_a_fresh_context():
    first = scenes.lamp_over_floor(16, 12).desc()
    second = scenes.glass_sphere_on_floor(24, 20).desc()
    s = A.make_settings(seed=6)
    with owe_cuda.Context() as c:
        c.set_settings(s)
        c.upload(first)
        c.build_bvh()
        c.run_pass(4)
        c.upload(second)
        c.build_bvh()
        c.reset_film()
        c.run_pass(4)
        replaced, n = c.resolve()
    with owe_cuda.Context() as c:
        c.set_settings(s)
        c.upload(second)
        c.build_bvh()
        c.run_pass(4)
        fresh, _ = c.resolve()
    assert replaced.shape == (20, 24, 3) and n.max() == 4
    assert np.array_equal(replaced, fresh)
