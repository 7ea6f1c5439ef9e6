"""Parity of the CUDA backend with the reference engine (GPU).

Ray casts: closest-hit boundary and primitive identities equal World::intersect's apart from rare
grazing ties, distances within the stated tolerance. Images: analytic known answers of the
reference's conformance suite (tests/test_backends.cpp) and statistical agreement with the
reference's own FP64 transport on the same scene (compareRenderers' block z-test), plus per-path
agreement where device and CPU paths draw the same random numbers.
"""
import math

import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from conftest import save_artifact
from oracle_ref import ReferenceEngine, block_z_test

pytestmark = pytest.mark.gpu

# Mixed precision: FP32 triangles and directions, FP64 origins; a triangle hit's distance is
# recomputed from the FP64 vertices, an analytic one refined in FP64. Every hit's distance agrees
# with World::intersect's to this relative tolerance.
T_REL_TOL = 1e-6


def _ctx(desc, settings=None):
    c = owe_cuda.Context()
    c.upload(desc)
    c.build_bvh()
    if settings is not None:
        c.set_settings(settings)
    return c


def test_cast_rays_match_world_intersect_on_displaced_sphere():
    sb = scenes.bvh_stress_room(64, 48, n_lon=256, n_lat=128)
    desc = sb.desc()
    ref = ReferenceEngine(desc)
    o, d = scenes.random_rays(200_000, 1234, (-2.8, -2.8, 0.1), (2.8, 2.8, 3.9), (-1.1, -1.1, 0.1), (1.1, 1.1, 2.3))
    rb, rp, rt = ref.cast_rays(o, d)
    with _ctx(desc) as c:
        info = c.bvh_info()
        assert info["triangles"] == 256 * 128 * 2
        gb, gp, gt = c.cast_rays(o, d)
    same = (gb == rb) & (gp == rp)
    frac = 1 - same.mean()
    # disagreements must be near-ties: the two distances agree although the primitives differ
    diff = ~same
    if diff.any():
        both = diff & (rb != A.KNONE) & (gb != A.KNONE)
        assert np.all(np.abs(gt[both] - rt[both]) <= 1e-4 * np.maximum(1, rt[both])), "a non-tie mismatch"
    assert frac < 1e-3, f"{frac:.2e} of rays hit another primitive"
    hit = same & (rb != A.KNONE)
    rel = np.abs(gt[hit] - rt[hit]) / np.maximum(rt[hit], 1e-9)
    # distances recomputed from the FP64 vertices once the FP32 traversal has found the triangle
    assert np.max(rel) <= T_REL_TOL, f"max relative t error {np.max(rel):.2e}"


def test_cast_rays_hit_analytic_shapes_like_the_reference():
    sb = scenes.glass_sphere_on_floor(32, 32)
    desc = sb.desc()
    ref = ReferenceEngine(desc)
    o, d = scenes.random_rays(50_000, 99, (-4, -6, 0.2), (4, -3, 4), (-1.2, -1.2, -0.5), (1.2, 1.2, 2.2))
    rb, rp, rt = ref.cast_rays(o, d)
    with _ctx(desc) as c:
        gb, gp, gt = c.cast_rays(o, d)
    assert np.mean(gb == rb) > 0.9999
    hit = (gb == rb) & (rb != A.KNONE)
    rel = np.abs(gt[hit] - rt[hit]) / rt[hit]
    # roots refined in FP64: what remains is the FP32 rounding of the ray's direction
    assert np.median(rel) < 1e-7 and np.quantile(rel, 0.999) < T_REL_TOL * 5, (np.median(rel), rel.max())


@pytest.mark.parametrize("rho", [0.0, 0.5, 0.8])
def test_white_furnace_closed_diffuse_sphere(rho):
    """L = Le / (1 - rho) inside a closed emitting diffuse sphere (tests/test_backends.cpp:349-378)."""
    desc = scenes.furnace_sphere(rho).desc()
    r = owe_cuda.CudaBackend().create_renderer(desc, A.make_settings(seed=1))
    r.run_pass(1024)
    img = r.resolve()
    assert abs(img[:, :, 1].mean() - 1 / (1 - rho)) < 0.01 / (1 - rho)
    st = r.stats()
    assert st["leaks"] == 0 and st["device_faults"] == 0, st
    r.close()


def test_lossless_dielectric_sphere_is_invisible():
    """tests/test_backends.cpp:380-407: n^2 law, Fresnel, TIR and dispersion keep L = 1."""
    desc = scenes.invisible_sphere().desc()
    r = owe_cuda.CudaBackend().create_renderer(desc, A.make_settings(seed=1))
    r.run_pass(1024)
    img = r.resolve()
    assert abs(img[:, :, 1].mean() - 1.0) < 0.004
    assert abs(img[6:18, 6:18, 1].mean() - 1.0) < 0.01
    r.close()


def _glass_settings(seed):
    return A.make_settings(seed=seed, max_depth=16, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)


@pytest.mark.parametrize("precision", [A.PRECISION_MIXED, A.PRECISION_FP64, A.PRECISION_FP32])
def test_glass_sphere_agrees_with_reference_statistically(precision):
    """The plain-method workload at 48 x 48: block z-test over independent seeds against the
    reference's FP64 transport (compareRenderers), for each precision instantiation."""
    desc = scenes.glass_sphere_on_floor(48, 48).desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(8):
            img, st = ref.render(_glass_settings(1000 + k), 64)
            runs_ref.append(img)
            s = _glass_settings(2000 + k)
            s.precision = precision
            c.set_settings(s)
            c.reset_film()
            c.run_pass(64)
            runs_gpu.append(c.resolve()[0])
            assert st["leaks"] == 0
        assert c.stats()["device_faults"] == 0
    save_artifact(f"glass_sphere_runs_{precision}", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


@pytest.mark.parametrize("precision,agree", [(A.PRECISION_MIXED, 0.97), (A.PRECISION_FP64, 0.995),
                                             (A.PRECISION_FP32, 0.9)])
def test_one_sample_paths_follow_the_reference_paths(precision, agree):
    """With one-sample passes both draw from the stream (hashCombine(seed, pixel), pass): most
    device paths make every decision the CPU path makes and return the same value. The all-FP64
    instantiation follows nearly every path; plain FP32 (origins rounded after every event, roots
    and distances in FP32) turns more decisions the other way."""
    desc = scenes.glass_sphere_on_floor(64, 64).desc()
    ref = ReferenceEngine(desc)
    s = _glass_settings(5)
    s.precision = precision
    img_ref, _ = ref.render(s, 1, passes=1)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        img_gpu = c.resolve()[0]
    save_artifact(f"one_sample_paths_{precision}", ref=img_ref, gpu=img_gpu)
    a, b = img_ref[:, :, 1].ravel(), img_gpu[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > agree, f"only {close.mean():.3f} of paths agree"


def test_hero_wavelength_render_agrees_with_reference_backend():
    """Four hero wavelengths (the reference's default) through its unchanged cpu Backend."""
    desc = scenes.glass_sphere_on_floor(32, 32).desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with _ctx(desc) as c:
        for k in range(6):
            s = A.make_settings(seed=300 + k, max_depth=16, rr_depth=4)
            img, st, _ = ref.render_backend(s, 64)
            runs_ref.append(img)
            c.set_settings(A.make_settings(seed=400 + k, max_depth=16, rr_depth=4))
            c.reset_film()
            c.run_pass(64)
            runs_gpu.append(c.resolve()[0])
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


def test_film_is_deterministic_and_passes_accumulate():
    desc = scenes.glass_sphere_on_floor(32, 32).desc()
    s = _glass_settings(11)
    with _ctx(desc, s) as c:
        c.run_pass(3)
        a, n = c.resolve()
        c.reset_film()
        c.run_pass(1)
        c.run_pass(2)
        b, n2 = c.resolve()
    assert np.array_equal(n, n2) and n.max() == 3
    assert np.array_equal(a, b), "a pass split into sub-passes must give the same film, bit for bit"


@pytest.mark.parametrize("integrator", [A.INTEGRATOR_PATH, A.INTEGRATOR_LIGHT])
def test_resolve_async_in_a_render_loop_matches_resolve(integrator):
    """owec_resolve_async after every pass of a loop, each image into its own page-locked buffer
    while the next passes run: every image equals the synchronous resolve of the same passes, bit
    for bit, and so do the sample counts."""
    import torch
    desc = scenes.lamp_over_floor(64, 48).desc()
    s = A.make_settings(seed=31, integrator=integrator)
    sync_imgs, sync_cnts = [], []
    with _ctx(desc, s) as c:
        for _ in range(5):
            c.run_pass(2)
            img, cnt = c.resolve()
            sync_imgs.append(img.copy())
            sync_cnts.append(cnt.copy())
    outs = [torch.empty((48, 64, 3), dtype=torch.float64, pin_memory=True).numpy() for _ in range(5)]
    cnts = [torch.empty((48, 64), dtype=torch.float64, pin_memory=True).numpy() for _ in range(5)]
    with _ctx(desc, s) as c:
        for k in range(5):
            c.run_pass(2)
            c.resolve_async(outs[k], cnts[k])
        c.resolve_wait()
    for k in range(5):
        assert np.array_equal(outs[k], sync_imgs[k]), k
        assert np.array_equal(cnts[k], sync_cnts[k]), k


def test_small_film_folds_many_samples_like_one_sample_passes():
    """A 16 x 16 film of 300 samples per pixel in one pass (the block-per-pixel fold) equals the same
    samples in ten passes of 30 (the thread-per-pixel fold), bit for bit."""
    desc = scenes.glass_sphere_on_floor(16, 16).desc()
    s = _glass_settings(12)
    with _ctx(desc, s) as c:
        c.run_pass(300)
        a, n = c.resolve()
        c.reset_film()
        for _ in range(10):
            c.run_pass(30)
        b, n2 = c.resolve()
    assert np.array_equal(n, n2) and n.max() == 300
    assert np.array_equal(a, b)


@pytest.mark.parametrize("integrator", ["path", "light"])
def test_switching_precision_in_one_context_matches_a_fresh_context(integrator):
    """The path state is sized per precision mode: an FP64 pass after a mixed one in the same
    context renders exactly what a fresh FP64 context renders (the FP64 records are larger)."""
    desc = scenes.lamp_over_floor(64, 48).desc()
    s64 = A.make_settings(seed=21, precision=A.PRECISION_FP64, integrator=integrator)
    with _ctx(desc) as c:
        c.set_settings(A.make_settings(seed=20, precision=A.PRECISION_MIXED, integrator=integrator))
        c.run_pass(700)  # 2M+ paths in flight, the most the mixed mode allocates
        c.set_settings(s64)
        c.run_pass(700)
        switched = c.resolve()[0]
        assert c.stats()["device_faults"] == 0
    with _ctx(desc, s64) as c:
        c.run_pass(700)
        fresh = c.resolve()[0]
    assert np.array_equal(switched, fresh)


@pytest.mark.parametrize("precision", [A.PRECISION_MIXED, A.PRECISION_FP64])
def test_reflected_moonlight_matches_the_analytic_answer(precision):
    """The reference's conformance check of a distant reflector (tests/test_backends.cpp:69-97): a
    floor lit only by a full-phase Lambertian moon 1e9 m away, within 1.5 % of (2/3) rho E_sun
    (R / d)^2 / pi, with no inconsistent regions and no leaks."""
    desc = scenes.reflected_moonlight().desc()
    s = A.make_settings(seed=1, precision=precision)
    with _ctx(desc, s) as c:
        c.run_pass(2048)
        img = c.resolve()[0]
        st = c.stats()
    expected = scenes.reflected_moonlight_expected()
    measured = float(img[:, :, 1].mean())
    assert abs(measured / expected - 1) < 0.015, (measured, expected, st)
    assert st["inconsistencies"] == 0 and st["leaks"] == 0 and st["device_faults"] == 0, st


@pytest.mark.parametrize("precision", [A.PRECISION_MIXED, A.PRECISION_FP64])
def test_planetary_ground_follows_the_reference(precision):
    """The reference's planetary-surface regression (benchmarks/regressions/planetary_ground.owe): the
    ground is a sphere of the Earth's radius, so a ray leaving it starts 6.4e6 m from the sphere's
    centre, where |o - c|^2 - R^2 cancels in FP64 and the reference switches to its double-double
    solve (intersectNearSphere). One-sample paths make the reference's decisions, 64-spp films on the
    same streams agree, and no path meets an inconsistent region."""
    desc = scenes.planetary_ground().desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=7, max_depth=8, precision=precision)
    one_ref, _ = ref.render(s, 1, passes=1)
    many_ref, st_ref = ref.render(s, 1, passes=64)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        one = c.resolve()[0]
        c.reset_film()
        c.run_pass(64)
        many = c.resolve()[0]
        st = c.stats()
    a, b = one_ref[..., 1], one[..., 1]
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.99, close.mean()
    assert abs(many[..., 1].mean() / many_ref[..., 1].mean() - 1) < 2e-3
    assert st["inconsistencies"] == 0 and st["leaks"] == 0 and st["device_faults"] == 0, st
    assert st_ref["inconsistencies"] == 0


@pytest.mark.parametrize("precision", [A.PRECISION_MIXED, A.PRECISION_FP64])
def test_a_screen_just_before_a_far_light_blocks_it(precision):
    """The reference's far next-event regression (benchmarks/regressions/far_nee_visibility.owe,
    tests/test_far_visibility.cpp): a screen 5 cm before a light 1e6 m away blocks all of its light,
    so the film is exactly black; moved aside or behind the light, the same paths see the light and
    give the same film, which the reference's on the same streams matches."""
    s = A.make_settings(seed=11, max_depth=2, precision=precision)
    films = {}
    for where in ("blocked", "side", "beyond"):
        with _ctx(scenes.far_nee_visibility(where).desc(), s) as c:
            c.run_pass(64)
            films[where] = c.resolve()[0]
            st = c.stats()
        assert st["inconsistencies"] == 0 and st["leaks"] == 0 and st["device_faults"] == 0, (where, st)
    assert not films["blocked"].any()
    assert films["side"][..., 1].mean() > 0
    assert np.array_equal(films["side"], films["beyond"])
    ref, _ = ReferenceEngine(scenes.far_nee_visibility("side").desc()).render(s, 1, passes=64)
    assert abs(films["side"][..., 1].mean() / ref[..., 1].mean() - 1) < 2e-3


@pytest.mark.parametrize("precision", [A.PRECISION_MIXED, A.PRECISION_FP64])
def test_lamp_in_a_full_feature_scene_follows_the_reference(precision):
    """The lamp over the floor with an absorbing sphere of 1e6 m far below the floor, out of every
    path's way but for those that leave the floor's edge: a sphere that size sends the scene to the
    Full instantiations. Their shadow queries stop at the shadow ray's end, short of the lamp: a
    window past it would find the lamp's own surface and darken the floor. One-sample paths make the
    reference's decisions and the 64-spp films agree."""
    sb = scenes.lamp_over_floor(24, 18)
    sb.sphere_body(1.0e6, (0.0, 0.0, -1.0e7), sb.medium_opaque(), sb.absorber())
    desc = sb.desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=5, max_depth=8, precision=precision)
    one_ref, _ = ref.render(s, 1, passes=1)
    many_ref, _ = ref.render(s, 1, passes=64)
    with _ctx(desc, s) as c:
        c.run_pass(1)
        one = c.resolve()[0]
        c.reset_film()
        c.run_pass(64)
        many = c.resolve()[0]
        st = c.stats()
    a, b = one_ref[..., 1], one[..., 1]
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.99, close.mean()
    assert abs(many[..., 1].mean() / many_ref[..., 1].mean() - 1) < 2e-3
    assert st["inconsistencies"] == 0 and st["leaks"] == 0 and st["device_faults"] == 0, st
