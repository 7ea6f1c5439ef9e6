"""Parity at the configurations' own sizes (GPU).

C2's ray-cast oracle: 10^7 seeded rays through the 2^20-triangle room, hit boundary and triangle
against World::intersect, distances against its FP64 ones. The images at the configurations' film
sizes and sample counts: the reference engine renders a pixel range (a band of rows; all of C1's
256 x 256), the device the whole film, and the two are compared where both rendered: on the same
sample streams (one-sample paths make the same decisions; the film of many samples has a mean
relative error below 1 %, at 4096 samples per pixel for C1) and over independent seeds
(compareRenderers' block z-test)."""
import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from conftest import save_artifact
from oracle_ref import ReferenceEngine

pytestmark = pytest.mark.gpu


def test_c2_ten_million_rays_match_world_intersect():
    sb = scenes.bvh_stress_room(64, 48)  # the 1024 x 512 UV sphere: 2^20 triangles
    desc = sb.desc()
    n = 10_000_000
    o, d = scenes.random_rays(n, 20240607, (-2.8, -2.8, 0.1), (2.8, 2.8, 3.9), (-1.1, -1.1, 0.1), (1.1, 1.1, 2.3))
    rb, rp, rt = ReferenceEngine(desc).cast_rays(o, d)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        assert c.bvh_info()["triangles"] == 1 << 20
        gb, gp, gt = c.cast_rays(o, d)
    same = (gb == rb) & (gp == rp)
    both = (rb != A.KNONE) & (gb != A.KNONE)
    # identities: every disagreement is a near-tie (the two crossings lie at the same distance)
    diff = ~same
    ties = diff & both & (np.abs(gt - rt) <= 1e-5 * np.maximum(1.0, rt))
    # a ray through a triangle's edge within FP32 rounding can take the neighbour's crossing or
    # pass on to the next surface: such edge cases are logged, and must stay below one in 10^6
    edge = diff & ~ties
    save_artifact("c2_edge_cases", o=o[edge], d=d[edge], ref=np.stack([rb[edge], rp[edge], rt[edge]], 1),
                  gpu=np.stack([gb[edge], gp[edge], gt[edge]], 1))
    assert edge.sum() <= 1e-6 * n, f"{int(edge.sum())} disagreements that are not near-ties"
    hit = same & (rb != A.KNONE)
    rel = np.abs(gt[hit] - rt[hit]) / rt[hit]
    stats = {"rays": n, "hits": int(hit.sum()), "ties": int(ties.sum()), "edge_cases": int(edge.sum()),
             "rel_median": float(np.median(rel)),
             "within_1e-6": float(np.mean(rel <= 1e-6)), "rel_max": float(rel.max())}
    save_artifact("c2_ray_cast_stats", **{k: np.array(v) for k, v in stats.items()})
    assert ties.sum() <= 1e-4 * n, stats
    # the traversal finds the triangle in FP32; the distance is then recomputed from the FP64
    # vertices: every hit on the reference's own triangle agrees to 1e-6 relative
    assert stats["rel_max"] <= 1e-6, stats


def test_c1_film_at_4096_spp_matches_the_reference_streams():
    """Same seed, same streams (4096 one-sample passes on both sides, as the device runs a pass):
    the mean relative error over the lit pixels stays below 1 %."""
    desc = scenes.glass_sphere_on_floor(24, 24).desc()
    s = A.make_settings(seed=0, max_depth=16, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    spp = 4096
    ref, _ = ReferenceEngine(desc).render(s, 1, passes=spp)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(s)
        c.run_pass(spp)
        gpu, n = c.resolve()
    assert n.min() == spp
    save_artifact("c1_4096spp", ref=ref, gpu=gpu)
    y_ref, y_gpu = ref[:, :, 1], gpu[:, :, 1]
    lit = y_ref > 1e-3 * y_ref.mean()
    rel = np.abs(y_gpu[lit] - y_ref[lit]) / y_ref[lit]
    assert rel.mean() < 0.01, (rel.mean(), rel.max())
    assert abs(y_gpu.mean() / y_ref.mean() - 1) < 0.005


def test_c5_fog_room_paths_follow_the_reference_and_agree_statistically():
    """The participating-medium configuration at a reduced size (sigma_s 0.5 /m, sigma_a 0.05 /m,
    HG g = 0.8, a PMMA heightfield panel, depth 24): one-sample paths make the reference's
    decisions, and independent 32-spp runs pass the block z-test."""
    from oracle_ref import block_z_test
    desc = scenes.fog_room(48, 36).desc()
    ref = ReferenceEngine(desc)
    s = A.make_settings(seed=5, max_depth=24, rr_depth=6)
    one_ref, _ = ref.render(s, 1, passes=1)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(s)
        c.run_pass(1)
        one_gpu = c.resolve()[0]
        a, b = one_ref[:, :, 1].ravel(), one_gpu[:, :, 1].ravel()
        close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
        assert close.mean() > 0.95, close.mean()
        runs_ref, runs_gpu = [], []
        for k in range(6):
            img, st = ref.render(A.make_settings(seed=100 + k, max_depth=24, rr_depth=6), 32)
            runs_ref.append(img)
            assert st["leaks"] == 0
            c.set_settings(A.make_settings(seed=200 + k, max_depth=24, rr_depth=6))
            c.reset_film()
            c.run_pass(32)
            runs_gpu.append(c.resolve()[0])
        assert c.stats()["device_faults"] == 0
    save_artifact("c5_fog_room_runs", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep


def _band(img, r0, r1):
    return img[r0:r1]


def _same_streams(ref, gpu, floor=1e-3):
    """Mean relative error of the Y channel over the pixels the reference lit."""
    y_ref, y_gpu = ref[..., 1], gpu[..., 1]
    lit = y_ref > floor * y_ref.mean()
    return float((np.abs(y_gpu[lit] - y_ref[lit]) / y_ref[lit]).mean())


def _one_sample_agreement(ref, gpu):
    a, b = ref[..., 1].ravel(), gpu[..., 1].ravel()
    return float((np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)).mean())


def _check_band(desc, settings_of, r0, r1, spp_same, runs, spp_run, name):
    """The device film of the whole frame against the reference's rows r0 .. r1 - 1: one-sample paths,
    spp_same samples on the same streams, and `runs` independent runs of spp_run each side."""
    from oracle_ref import block_z_test
    ref = ReferenceEngine(desc)
    w = desc.detector.width
    px = (r0 * w, r1 * w)
    one_ref, _ = ref.render(settings_of(0), 1, passes=1, pixel_begin=px[0], pixel_end=px[1])
    many_ref, st_ref = ref.render(settings_of(0), 1, passes=spp_same, pixel_begin=px[0], pixel_end=px[1])
    runs_ref = [ref.render(settings_of(100 + k), spp_run, pixel_begin=px[0], pixel_end=px[1])[0][r0:r1]
                for k in range(runs)]
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(settings_of(0))
        c.run_pass(1)
        one_gpu = c.resolve()[0]
        c.reset_film()
        c.run_pass(spp_same)
        many_gpu = c.resolve()[0]
        runs_gpu = []
        for k in range(runs):
            c.set_settings(settings_of(200 + k))
            c.reset_film()
            c.run_pass(spp_run)
            runs_gpu.append(c.resolve()[0][r0:r1])
        st = c.stats()
    save_artifact(name, one_ref=one_ref[r0:r1], one_gpu=one_gpu[r0:r1], many_ref=many_ref[r0:r1],
                  many_gpu=many_gpu[r0:r1], runs_ref=np.array(runs_ref), runs_gpu=np.array(runs_gpu))
    assert st["device_faults"] == 0 and st_ref["leaks"] == 0
    agree = _one_sample_agreement(one_ref[r0:r1], one_gpu[r0:r1])
    assert agree > 0.95, agree
    err = _same_streams(many_ref[r0:r1], many_gpu[r0:r1])
    assert err < 0.01, err
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep
    return agree, err, rep


def test_c1_at_its_configuration():
    """C1 as configured (256 x 256, 64 spp, one wavelength per path, depth 16, roulette after 4,
    seed 0): the whole film on the same streams and eight independent 64-spp runs a side; and a band
    of 32 rows at 4096 spp on the same streams, mean relative error below 1 %."""
    desc = scenes.glass_sphere_on_floor(256, 256).desc()

    def settings_of(seed):
        return A.make_settings(seed=seed, max_depth=16, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)

    _check_band(desc, settings_of, 0, 256, 64, 8, 64, "c1_config")
    ref = ReferenceEngine(desc)
    r0, r1 = 112, 144
    band, _ = ref.render(settings_of(0), 1, passes=4096, pixel_begin=r0 * 256, pixel_end=r1 * 256)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(settings_of(0))
        c.run_pass(4096)
        gpu, n = c.resolve()
    assert n.min() == 4096
    err = _same_streams(band[r0:r1], gpu[r0:r1])
    assert err < 0.01, err


def test_c2_band_at_its_configuration():
    """C2's frame (1920 x 1080, hero-4, depth 12, the 2^20-triangle room): eight rows through the
    displaced sphere, one-sample paths, 256 spp on the same streams, and six independent 32-spp runs."""
    desc = scenes.bvh_stress_room(1920, 1080).desc()

    def settings_of(seed):
        return A.make_settings(seed=seed, max_depth=12, rr_depth=6, wavelength_mode=A.WAVELENGTHS_HERO4)

    _check_band(desc, settings_of, 536, 544, 256, 6, 32, "c2_band")


def test_c2_paths_leaving_the_mesh_meet_no_inconsistent_region():
    """Paths that leave the displaced sphere near a concave edge meet the neighbouring triangle from
    the room, as the reference's mesh departure has them (only the departed triangle is excluded
    near the anchor): none of 2 M mixed-precision paths of C2's room meets the mesh from inside.
    (Excluding the whole departed mesh near the anchor let about 7 in 10^6 paths into the body.)"""
    desc = scenes.bvh_stress_room(960, 540).desc()
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_settings(A.make_settings(seed=3, max_depth=12, rr_depth=6))
        c.run_pass(4)
        st = c.stats()
    assert st["paths"] == 960 * 540 * 4
    assert st["inconsistencies"] == 0 and st["leaks"] == 0 and st["device_faults"] == 0, st


def test_c5_band_at_its_configuration():
    """C5's frame (1920 x 1080, depth 24, the fog-filled caustic room: 6.29 M triangles with the
    1024 x 1024 heightfield panel): sixteen rows across the panel, one-sample paths, 64 spp on the
    same streams, and six independent 16-spp runs."""
    sb, _ = scenes.caustic_room(1920, 1080)
    desc = sb.desc()

    def settings_of(seed):
        return A.make_settings(seed=seed, max_depth=24, rr_depth=6, wavelength_mode=A.WAVELENGTHS_HERO4)

    _check_band(desc, settings_of, 640, 656, 64, 6, 16, "c5_band")
