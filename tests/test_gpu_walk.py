"""Forward light walks on the GPU (the reference's Tracer::walk) against the reference engine:
a point source imaged by the cemented achromat onto a detector at its paraxial focus."""
import math

import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from oracle_ref import ReferenceEngine

pytestmark = pytest.mark.gpu


def _walk_gpu(desc, w, n, chunk=1 << 20):
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.walk_reset()
        for first in range(0, n, chunk):
            c.walk(w, first, min(chunk, n - first))
        return c.walk_resolve()


def test_achromat_primary_transmission_walks_follow_the_reference_walks():
    """Deterministic Fresnel weights, one wavelength: each device walk makes the CPU walk's
    decisions, so the binned images agree bin for bin to rounding of the landing points."""
    sb, info = scenes.achromat_scene(film=64, half_size=2.5e-4)
    desc = sb.desc()
    w = scenes.achromat_walk(info, seed=3, mode=A.WALK_PRIMARY_TRANSMISSION, lambda_range=(587.5618, 587.5618))
    n = 200_000
    ref_bins, ref_st = ReferenceEngine(desc).walk(w, 0, n)
    gpu_bins, gpu_st = _walk_gpu(desc, w, n)
    assert gpu_st["faults"] == 0
    assert abs(gpu_st["binned"] - ref_st["binned"]) <= 1e-3 * n
    assert abs(gpu_bins.sum() - ref_bins.sum()) <= 2e-3 * ref_bins.sum()
    # the spot: the same centroid and RMS radius
    ys, xs = np.mgrid[0:64, 0:64]
    for b in (ref_bins, gpu_bins):
        b /= b.sum()
    rc = [(b * xs).sum() for b in (ref_bins, gpu_bins)]
    rr = [math.sqrt((b * ((xs - 31.5) ** 2 + (ys - 31.5) ** 2)).sum()) for b in (ref_bins, gpu_bins)]
    assert abs(rc[0] - rc[1]) < 0.05 and abs(rr[0] - rr[1]) < 0.02 * rr[0]
    assert np.abs(gpu_bins - ref_bins).sum() < 0.01


def test_achromat_stochastic_walks_with_ghosts_agree_statistically():
    """Monte-Carlo branching at every face (ghost reflections, depth 32) over the visible range:
    the device and the reference estimate the same image."""
    sb, info = scenes.achromat_scene(film=32, half_size=2.5e-4)
    desc = sb.desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    for k in range(6):
        w = scenes.achromat_walk(info, seed=100 + k)
        runs_ref.append(ref.walk(w, 0, 100_000)[0])
        w = scenes.achromat_walk(info, seed=200 + k)
        runs_gpu.append(_walk_gpu(desc, w, 100_000)[0])
    a, b = np.array(runs_ref), np.array(runs_gpu)
    # 4 x 4 blocks of 8 x 8 bins
    A4 = a.reshape(6, 4, 8, 4, 8).sum((2, 4))
    B4 = b.reshape(6, 4, 8, 4, 8).sum((2, 4))
    se = np.sqrt(A4.var(0, ddof=1) / 6 + B4.var(0, ddof=1) / 6)
    z = (B4.mean(0) - A4.mean(0)) / np.where(se > 0, se, 1)
    assert np.all(np.abs(z[se > 0]) < 4.5), z
    assert abs(B4.mean(0).sum() / A4.mean(0).sum() - 1) < 0.01


def test_walk_film_is_deterministic_across_batch_splits():
    sb, info = scenes.achromat_scene(film=32, half_size=2.5e-4)
    desc = sb.desc()
    w = scenes.achromat_walk(info, seed=9)
    a, _ = _walk_gpu(desc, w, 300_000, chunk=300_000)
    b, _ = _walk_gpu(desc, w, 300_000, chunk=70_000)
    assert np.array_equal(a, b)


def _spot(bins, half):
    """Centroid (x, y) and RMS radius about it of a binned spot, in metres on the detector."""
    n = bins.shape[0]
    w = bins / bins.sum()
    c = (np.arange(n) + 0.5) / n * 2 * half - half
    X, Y = np.meshgrid(c, -c)
    cx, cy = (w * X).sum(), (w * Y).sum()
    return cx, cy, math.sqrt((w * ((X - cx) ** 2 + (Y - cy) ** 2)).sum())


def test_c3_lens_at_its_configuration():
    """C3 as configured: the cemented achromat imaging a point source 10 m away onto a 1024 x 1024
    detector placed at the paraxial focus the reference's own paraxial analysis gives
    (paraxialAnalysis, as tests/test_instruments.cpp:249 places it); 10^9 walks over 380-780 nm,
    Monte-Carlo Fresnel branching with ghosts, depth 32. The spot diagram (centroid, RMS radius) of
    the 10^9 walks against the reference's Tracer::walk over a subsample, and the image error of the
    same 2^22 walks (common random numbers) bin for bin."""
    from oracle_ref import paraxial_image_distance
    sb, info = scenes.achromat_scene(film=1024, half_size=2.5e-4)
    wl = 587.5618
    back = paraxial_image_distance([0.0615, -0.0446, -0.129], [0.006, 0.0025], [scenes.NBK7, scenes.SF5], 10.0, wl)
    assert abs(0.0085 + back - info["z_focus"]) < 1e-9  # the detector where the reference puts the focus
    desc = sb.desc()
    w = scenes.achromat_walk(info, seed=5, max_events=32)
    sub = 1 << 22
    ref_bins, ref_st = ReferenceEngine(desc).walk(w, 0, sub)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.walk(w, 0, sub)
        same, st = c.walk_resolve()
        c.walk_reset()
        total = 10 ** 9
        for first in range(0, total, 1 << 27):
            c.walk(w, first, min(1 << 27, total - first))
        full, st_full = c.walk_resolve()
    assert st["faults"] == 0 and st_full["faults"] == 0 and st_full["walks"] == total
    # the same walks: the same image, up to landing points that rounding moves across a bin edge
    assert np.abs(same - ref_bins).sum() <= 0.01 * ref_bins.sum(), np.abs(same - ref_bins).sum() / ref_bins.sum()
    half = info["half"]
    rx, ry, rr = _spot(ref_bins, half)
    gx, gy, gr = _spot(full, half)
    bin_size = 2 * half / 1024
    assert abs(gx - rx) < 0.25 * bin_size and abs(gy - ry) < 0.25 * bin_size, (gx, rx, gy, ry)
    assert abs(gr / rr - 1) < 0.02, (gr, rr)
    assert abs(full.sum() / ref_bins.sum() - 1) < 0.005
