"""The path-replay adjoint of the differentiable caustic: the gradient of an L2 loss on the wall's
irradiance with respect to the heights of the slab's exit face, against FP64 central finite
differences of the reference engine's own walks (Tracer::walk) with common random numbers."""
import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from oracle_ref import ReferenceEngine

pytestmark = pytest.mark.gpu

N = 32          # heightfield vertices per side
BINS = 64
WALKS = 1 << 18


def _heights(seed=4, amplitude=1.5e-4):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:N, 0:N] / (N - 1)
    h = np.zeros((N, N))
    for _ in range(6):
        fx, fy, ph = rng.uniform(1, 3), rng.uniform(1, 3), rng.uniform(0, 2 * np.pi)
        h += np.sin(np.pi * fx * x + ph) * np.sin(np.pi * fy * y)
    h *= amplitude / np.abs(h).max()
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = 0  # the border is shared with the slab's sides
    return h


def _ref_loss(h, info_seed, target):
    sb, info = scenes.caustic_slab_scene(n=N, heights=h, wall_bins=BINS)
    w = scenes.caustic_walk(info, seed=info_seed)
    bins, _ = ReferenceEngine(sb.desc()).walk(w, 0, WALKS)
    return float(((bins - target) ** 2).sum()), bins


def test_adjoint_gradient_matches_fp64_central_differences():
    h = _heights()
    sb, info = scenes.caustic_slab_scene(n=N, heights=h, wall_bins=BINS)
    desc = sb.desc()
    target = scenes.gaussian_blobs(BINS, count=16, seed=3, sigma_range=(2.0, 6.0)) * 0.4
    w = scenes.caustic_walk(info, seed=7)
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["thickness"], h)
        c.walk(w, 0, WALKS)
        bins, st = c.walk_resolve()
        assert st["faults"] == 0 and st["binned"] > 0.99 * WALKS
        g = 2 * (bins - target)
        grad = c.walk_adjoint(w, 0, WALKS, g).reshape(N, N)
    # the forward agrees with the reference's walks
    _, ref_bins = _ref_loss(h, 7, target)
    assert np.abs(bins - ref_bins).sum() <= 1e-2 * ref_bins.sum()
    # central differences on 32 interior vertices with a clear gradient
    rng = np.random.default_rng(11)
    interior = [(j, i) for j in range(2, N - 2) for i in range(2, N - 2)]
    strong = [v for v in interior if abs(grad[v]) > 0.2 * np.abs(grad).max()]
    picks = [strong[k] for k in rng.choice(len(strong), size=min(32, len(strong)), replace=False)]
    eps = 1e-8
    rel = []
    for (j, i) in picks:
        hp, hm = h.copy(), h.copy()
        hp[j, i] += eps
        hm[j, i] -= eps
        fd = (_ref_loss(hp, 7, target)[0] - _ref_loss(hm, 7, target)[0]) / (2 * eps)
        rel.append(abs(grad[j, i] - fd) / abs(fd))
    rel = np.array(rel)
    assert np.median(rel) < 0.02, rel
    assert np.mean(rel < 0.05) > 0.85, rel


def test_adjoint_costs_at_most_three_forward_passes():
    h = _heights()
    sb, info = scenes.caustic_slab_scene(n=N, heights=h, wall_bins=BINS)
    w = scenes.caustic_walk(info, seed=1)
    with owe_cuda.Context() as c:
        c.upload(sb.desc())
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["thickness"], h)
        fw, ad = [], []
        for _ in range(3):
            c.walk(w, 0, 1 << 22)
            fw.append(c.walk_timing()[0])
            g = np.ones(BINS * BINS)
            c.walk_adjoint(w, 0, 1 << 22, g)
            ad.append(c.walk_timing()[1])
    assert min(ad) <= 3 * min(fw), (fw, ad)
