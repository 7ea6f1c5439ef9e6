"""The path-replay adjoint of the differentiable caustic: the gradient of an L2 loss on the wall's
irradiance with respect to the heights of the slab's exit face, taken through the
torch.autograd.Function over owec_walk / owec_walk_adjoint, against FP64 central finite differences
of the reference engine's own walks (Tracer::walk) with common random numbers.

The finite difference of vertex k needs only the walks that can meet the triangles around k: the
beam crosses the flat entry face at normal incidence, so a walk reaches the exit face where it
entered, and every walk outside the vertex's star repeats the same arithmetic at h + eps and
h - eps and cancels exactly. The reference runs just those walks (oweref_walk_in_box) at both
heights; the loss difference is then exact to second order in eps."""
import numpy as np
import pytest
import torch

import owe_autograd
import owe_cuda
import scenes
from oracle_ref import ReferenceEngine, normalise_walk_bins

pytestmark = pytest.mark.gpu


def _random_heights(n, seed=4, amplitude=1.5e-4):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:n, 0:n] / (n - 1)
    h = np.zeros((n, n))
    for _ in range(6):
        fx, fy, ph = rng.uniform(1, 3), rng.uniform(1, 3), rng.uniform(0, 2 * np.pi)
        h += np.sin(np.pi * fx * x + ph) * np.sin(np.pi * fy * y)
    h *= amplitude / np.abs(h).max()
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = 0  # the border is shared with the slab's sides
    return h


def _check_gradient(n, bins, walks, h, target, eps, vertices=32, seed=11):
    """Adjoint gradient (autograd over the CUDA forward/backward pair) against reference central
    differences on `vertices` interior vertices drawn uniformly; returns the relative errors."""
    sb, info = scenes.caustic_slab_scene(n=n, heights=h, wall_bins=bins)
    w = scenes.caustic_walk(info, seed=7)
    with owe_cuda.Context() as c:
        c.upload(sb.desc())
        c.build_bvh()
        heights = torch.tensor(h.ravel(), dtype=torch.float64, requires_grad=True)
        film = owe_autograd.walk_film(heights, c, info["heightfield"], info["thickness"], w, 0, walks)
        loss = ((film - torch.from_numpy(target)) ** 2).sum()
        loss.backward()
        grad = heights.grad.numpy().reshape(n, n)
        gpu_bins = film.detach().numpy()
    ref_full, _ = ReferenceEngine(sb.desc()).walk(w, 0, walks)
    # the forward agrees with the reference's walks
    assert np.abs(gpu_bins - ref_full).sum() <= 1e-3 * ref_full.sum()
    g = 2 * (ref_full - target)
    xs = np.linspace(-info["half"], info["half"], n)
    rng = np.random.default_rng(seed)
    picks = [(int(j), int(i)) for j, i in rng.integers(1, n - 1, size=(vertices, 2))]
    fd = []
    for (j, i) in picks:
        # the star of the vertex, widened by a cell: every walk that can meet its triangles
        box = [xs[max(i - 2, 0)], xs[min(i + 2, n - 1)], xs[max(j - 2, 0)], xs[min(j + 2, n - 1)], -1.0, 1.0]
        side = []
        for sgn in (1, -1):
            hh = h.copy()
            hh[j, i] += sgn * eps
            sbh, _ = scenes.caustic_slab_scene(n=n, heights=hh, wall_bins=bins)
            raw, _ = ReferenceEngine(sbh.desc()).walk_in_box(w, 0, walks, box)
            side.append(normalise_walk_bins(w, raw.ravel(), walks))
        fd.append(float((g * (side[0] - side[1])).sum() / (2 * eps)))
    fd = np.array(fd)
    adj = np.array([grad[v] for v in picks])
    return adj, fd, picks


def test_adjoint_gradient_at_the_caustic_configuration():
    """C4 as configured: a 256 x 256 heightfield at its initial heights (0), a 512 x 512 wall, 2^24
    walks, the L2 loss to 64 seeded Gaussian blobs of sigma 5-20 bins; every one of 32 uniformly
    drawn interior vertices within 2 % of the reference's central difference."""
    n, bins, walks = 256, 512, 1 << 24
    target = scenes.gaussian_blobs(bins, count=64, seed=3, sigma_range=(5.0, 20.0))
    adj, fd, picks = _check_gradient(n, bins, walks, np.zeros((n, n)), target, eps=1e-11)
    rel = np.abs(adj - fd) / np.abs(fd)
    assert np.all(rel < 0.02), list(zip(picks, adj, fd, rel))


def test_adjoint_gradient_on_a_curved_heightfield():
    """The same check away from the flat slab (tilted triangles: oblique refraction, Fresnel
    slopes) on a smaller case: 32 x 32 heights of seeded sine bumps, 64 x 64 bins, 2^18 walks."""
    n, bins, walks = 32, 64, 1 << 18
    target = scenes.gaussian_blobs(bins, count=16, seed=3, sigma_range=(2.0, 6.0)) * 0.4
    adj, fd, picks = _check_gradient(n, bins, walks, _random_heights(n), target, eps=1e-11)
    rel = np.abs(adj - fd) / np.abs(fd)
    assert np.all(rel < 0.02), list(zip(picks, adj, fd, rel))


def test_adjoint_costs_at_most_three_forward_passes():
    n, bins = 32, 64
    h = _random_heights(n)
    sb, info = scenes.caustic_slab_scene(n=n, heights=h, wall_bins=bins)
    w = scenes.caustic_walk(info, seed=1)
    with owe_cuda.Context() as c:
        c.upload(sb.desc())
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["thickness"], h)
        fw, ad = [], []
        for _ in range(3):
            c.walk(w, 0, 1 << 22)
            fw.append(c.walk_timing()[0])
            g = np.ones(bins * bins)
            c.walk_adjoint(w, 0, 1 << 22, g)
            ad.append(c.walk_timing()[1])
    assert min(ad) <= 3 * min(fw), (fw, ad)
