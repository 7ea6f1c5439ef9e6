"""The camera-path adjoint (owec_path_adjoint): the gradient of a loss on the camera film with respect
to the heights of a refractive heightfield, by path replay.

The check scene is a PMMA panel with a heightfield top held above a Lambertian floor and seen from
above, so that the image is the floor seen through the refracting heights; a lamp at the side lights
the floor with a strong falloff, next-event estimation and MIS emission hits reach it, and a dim sky
lights the rest. With fixed decisions the adjoint is the derivative of the film's estimator at its
own random numbers, which is what central differences of the reference engine's own renders
(CpuRenderer's pass loop, the same sample streams) measure at a small eps: the two must agree vertex
by vertex. The gradients are taken through the torch.autograd.Function over the owec_pass /
owec_path_adjoint pair (the two-phase adjoint: wavefront to the first heightfield crossing, then the
derivative replay from the checkpoints); the full replay from the camera checks the replayed film."""
import numpy as np
import pytest
import torch

import owe_autograd
import owe_cuda
import owec_abi as A
import scenes
from conftest import save_artifact
from oracle_ref import ReferenceEngine

pytestmark = pytest.mark.gpu

N = 16
W = H = 32
SPP = 64


def _heights(seed=2, amplitude=1e-3):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:N, 0:N] / (N - 1)
    h = np.zeros((N, N))
    for _ in range(5):
        fx, fy, ph = rng.uniform(1, 3), rng.uniform(1, 3), rng.uniform(0, 2 * np.pi)
        h += np.sin(np.pi * fx * x + ph) * np.sin(np.pi * fy * y)
    h *= amplitude / np.abs(h).max()
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = 0  # the border is shared with the slab's sides
    return h


def _settings(precision, max_depth=6, rr_depth=3):
    return A.make_settings(seed=5, max_depth=max_depth, rr_depth=rr_depth, wavelength_mode=A.WAVELENGTHS_HERO4,
                           precision=precision)


def _loss_weights(seed=9):
    return np.random.default_rng(seed).normal(size=(H, W, 3))


def _adjoint(h, settings, fog=None, fixed=True):
    sb, info = scenes.refraction_panel(n=N, heights=h, width=W, height=H, fog=fog)
    g = _loss_weights()
    with owe_cuda.Context() as c:
        c.set_settings(settings)
        c.upload(sb.desc())
        c.build_bvh()
        heights = torch.tensor(h.ravel(), dtype=torch.float64, requires_grad=True)
        film = owe_autograd.camera_film(heights, c, info["heightfield"], info["base_z"], 0, SPP, fixed_decisions=fixed)
        (film * torch.from_numpy(g)).sum().backward()
        grad = heights.grad.numpy().reshape(N, N)
        _, st = c.path_adjoint(0, SPP, g, with_stats=True, fixed_decisions=fixed)[:2]
        full, st_full, replay = c.path_adjoint(0, SPP, g, replay=True, with_stats=True, fixed_decisions=fixed)
        return grad, film.detach().numpy(), replay, full.reshape(N, N), st, st_full


def _reference_differences(h, settings, picks, eps, fog=None):
    """Central differences of sum(g * film) of the reference's renders at h +- eps e_k."""
    g = _loss_weights()
    fd = []
    for (j, i) in picks:
        side = []
        for sgn in (1, -1):
            hh = h.copy()
            hh[j, i] += sgn * eps
            sb, _ = scenes.refraction_panel(n=N, heights=hh, width=W, height=H, fog=fog)
            img, _ = ReferenceEngine(sb.desc()).render(settings, 1, passes=SPP, first_pass=0)
            side.append(img)
        fd.append(float((g * (side[0] - side[1])).sum() / (2 * eps)))
    return np.array(fd)


def _check(precision, fog=None, tol=0.02):
    h = _heights()
    s = _settings(precision)
    grad, film, replay, full, st, st_full = _adjoint(h, s, fog=fog)
    assert st["faults"] == 0 and st["dropped"] == 0, st
    assert st["paths"] == W * H * SPP and st["heightfield"] > 0.2 * st["paths"], st
    # both ways reach the heightfield with the same paths (up to a decision a rounding may turn)
    assert abs(st_full["heightfield"] - st["heightfield"]) <= 1e-4 * st["heightfield"], (st, st_full)
    # the full replay walks the forward's paths: the same film
    assert np.allclose(replay, film, rtol=1e-6, atol=1e-9 * np.abs(film).max()), np.abs(replay - film).max()
    # and the same gradient as the replay from the checkpoints
    assert np.linalg.norm(full - grad) <= 1e-3 * np.linalg.norm(grad), np.abs(full - grad).max()
    rng = np.random.default_rng(11)
    picks = [(int(j), int(i)) for j, i in rng.integers(1, N - 1, size=(32, 2))]
    # Two step sizes: a vertex whose differences disagree between them has a path decision (a branch,
    # an edge, a shadow boundary) within eps of its height, where the difference measures a jump,
    # not the derivative; such vertices are left out, at most two of them.
    fd = _reference_differences(h, s, picks, eps=1e-10, fog=fog)
    fd2 = _reference_differences(h, s, picks, eps=3e-11, fog=fog)
    smooth = np.abs(fd - fd2) <= 1e-2 * np.abs(fd2) + 1e-6 * np.abs(fd2).max()
    assert smooth.sum() >= len(picks) - 2, list(zip(picks, fd, fd2))
    adj = np.array([grad[v] for v in picks])
    err = np.abs(adj - fd2)
    ok = ~smooth | (err <= tol * np.abs(fd2) + 1e-3 * np.abs(fd2[smooth]).max())
    if not ok.all():
        save_artifact(f"path_adjoint_{precision}_{fog is not None}", adj=adj, fd=fd, fd2=fd2, picks=np.array(picks))
    assert ok.all(), list(zip(picks, adj, fd2, smooth))


def test_path_adjoint_matches_reference_differences_fp64():
    _check(A.PRECISION_FP64)


def test_path_adjoint_matches_reference_differences_in_fog_fp64():
    _check(A.PRECISION_FP64, fog=(0.3, 0.03, 0.6))


def test_path_adjoint_matches_reference_differences_mixed():
    # the product's precision: FP32 geometry may turn a path's decision the other way than the
    # reference's FP64 does, which a per-vertex comparison sees as noise
    _check(A.PRECISION_MIXED, tol=0.05)


def test_path_adjoint_refuses_what_it_does_not_differentiate():
    sb, info = scenes.refraction_panel(n=N, width=W, height=H)
    with owe_cuda.Context() as c:
        c.upload(sb.desc())
        c.build_bvh()
        with pytest.raises(RuntimeError, match="no heightfield"):
            c.path_adjoint(0, 1, np.zeros((H, W, 3)))
        c.set_heightfield(info["heightfield"], info["base_z"], np.zeros(N * N))
        c.set_settings(A.make_settings(seed=1, integrator=A.INTEGRATOR_LIGHT))
        with pytest.raises(RuntimeError, match="path integrator"):
            c.path_adjoint(0, 1, np.zeros((H, W, 3)))


def test_gradient_descent_recovers_the_heights():
    """An inverse problem through owe_autograd.camera_film: Adam, from flat heights, matches the film
    of seeded target heights (3 mm bumps, 1024 spp) with the default (unbiased) gradient, each step's
    gradient from a replay on other sample streams than its film. The heights' RMS distance to the
    target falls below half of where it started, and the loss of a fresh 1024-spp film falls with it."""
    w = h = 64
    target_h = _heights(seed=4, amplitude=3e-3)
    sb, info = scenes.refraction_panel(n=N, width=w, height=h)
    hf, base_z = info["heightfield"], info["base_z"]
    interior = np.zeros((N, N))
    interior[1:-1, 1:-1] = 1
    mask = torch.from_numpy(interior.ravel())
    with owe_cuda.Context() as c:
        c.set_settings(_settings(A.PRECISION_MIXED))
        c.upload(sb.desc())
        c.build_bvh()
        with torch.no_grad():
            target = owe_autograd.camera_film(torch.from_numpy(target_h.ravel()), c, hf, base_z, 1 << 20, 1024)

        def loss_of(heights, first, spp):
            with torch.no_grad():
                return float(((owe_autograd.camera_film(heights, c, hf, base_z, first, spp) - target) ** 2).mean())

        heights = torch.zeros(N * N, dtype=torch.float64, requires_grad=True)
        steps, spp = 200, 64
        opt = torch.optim.Adam([heights], lr=1e-4)
        decay = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=0.1 ** (1.0 / steps))
        loss0 = loss_of(heights.detach(), 1 << 22, 1024)
        for k in range(steps):
            opt.zero_grad()
            film = owe_autograd.camera_film(heights * mask, c, hf, base_z, 2 * k * spp, spp,
                                            adjoint_pass=(2 * k + 1) * spp)
            ((film - target) ** 2).mean().backward()
            opt.step()
            decay.step()
        final = (heights.detach() * mask).numpy()
        loss1 = loss_of(torch.from_numpy(final), 1 << 22, 1024)
    rmse0 = np.sqrt((target_h ** 2).mean())
    rmse1 = np.sqrt(((final.reshape(N, N) - target_h) ** 2).mean())
    save_artifact("path_adjoint_descent", target=target_h, final=final.reshape(N, N), losses=np.array([loss0, loss1]))
    assert rmse1 < 0.5 * rmse0, (rmse0, rmse1, loss0, loss1)
    assert loss1 < loss0, (loss0, loss1)
