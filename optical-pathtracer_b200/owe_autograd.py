"""torch.autograd.Function wrappers over the backend's forward/backward pairs, for the gradient tests.

The C ABI exposes each differentiable measurement as a forward call and a backward call:

    walk film      forward  owec_set_heightfield + owec_walk + owec_walk_resolve
                   backward owec_walk_adjoint (path replay of the same walks)
    camera film    forward  owec_set_heightfield + owec_pass + owec_resolve
                   backward owec_path_adjoint (path replay of the same camera paths)

Here each pair becomes one torch.autograd.Function of the heightfield's heights, so that a loss
written in torch differentiates through the renderer with loss.backward(). The functions run on the
CPU side of torch: heights, films and gradients are float64 tensors on the host, copied through
the C ABI; the device work is the library's. The heightfield optimisation of the large camera
configuration (bench.py --c5) runs through camera_film.
"""
import numpy as np
import torch


def _ensure_heights(context, boundary, base_z, h):
    """Sets the heightfield unless the context already holds exactly these heights (a backward call
    must differentiate at the heights of its own forward call)."""
    cur = getattr(context, "_hf_heights", None)
    if cur is None or cur.shape != h.shape or not np.array_equal(cur, h) or getattr(context, "_hf_boundary", None) != boundary:
        context.set_heightfield(boundary, base_z, h)


class WalkFilm(torch.autograd.Function):
    """bins(heights): the irradiance the forward walks first .. first + n - 1 bin on their target,
    as a function of the heightfield's heights (one per vertex of the heightfield mesh)."""

    @staticmethod
    def forward(ctx, heights, context, boundary, base_z, desc, first, n):
        h = heights.detach().cpu().numpy().astype(np.float64).ravel()
        _ensure_heights(context, boundary, base_z, h)
        context.walk_reset()
        context.walk(desc, first, n)
        bins, stats = context.walk_resolve()
        if stats["faults"]:
            raise RuntimeError(f"walk film: {stats['faults']} walks ran out of their bounds")
        ctx.args = (context, boundary, base_z, desc, first, n, h, heights.shape)
        return torch.from_numpy(bins).to(heights.dtype)

    @staticmethod
    def backward(ctx, grad_bins):
        context, boundary, base_z, desc, first, n, h, shape = ctx.args
        _ensure_heights(context, boundary, base_z, h)
        g = grad_bins.detach().cpu().numpy().astype(np.float64)
        dh = context.walk_adjoint(desc, first, n, g)
        return torch.from_numpy(dh.reshape(shape)).to(grad_bins.dtype), None, None, None, None, None, None


class CameraFilm(torch.autograd.Function):
    """image(heights): the resolved camera film (height x width x 3, XYZ) of `spp` samples per pixel
    from sample stream `first_pass` on, as a function of the heightfield's heights. The backward pass
    is the gradient of the expected film, or with fixed_decisions the derivative of this film's
    estimator at its own random numbers (what central differences with common random numbers
    measure). The backward pass replays the forward pass's sample streams unless adjoint_pass names
    another block of spp streams: an optimiser of a loss that is not linear in the film wants that,
    since the film's noise and the gradient's noise then do not correlate."""

    @staticmethod
    def forward(ctx, heights, context, boundary, base_z, first_pass, spp, fixed_decisions, adjoint_pass=None):
        h = heights.detach().cpu().numpy().astype(np.float64).ravel()
        _ensure_heights(context, boundary, base_z, h)
        context.reset_film()
        context.set_pass_index(first_pass)
        context.run_pass(spp)
        img, _ = context.resolve(samples=False)
        replay = first_pass if adjoint_pass is None else adjoint_pass
        ctx.args = (context, boundary, base_z, replay, spp, fixed_decisions, h, heights.shape)
        return torch.from_numpy(np.array(img)).to(heights.dtype)

    @staticmethod
    def backward(ctx, grad_img):
        context, boundary, base_z, first_pass, spp, fixed, h, shape = ctx.args
        _ensure_heights(context, boundary, base_z, h)
        g = grad_img.detach().cpu().numpy().astype(np.float64)
        dh = context.path_adjoint(first_pass, spp, g, fixed_decisions=fixed)
        return torch.from_numpy(dh.reshape(shape)).to(grad_img.dtype), None, None, None, None, None, None, None


def walk_film(heights, context, boundary, base_z, desc, first, n):
    """The walk film as a differentiable function of `heights` (a float64 tensor)."""
    return WalkFilm.apply(heights, context, boundary, base_z, desc, first, n)


def camera_film(heights, context, boundary, base_z, first_pass, spp, fixed_decisions=False, adjoint_pass=None):
    """The camera film as a differentiable function of `heights` (a float64 tensor)."""
    return CameraFilm.apply(heights, context, boundary, base_z, first_pass, spp, fixed_decisions, adjoint_pass)
