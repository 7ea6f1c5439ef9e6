"""The torch.autograd.Function wrappers' host logic on CPU: a stand-in context whose film is a fixed
linear map of the heights, so that the wrapper's backward must return the map's transpose applied to
the incoming gradient, and must differentiate at the heights of its own forward call."""
import numpy as np
import torch

import owe_autograd


class LinearContext:
    """The Context calls the wrappers make, with film = M @ heights."""

    def __init__(self, n_heights, n_bins, seed=0):
        self.M = np.random.default_rng(seed).normal(size=(n_bins, n_heights))
        self.sets = 0

    def set_heightfield(self, boundary, base_z, heights):
        self._hf_heights = np.array(heights, np.float64).ravel()
        self._hf_boundary = boundary
        self.sets += 1

    # walk film
    def walk_reset(self):
        pass

    def walk(self, desc, first, n):
        self._film = self.M @ self._hf_heights

    def walk_resolve(self):
        return self._film.copy(), {"faults": 0}

    def walk_adjoint(self, desc, first, n, g):
        # the adjoint at the context's current heights (here the map does not depend on them)
        return self.M.T @ np.asarray(g).ravel()


def test_walk_film_gradient_is_the_adjoint_of_the_forward():
    c = LinearContext(12, 30)
    h = torch.tensor(np.linspace(-1, 1, 12), dtype=torch.float64, requires_grad=True)
    target = torch.linspace(0, 1, 30, dtype=torch.float64)
    film = owe_autograd.walk_film(h, c, 3, 0.0, None, 0, 100)
    loss = ((film - target) ** 2).sum()
    loss.backward()
    expect = c.M.T @ (2 * (c.M @ h.detach().numpy() - target.numpy()))
    assert np.allclose(h.grad.numpy(), expect, rtol=1e-12, atol=1e-12)


def test_backward_restores_the_heights_of_its_forward():
    c = LinearContext(4, 5)
    h1 = torch.tensor([0.1, 0.2, 0.3, 0.4], dtype=torch.float64, requires_grad=True)
    f1 = owe_autograd.walk_film(h1, c, 0, 0.0, None, 0, 10)
    # another forward at other heights moves the context's heightfield
    owe_autograd.walk_film(torch.zeros(4, dtype=torch.float64), c, 0, 0.0, None, 0, 10)
    assert np.array_equal(c._hf_heights, np.zeros(4))
    f1.sum().backward()
    assert np.array_equal(c._hf_heights, h1.detach().numpy())


class LinearCameraContext(LinearContext):
    """The camera-film calls, with film = M @ heights (one channel) and a record of the sample
    streams each call used."""

    def reset_film(self):
        pass

    def set_pass_index(self, first):
        self.first = first

    def run_pass(self, spp):
        self.forward_streams = (self.first, spp)
        self._film = self.M @ self._hf_heights

    def resolve(self, samples=False):
        return self._film.reshape(-1, 1, 1).repeat(3, axis=2), None

    def path_adjoint(self, first_pass, spp, g, fixed_decisions=False):
        self.adjoint_streams = (first_pass, spp, fixed_decisions)
        return self.M.T @ np.asarray(g)[:, 0, 1]


def test_camera_film_replays_the_streams_it_is_given():
    c = LinearCameraContext(6, 9)
    h = torch.tensor(np.linspace(-1, 1, 6), dtype=torch.float64, requires_grad=True)
    film = owe_autograd.camera_film(h, c, 2, 0.0, 40, 8)
    film[:, 0, 1].sum().backward()
    assert c.forward_streams == (40, 8) and c.adjoint_streams == (40, 8, False)
    assert np.allclose(h.grad.numpy(), c.M.T @ np.ones(9), rtol=1e-12)
    h.grad = None
    film = owe_autograd.camera_film(h, c, 2, 0.0, 40, 8, adjoint_pass=48)
    film[:, 0, 1].sum().backward()
    assert c.forward_streams == (40, 8) and c.adjoint_streams == (48, 8, False)
