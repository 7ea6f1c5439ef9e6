"""The multi-GPU render's host logic on CPU: the split of the sample streams across ranks and the
film reduction, with world_size 2 over gloo. The device context is replaced by a stand-in whose
film is a deterministic function of (pixel, stream), so that two ranks must reproduce one rank's
film exactly."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import distributed as D

W, H = 7, 5


class FakeContext:
    """The owe_cuda.Context calls distributed.render makes, on a film of known samples."""

    def __init__(self):
        self.width, self.height = W, H
        self.pass_index = 0
        self.sums = np.zeros((H, W, 3))
        self.samples = np.zeros((H, W))
        self.streams = []

    def set_pass_index(self, i):
        self.pass_index = int(i)

    def run_pass(self, spp):
        y, x = np.mgrid[0:H, 0:W]
        for s in range(self.pass_index, self.pass_index + spp):
            self.streams.append(s)
            v = np.sin(0.37 * s + 0.11 * x + 0.05 * y)
            self.sums += np.stack([v, v * v, 1 + v], axis=-1)
            self.samples += 1
        self.pass_index += spp

    def read_film(self):
        return self.sums.copy(), self.samples.copy()


def test_stream_blocks_partition_the_streams():
    for total in (0, 1, 5, 64, 1001):
        for world in (1, 2, 3, 8):
            blocks = [D.stream_block(total, world, r) for r in range(world)]
            covered = [s for f, c in blocks for s in range(f, f + c)]
            assert covered == list(range(total))
            sizes = [c for _, c in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.stream_block(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, total, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ctx = FakeContext()
        mean = D.render(ctx, total, spp_per_pass=3)
        np.save(os.path.join(out, f"mean{rank}.npy"), mean)
        np.save(os.path.join(out, f"streams{rank}.npy"), np.array(ctx.streams))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_one_device_film(tmp_path):
    total = 11
    one = FakeContext()
    one.run_pass(total)
    expect = one.sums / one.samples[..., None]
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, total, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    m0, m1 = np.load(tmp_path / "mean0.npy"), np.load(tmp_path / "mean1.npy")
    s0, s1 = np.load(tmp_path / "streams0.npy"), np.load(tmp_path / "streams1.npy")
    assert list(s0) + list(s1) == list(range(total))
    assert np.array_equal(m0, m1)
    assert np.allclose(m0, expect, rtol=1e-13, atol=1e-13)


class FakeAdjointContext:
    """The adjoint calls of distributed.walk_gradient / path_gradient on a known function: the
    gradient of a block of walks or samples is the mean over them of a per-index vector, as the
    library normalises by the walks (samples) of its own call."""

    _hf_n = 9

    @staticmethod
    def _g(k):
        return np.sin(0.3 * k + np.arange(9))

    def walk_adjoint(self, desc, first, n, g):
        return sum(self._g(k) for k in range(first, first + n)) / n * float(np.sum(g))

    def path_adjoint(self, first_pass, spp, g):
        return sum(self._g(k) for k in range(first_pass, first_pass + spp)) / spp * float(np.sum(g))


def _grad_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        c = FakeAdjointContext()
        g = np.full(4, 0.5)
        np.save(os.path.join(out, f"walk{rank}.npy"), D.walk_gradient(c, None, 13, g))
        np.save(os.path.join(out, f"path{rank}.npy"), D.path_gradient(c, 7, g, first_pass=3))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_one_device_gradient(tmp_path):
    c = FakeAdjointContext()
    g = np.full(4, 0.5)
    walk1 = c.walk_adjoint(None, 0, 13, g)
    path1 = c.path_adjoint(3, 7, g)
    port = _free_port()
    mp.start_processes(_grad_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for name, one in (("walk", walk1), ("path", path1)):
        a, b = np.load(tmp_path / f"{name}0.npy"), np.load(tmp_path / f"{name}1.npy")
        assert np.array_equal(a, b)
        assert np.allclose(a, one, rtol=1e-13, atol=1e-13)
