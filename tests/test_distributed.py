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
