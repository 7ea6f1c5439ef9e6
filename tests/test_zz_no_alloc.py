"""owec_walk_adjoint_noalloc: the heightfield adjoint for callers that may not allocate device
memory while they run (an optimiser inside an application that fixed its GPU memory at start-up,
or one sharing the device with a framework whose allocator holds the free memory: for them a
cudaMalloc can fail and every cudaMalloc / cudaFree pair stalls the device). Its scratch is a
fixed array in the library; this file checks it against owec_walk_adjoint, which allocates its
scratch per call, on two calls in a row, and that it refuses sizes beyond that array.

Named to be collected last, so that a run stopping at its first failure has run the rest."""
import ctypes

import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes

pytestmark = pytest.mark.gpu

N = 32
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
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = 0
    return h


def _context():
    sb, info = scenes.caustic_slab_scene(n=N, heights=_heights(), wall_bins=BINS)
    c = owe_cuda.Context()
    c.upload(sb.desc())
    c.build_bvh()
    c.set_heightfield(info["heightfield"], info["thickness"], _heights())
    return c, info


def test_noalloc_adjoint_equals_the_allocating_one_on_two_calls():
    c, info = _context()
    with c:
        w = scenes.caustic_walk(info, seed=7)
        c.walk(w, 0, WALKS)
        bins, _ = c.walk_resolve()
        target = scenes.gaussian_blobs(BINS, count=16, seed=3, sigma_range=(2.0, 6.0)) * 0.4
        g = 2 * (bins.ravel() - target.ravel())
        ref = c.walk_adjoint(w, 0, WALKS, g)
        first = c.walk_adjoint_noalloc(w, 0, WALKS, g)
        # the second call finds the first call's contents in the shared scratch
        start = np.linspace(-1, 1, ref.size)
        second = c.walk_adjoint_noalloc(w, 0, WALKS, g, dheights=start)
    assert np.abs(ref).max() > 0
    # the same sums in another order of atomic additions
    tol = 1e-9 * np.abs(ref).max()
    assert np.allclose(first, ref, rtol=1e-9, atol=tol)
    assert np.allclose(second - start, ref, rtol=1e-9, atol=tol)


def test_noalloc_adjoint_refuses_a_film_beyond_its_scratch():
    c, info = _context()
    with c:
        w = scenes.caustic_walk(info, seed=7)
        w.width = w.height = 1024  # 2^20 bins: beyond the 512 x 512 the fixed scratch holds
        g = np.zeros(16)  # not read: the size check comes first
        out = np.zeros(N * N)
        st = c.lib.owec_walk_adjoint_noalloc(c.handle, ctypes.byref(w), 0, 1024, g.ctypes.data_as(A.c_double_p),
                                             out.ctypes.data_as(A.c_double_p))
        assert st == A.E_INVALID
        assert "512 x 512" in c.lib.owec_last_error().decode()
        assert not out.any()


def _noalloc_status(c, w, nh):
    g = np.zeros(w.width * w.height)
    out = np.zeros(nh)
    st = c.lib.owec_walk_adjoint_noalloc(c.handle, ctypes.byref(w), 0, 1024, g.ctypes.data_as(A.c_double_p),
                                         out.ctypes.data_as(A.c_double_p))
    return st, c.lib.owec_last_error().decode(), out


def test_noalloc_adjoint_refuses_when_the_fp64_primitives_were_not_built():
    # the BVH built under FP32 has no FP64 primitives; the mixed precision set afterwards would need
    # them, and preparing them allocates: the call must refuse instead
    sb, info = scenes.caustic_slab_scene(n=N, heights=_heights(), wall_bins=BINS)
    with owe_cuda.Context() as c:
        c.set_settings(A.make_settings(seed=0, precision=A.PRECISION_FP32))
        c.upload(sb.desc())
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["thickness"], _heights())
        c.set_settings(A.make_settings(seed=0, precision=A.PRECISION_MIXED))
        st, msg, out = _noalloc_status(c, scenes.caustic_walk(info, seed=7), N * N)
        assert st == A.E_STATE, msg
        assert "FP64 primitives" in msg
        assert not out.any()


def test_noalloc_adjoint_refuses_a_new_scene_without_its_heightfield_and_bvh():
    # uploading a scene discards the BVH and the heightfield of the previous one: building them
    # allocates, so the call refuses until the caller has done that set-up
    sb, info = scenes.caustic_slab_scene(n=N, heights=_heights(), wall_bins=BINS)
    with owe_cuda.Context() as c:
        c.upload(sb.desc())
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["thickness"], _heights())
        c.upload(sb.desc())
        st, msg, out = _noalloc_status(c, scenes.caustic_walk(info, seed=7), N * N)
        assert st == A.E_STATE, msg
        assert not out.any()
