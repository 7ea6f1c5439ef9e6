"""The multi-GPU render's device half on one GPU: two contexts that render the two stream blocks
of a split (owec_set_pass_index) and add their films (owec_read_film) give the one-context film."""
import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
import distributed as D

pytestmark = pytest.mark.gpu


def test_two_stream_blocks_add_up_to_one_render():
    desc = scenes.glass_sphere_on_floor(24, 24).desc()
    s = A.make_settings(seed=9, max_depth=16, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    total = 7
    with owe_cuda.Context() as one:
        one.upload(desc)
        one.build_bvh()
        one.set_settings(s)
        one.run_pass(total)
        ref_sums, ref_n = one.read_film()
        ref_mean, _ = one.resolve()
    sums, n = np.zeros_like(ref_sums), np.zeros_like(ref_n)
    for rank in range(2):
        first, count = D.stream_block(total, 2, rank)
        with owe_cuda.Context() as c:
            c.upload(desc)
            c.build_bvh()
            c.set_settings(s)
            c.set_pass_index(first)
            c.run_pass(count)
            a, b = c.read_film()
            sums += a
            n += b
    assert np.array_equal(n, ref_n) and ref_n.max() == total
    assert np.allclose(sums, ref_sums, rtol=1e-12, atol=1e-12 * np.abs(ref_sums).max())
    mean = sums / n[..., None]
    assert np.allclose(mean, ref_mean, rtol=1e-12, atol=1e-12 * np.abs(ref_mean).max())
