"""GPU parity for the optics no configuration uses: Cauchy and tabulated index models, smooth and
rough conductors (n + ik), the rough GGX dielectric, and null boundaries with a scattering medium
behind them, whose next-event shadow rays take the ordered walk (kShadow) through them. Each against
the reference engine's own FP64 transport on the same scene: the per-path agreement of one-sample
passes (both draw the same random numbers), one material at a time filling the view, and
compareRenderers' block z-test over independent seeds, for each precision instantiation."""
import numpy as np
import pytest

import owec_abi as A
import owe_cuda
import scenes
from conftest import save_artifact
from oracle_ref import ReferenceEngine, block_z_test

pytestmark = pytest.mark.gpu


def _settings(seed, precision=A.PRECISION_MIXED):
    return A.make_settings(seed=seed, max_depth=12, rr_depth=5, wavelength_mode=A.WAVELENGTHS_HERO4,
                           precision=precision)


@pytest.mark.parametrize("material", scenes.GALLERY)
def test_one_sample_paths_through_each_material(material):
    """One material filling the view: its one-sample paths against the reference's."""
    desc = scenes.materials_gallery(48, 48, fog_box=False, objects=(material,)).desc()
    ref = ReferenceEngine(desc)
    s = _settings(3)
    img_ref, _ = ref.render(s, 1, passes=1)
    with owe_cuda.Context() as c:
        c.set_settings(s)
        c.upload(desc)
        c.build_bvh()
        c.run_pass(1)
        img = c.resolve()[0]
        assert c.stats()["device_faults"] == 0
    save_artifact(f"material_{material}", ref=img_ref, gpu=img)
    a, b = img_ref[:, :, 1].ravel(), img[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.95, f"{material}: only {close.mean():.3f} of paths agree"


@pytest.mark.parametrize("fog_box", [False, True])
def test_one_sample_paths_follow_the_reference(fog_box):
    desc = scenes.materials_gallery(64, 48, fog_box=fog_box).desc()
    ref = ReferenceEngine(desc)
    s = _settings(3)
    img_ref, st_ref = ref.render(s, 1, passes=1)
    with owe_cuda.Context() as c:
        c.set_settings(s)
        c.upload(desc)
        c.build_bvh()
        c.run_pass(1)
        img = c.resolve()[0]
        st = c.stats()
    save_artifact(f"gallery_one_sample_{fog_box}", ref=img_ref, gpu=img)
    a, b = img_ref[:, :, 1].ravel(), img[:, :, 1].ravel()
    close = np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), 1e-3)
    assert close.mean() > 0.95, f"only {close.mean():.3f} of paths agree"
    assert st["device_faults"] == 0 and st["leaks"] == 0 and st_ref["leaks"] == 0
    if fog_box:
        assert st["shadow_rays"] > 0


@pytest.mark.parametrize("precision", [A.PRECISION_MIXED, A.PRECISION_FP64, A.PRECISION_FP32])
@pytest.mark.parametrize("fog_box", [False, True])
def test_gallery_agrees_with_reference_statistically(fog_box, precision):
    desc = scenes.materials_gallery(48, 36, fog_box=fog_box).desc()
    ref = ReferenceEngine(desc)
    runs_ref, runs_gpu = [], []
    with owe_cuda.Context() as c:
        c.upload(desc)
        c.build_bvh()
        for k in range(8):
            img, _ = ref.render(_settings(100 + k), 1, passes=32, first_pass=0)
            runs_ref.append(img)
            c.set_settings(_settings(200 + k, precision))
            c.reset_film()
            c.run_pass(32)
            runs_gpu.append(c.resolve()[0])
        st = c.stats()
    assert st["device_faults"] == 0
    # plain FP32 rounds every origin to FP32, which now and then puts a path on the wrong side of a
    # sphere: a leak; the product's modes must have none
    assert st["leaks"] <= (1e-4 * st["paths"] if precision == A.PRECISION_FP32 else 0), st
    save_artifact(f"gallery_runs_{fog_box}_{precision}", ref=np.array(runs_ref), gpu=np.array(runs_gpu))
    ok, rep = block_z_test(runs_ref, runs_gpu)
    assert ok, rep
