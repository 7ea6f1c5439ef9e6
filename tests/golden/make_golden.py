"""Writes the golden vectors of tests/golden/ from the reference engine compiled from its own
sources (oracle/_ref/liboweref.so, built by oracle/Makefile where the reference sources are).

    python tests/golden/make_golden.py

Each file holds the inputs that are not regenerated from the scene builders (rays, settings) and
the reference's outputs: World::intersect hits, a film of one-sample passes (CpuRenderer::pass's
loop), Tracer::walk bins. tests/test_golden.py checks the CPU restatement (oracle/owe_oracle.cpp)
against them, so the oracle stays pinned where the reference cannot be built."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "optical-pathtracer_b200"), os.path.dirname(HERE)]

import owec_abi as A  # noqa: E402
import scenes  # noqa: E402
from oracle_ref import ReferenceEngine  # noqa: E402


def rays():
    sb = scenes.bvh_stress_room(8, 8, n_lon=64, n_lat=32)
    o, d = scenes.random_rays(4096, 77, (-2.8, -2.8, 0.1), (2.8, 2.8, 3.9), (-1.1, -1.1, 0.1), (1.1, 1.1, 2.3))
    b, p, t = ReferenceEngine(sb.desc()).cast_rays(o, d)
    np.savez_compressed(os.path.join(HERE, "world_intersect_room64x32.npz"), o=o, d=d, boundary=b, prim=p, t=t)


def film():
    desc = scenes.glass_sphere_on_floor(16, 16).desc()
    s = A.make_settings(seed=0, max_depth=16, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    xyz, st = ReferenceEngine(desc).render(s, 1, passes=4)
    np.savez_compressed(os.path.join(HERE, "film_glass_sphere_16x16_4pass.npz"), xyz=xyz, seed=0, max_depth=16,
                        rr_depth=4, passes=4, paths=st["paths"])


def walks():
    sb, info = scenes.achromat_scene(film=32, half_size=2.5e-4)
    w = scenes.achromat_walk(info, seed=5, mode=A.WALK_PRIMARY_TRANSMISSION)
    bins, st = ReferenceEngine(sb.desc()).walk(w, 0, 20_000)
    np.savez_compressed(os.path.join(HERE, "walk_achromat_32x32.npz"), bins=bins, walks=20_000, seed=5,
                        binned=st["binned"], escaped=st["escaped"], events=st["events"])


if __name__ == "__main__":
    rays()
    film()
    walks()
    print("golden vectors written to", HERE)
