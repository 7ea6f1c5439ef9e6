"""The CPU restatement (oracle/owe_oracle.cpp) against the golden vectors the reference engine
wrote (tests/golden/make_golden.py): World::intersect hits, a film of one-sample passes and
Tracer::walk bins. These pin the oracle without the reference being built."""
import os

import numpy as np
import pytest

import owec_abi as A
import scenes
from oracle_ref import PortEngine

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_ray_casts_equal_world_intersect_golden():
    g = _load("world_intersect_room64x32.npz")
    sb = scenes.bvh_stress_room(8, 8, n_lon=64, n_lat=32)
    b, p, t = PortEngine(sb.desc()).cast_rays(g["o"], g["d"])
    assert np.array_equal(b, g["boundary"]) and np.array_equal(p, g["prim"])
    hit = g["boundary"] != A.KNONE
    assert hit.mean() > 0.9
    assert np.allclose(t[hit], g["t"][hit], rtol=1e-12, atol=0)


def test_one_sample_film_equals_golden():
    g = _load("film_glass_sphere_16x16_4pass.npz")
    desc = scenes.glass_sphere_on_floor(16, 16).desc()
    s = A.make_settings(seed=int(g["seed"]), max_depth=int(g["max_depth"]), rr_depth=int(g["rr_depth"]),
                        wavelength_mode=A.WAVELENGTHS_UNIFORM1)
    xyz, st = PortEngine(desc).render(s, 1, passes=int(g["passes"]))
    assert st["paths"] == int(g["paths"])
    close = np.abs(xyz - g["xyz"]) <= 1e-9 * np.maximum(np.abs(g["xyz"]), 1e-12)
    assert close.mean() > 0.99


def test_walk_bins_equal_golden():
    g = _load("walk_achromat_32x32.npz")
    sb, info = scenes.achromat_scene(film=32, half_size=2.5e-4)
    w = scenes.achromat_walk(info, seed=int(g["seed"]), mode=A.WALK_PRIMARY_TRANSMISSION)
    bins, st = PortEngine(sb.desc()).walk(w, 0, int(g["walks"]))
    assert st["binned"] == int(g["binned"]) and st["escaped"] == int(g["escaped"])
    assert np.allclose(bins, g["bins"], rtol=1e-9, atol=1e-12 * np.abs(g["bins"]).max())
