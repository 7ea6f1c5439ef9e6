"""ctypes access to the oracle libraries under oracle/ (test infrastructure).

`ReferenceEngine` drives oracle/_ref/liboweref.so: the reference engine compiled from its own sources
with oracle/ref_driver.cpp, taking the same owec_scene_desc as the CUDA backend.
"""
import ctypes
import os

import numpy as np
import pytest

import owec_abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liboweref.so")

_ref = None


def ref_lib():
    """The reference engine, or a pytest skip when it was not built (no reference sources here)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            pytest.skip("oracle/_ref/liboweref.so is not built (the reference sources were absent)")
        lib = ctypes.CDLL(REF_LIB)
        P = ctypes.c_void_p
        lib.oweref_last_error.restype = ctypes.c_char_p
        lib.oweref_scene_create.restype = P
        lib.oweref_scene_create.argtypes = [ctypes.POINTER(A.SceneDesc)]
        lib.oweref_scene_destroy.argtypes = [P]
        lib.oweref_render.argtypes = [P, ctypes.POINTER(A.Settings), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, A.c_double_p, A.c_double_p,
                                      ctypes.POINTER(A.Stats)]
        lib.oweref_render_backend.argtypes = [P, ctypes.POINTER(A.Settings), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              A.c_double_p, ctypes.POINTER(A.Stats), A.c_double_p]
        lib.oweref_cast_rays.argtypes = [P, ctypes.c_uint64, A.c_double_p, A.c_double_p, ctypes.c_int, A.c_u32_p,
                                         A.c_u32_p, A.c_double_p]
        lib.oweref_scene_info.argtypes = [P, A.c_double_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), A.c_double_p,
                                          A.c_u32_p]
        lib.oweref_medium_index.argtypes = [P, ctypes.c_uint32, ctypes.c_double, A.c_double_p]
        lib.oweref_walk.argtypes = [P, ctypes.POINTER(A.WalkDesc), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                    A.c_double_p, ctypes.POINTER(ctypes.c_uint64)]
        lib.oweref_walk_in_box.argtypes = [P, ctypes.POINTER(A.WalkDesc), ctypes.c_uint64, ctypes.c_uint64, A.c_double_p,
                                           ctypes.c_int, A.c_double_p, ctypes.POINTER(ctypes.c_uint64)]
        lib.oweref_paraxial_image_distance.argtypes = [ctypes.c_int, A.c_double_p, A.c_double_p, A.c_double_p,
                                                       ctypes.c_double, ctypes.c_double, A.c_double_p]
        _ref = lib
    return _ref


class ReferenceEngine:
    """The reference's own FP64 transport on the same scene description."""

    def __init__(self, desc):
        self.lib = ref_lib()
        self.desc = desc
        self.h = self.lib.oweref_scene_create(ctypes.byref(desc))
        if not self.h:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        self.w, self.hgt = desc.detector.width, desc.detector.height

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oweref_scene_destroy(self.h)
            self.h = None

    def render(self, settings, spp, passes=1, first_pass=0, threads=0, pixel_begin=0, pixel_end=0):
        """Per-pixel means (height, width, 3) of `passes` passes of `spp` (the raw sums divided by
        the sample count) and the transport statistics."""
        n = self.w * self.hgt
        xyz = np.zeros(3 * n)
        samples = np.zeros(n)
        st = A.Stats()
        r = self.lib.oweref_render(self.h, ctypes.byref(settings), spp, passes, first_pass, threads, pixel_begin,
                                   pixel_end, xyz.ctypes.data_as(A.c_double_p), samples.ctypes.data_as(A.c_double_p),
                                   ctypes.byref(st))
        if r != 0:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        xyz = xyz.reshape(n, 3) / np.maximum(samples, 1)[:, None]
        return xyz.reshape(self.hgt, self.w, 3), st.as_dict()

    def render_backend(self, settings, spp, passes=1, threads=0):
        n = self.w * self.hgt
        xyz = np.zeros(3 * n)
        st = A.Stats()
        sec = ctypes.c_double()
        r = self.lib.oweref_render_backend(self.h, ctypes.byref(settings), spp, passes, threads,
                                           xyz.ctypes.data_as(A.c_double_p), ctypes.byref(st), ctypes.byref(sec))
        if r != 0:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        return xyz.reshape(self.hgt, self.w, 3), st.as_dict(), sec.value

    def cast_rays(self, o, d, threads=0):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        n = len(o)
        b = np.zeros(n, np.uint32)
        p = np.zeros(n, np.uint32)
        t = np.zeros(n)
        r = self.lib.oweref_cast_rays(self.h, n, o.ctypes.data_as(A.c_double_p), d.ctypes.data_as(A.c_double_p),
                                      threads, b.ctypes.data_as(A.c_u32_p), p.ctypes.data_as(A.c_u32_p),
                                      t.ctypes.data_as(A.c_double_p))
        if r != 0:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        return b, p, t

    def walk(self, desc, first, n, threads=0):
        """Tracer::walk for n walks, binned as owec_walk bins them; returns (bins normalised like
        owec_walk_resolve, stats)."""
        nb = desc.width * desc.height
        bins = np.zeros(nb)
        st = (ctypes.c_uint64 * 4)()
        r = self.lib.oweref_walk(self.h, ctypes.byref(desc), first, n, threads, bins.ctypes.data_as(A.c_double_p), st)
        if r != 0:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        return normalise_walk_bins(desc, bins, n), {"walks": st[0], "binned": st[1], "escaped": st[2],
                                                    "events": st[3]}

    def walk_in_box(self, desc, first, n, box, threads=0):
        """The walks of first .. first + n - 1 whose emission point lies in box (xmin, xmax, ymin,
        ymax, zmin, zmax, world coordinates): their binned throughput as raw sums (not normalised)
        and the number of them that ran."""
        nb = desc.width * desc.height
        bins = np.zeros(nb)
        st = (ctypes.c_uint64 * 4)()
        b = np.ascontiguousarray(box, np.float64)
        r = self.lib.oweref_walk_in_box(self.h, ctypes.byref(desc), first, n, b.ctypes.data_as(A.c_double_p), threads,
                                        bins.ctypes.data_as(A.c_double_p), st)
        if r != 0:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        return bins.reshape(desc.height, desc.width), int(st[0])

    def info(self):
        pdfs = np.zeros(64)
        n = ctypes.c_int()
        radius = ctypes.c_double()
        region = ctypes.c_uint32()
        r = self.lib.oweref_scene_info(self.h, pdfs.ctypes.data_as(A.c_double_p), 64, ctypes.byref(n),
                                       ctypes.byref(radius), ctypes.byref(region))
        if r != 0:
            raise RuntimeError(self.lib.oweref_last_error().decode())
        return {"light_pdfs": pdfs[: n.value].tolist(), "scene_radius": radius.value, "region": region.value}

    def index(self, region, lam):
        v = ctypes.c_double()
        self.lib.oweref_medium_index(self.h, region, lam, ctypes.byref(v))
        return v.value


def paraxial_image_distance(radii, thickness, glasses, object_distance, wavelength):
    """The reference's paraxialAnalysis: image distance behind the last vertex for spherical surfaces
    `radii` (m), `thickness` between them (m) and Sellmeier `glasses` ((B1, B2, B3), (C1, C2, C3))
    after each surface but the last, relative to air, in air."""
    lib = ref_lib()
    r = np.ascontiguousarray(radii, np.float64)
    t = np.ascontiguousarray(thickness, np.float64)
    c = np.ascontiguousarray([v for B, C in glasses for v in list(B) + list(C)], np.float64)
    out = ctypes.c_double()
    st = lib.oweref_paraxial_image_distance(len(r), r.ctypes.data_as(A.c_double_p), t.ctypes.data_as(A.c_double_p),
                                            c.ctypes.data_as(A.c_double_p), object_distance, wavelength, ctypes.byref(out))
    if st != 0:
        raise RuntimeError(lib.oweref_last_error().decode())
    return out.value


def normalise_walk_bins(desc, bins, n):
    """Binned throughput sums as irradiance per unit source intensity / irradiance, as
    owec_walk_resolve reports them: times (source measure) / (walks * bin area)."""
    if desc.source_kind == A.SOURCE_POINT:
        measure = 2 * np.pi * (1 - np.cos(desc.extent))
    elif desc.source_kind == A.SOURCE_COLLIMATED:
        measure = np.pi * desc.extent ** 2
    else:
        measure = 4 * desc.extent ** 2
    bin_area = (2 * desc.half_x / desc.width) * (2 * desc.half_y / desc.height)
    return (bins * measure / (n * bin_area)).reshape(desc.height, desc.width)


def block_z_test(runs_a, runs_b, block=6):
    """compareRenderers' statistics (src/owe/backends/compare.cpp:66-119): per-run block means of
    XYZ, z-scores of the two renderers' means over independent runs. Returns (consistent, report)."""
    def blocks(img):
        h, w, _ = img.shape
        by, bx = (h + block - 1) // block, (w + block - 1) // block
        out = np.zeros((by, bx, 3))
        cnt = np.zeros((by, bx, 1))
        yi = (np.arange(h) // block)[:, None]
        xi = (np.arange(w) // block)[None, :]
        cell = (yi * bx + xi).ravel()
        np.add.at(out.reshape(-1, 3), cell, img.reshape(-1, 3))
        np.add.at(cnt.reshape(-1, 1), cell, 1.0)
        return (out / np.maximum(cnt, 1)).ravel()

    def mean_se(xs):
        xs = np.asarray(xs)
        n = len(xs)
        m = xs.mean(0)
        se = np.sqrt(((xs - m) ** 2).sum(0) / (n - 1) / n)
        return m, se

    ba = np.array([blocks(r) for r in runs_a])
    bb = np.array([blocks(r) for r in runs_b])
    ia = np.array([r[:, :, 1].mean() for r in runs_a])
    ib = np.array([r[:, :, 1].mean() for r in runs_b])
    ma, sa = mean_se(ia)
    mb, sb = mean_se(ib)
    se = np.hypot(sa, sb)
    z_image = (mb - ma) / se if se > 0 else (0.0 if mb == ma else np.inf)
    mA, sA = mean_se(ba)
    mB, sB = mean_se(bb)
    s = np.hypot(sA, sB)
    ok = s > 0
    z = np.where(ok, (mB - mA) / np.where(ok, s, 1), 0.0)
    bad_zero = int(np.sum(~ok & (mA != mB)))
    tests = int(ok.sum()) + bad_zero
    over4 = int(np.sum(np.abs(z[ok]) > 4)) + bad_zero
    chi2 = float(np.sum(z[ok] ** 2) / max(1, tests))
    consistent = abs(z_image) < 4 and over4 <= max(1, tests // 100) and chi2 < 2
    report = {"meanA": float(ma), "meanB": float(mb), "seA": float(sa), "seB": float(sb), "zImage": float(z_image),
              "tests": tests, "over4": over4, "chi2PerTest": chi2, "maxAbsZ": float(np.max(np.abs(z))) if tests else 0}
    return consistent, report


PORT_LIB = os.path.join(ROOT, "oracle", "_build", "libowe_oracle.so")
_port = None


def port_lib():
    """The CPU restatement (oracle/owe_oracle.cpp), built by __graft_entry__.build()."""
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            raise RuntimeError("oracle/_build/libowe_oracle.so is not built (run __graft_entry__.build())")
        lib = ctypes.CDLL(PORT_LIB)
        P = ctypes.c_void_p
        lib.oweport_last_error.restype = ctypes.c_char_p
        lib.oweport_scene_create.restype = P
        lib.oweport_scene_create.argtypes = [ctypes.POINTER(A.SceneDesc)]
        lib.oweport_scene_destroy.argtypes = [P]
        lib.oweport_render.argtypes = lib_render_args = [P, ctypes.POINTER(A.Settings), ctypes.c_int, ctypes.c_int,
                                                          ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                                          A.c_double_p, A.c_double_p, ctypes.POINTER(A.Stats)]
        lib.oweport_cast_rays.argtypes = [P, ctypes.c_uint64, A.c_double_p, A.c_double_p, ctypes.c_int, A.c_u32_p,
                                          A.c_u32_p, A.c_double_p]
        lib.oweport_light_pdfs.argtypes = [P, A.c_double_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        lib.oweport_walk.argtypes = [P, ctypes.POINTER(A.WalkDesc), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                     A.c_double_p, ctypes.POINTER(ctypes.c_uint64)]
        _port = lib
    return _port


class PortEngine:
    """The oracle's own restatement of the reference transport, on the same scene description."""

    def __init__(self, desc):
        self.lib = port_lib()
        self.desc = desc
        self.h = self.lib.oweport_scene_create(ctypes.byref(desc))
        if not self.h:
            raise RuntimeError(self.lib.oweport_last_error().decode())
        self.w, self.hgt = desc.detector.width, desc.detector.height

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oweport_scene_destroy(self.h)
            self.h = None

    def render(self, settings, spp, passes=1, first_pass=0, threads=0, pixel_begin=0, pixel_end=0):
        n = self.w * self.hgt
        xyz = np.zeros(3 * n)
        samples = np.zeros(n)
        st = A.Stats()
        r = self.lib.oweport_render(self.h, ctypes.byref(settings), spp, passes, first_pass, threads, pixel_begin,
                                    pixel_end, xyz.ctypes.data_as(A.c_double_p), samples.ctypes.data_as(A.c_double_p),
                                    ctypes.byref(st))
        if r != 0:
            raise RuntimeError(self.lib.oweport_last_error().decode())
        xyz = xyz.reshape(n, 3) / np.maximum(samples, 1)[:, None]
        return xyz.reshape(self.hgt, self.w, 3), st.as_dict()

    def cast_rays(self, o, d, threads=0):
        o = np.ascontiguousarray(o, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        n = len(o)
        b = np.zeros(n, np.uint32)
        p = np.zeros(n, np.uint32)
        t = np.zeros(n)
        r = self.lib.oweport_cast_rays(self.h, n, o.ctypes.data_as(A.c_double_p), d.ctypes.data_as(A.c_double_p),
                                       threads, b.ctypes.data_as(A.c_u32_p), p.ctypes.data_as(A.c_u32_p),
                                       t.ctypes.data_as(A.c_double_p))
        if r != 0:
            raise RuntimeError(self.lib.oweport_last_error().decode())
        return b, p, t

    def walk(self, desc, first, n, threads=0):
        """The restated Tracer::walk, binned like owec_walk; (bins, stats)."""
        nb = desc.width * desc.height
        bins = np.zeros(nb)
        st = (ctypes.c_uint64 * 4)()
        r = self.lib.oweport_walk(self.h, ctypes.byref(desc), first, n, threads, bins.ctypes.data_as(A.c_double_p), st)
        if r != 0:
            raise RuntimeError(self.lib.oweport_last_error().decode())
        return normalise_walk_bins(desc, bins, n), {"walks": st[0], "binned": st[1], "escaped": st[2], "events": st[3]}

    def light_pdfs(self):
        out = np.zeros(64)
        n = ctypes.c_int()
        self.lib.oweport_light_pdfs(self.h, out.ctypes.data_as(A.c_double_p), 64, ctypes.byref(n))
        return out[: n.value].tolist()
