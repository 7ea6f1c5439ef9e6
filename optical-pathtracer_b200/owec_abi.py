"""ctypes mirror of include/owec.h: the scene description structs and the loader of the CUDA
library (csrc -> owe_cuda/libowec.so).

The structs are byte-for-byte the C structs, so one description feeds the CUDA backend, the CPU
restatement in oracle/ and the reference engine's own driver alike.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libowec.so")

ABI_VERSION = 5

OK = 0
E_INVALID, E_CUDA, E_NOMEM, E_STATE, E_DEVICE_FAULT, E_UNSUPPORTED = -1, -2, -3, -4, -5, -6

SPEC_CONSTANT, SPEC_TABULATED, SPEC_BLACKBODY = 0, 1, 2
INDEX_CONSTANT, INDEX_CAUCHY, INDEX_SELLMEIER, INDEX_CIDDOR, INDEX_TABULATED = 0, 1, 2, 3, 4
SURF_NULL, SURF_DIELECTRIC, SURF_DIFFUSE, SURF_CONDUCTOR, SURF_MIRROR, SURF_ABSORBER, SURF_DETECTOR = range(7)
SHAPE_SPHERE, SHAPE_SAG, SHAPE_PLANE, SHAPE_CYLINDER, SHAPE_MESH, SHAPE_CONE, SHAPE_TORUS, SHAPE_ROUND_WALL, \
    SHAPE_DOME, SHAPE_WAVES = range(10)
APERTURE_DISK, APERTURE_RECT, APERTURE_ELLIPSE, APERTURE_DISK_HOLE = 0, 1, 2, 3
SKY_NONE, SKY_UNIFORM, SKY_GRADIENT = 0, 1, 2
DETECTOR_OBSERVER, DETECTOR_SENSOR = 0, 1
WAVELENGTHS_HERO4, WAVELENGTHS_UNIFORM1 = 0, 1
PRECISION_MIXED, PRECISION_FP32, PRECISION_FP64 = 0, 1, 2
ADJOINT_FIXED_DECISIONS = 1
REGION_OUTSIDE = 0xFFFFFFFF
KNONE = 0xFFFFFFFE  # the reference's kNone: "no boundary"

c_double_p = ctypes.POINTER(ctypes.c_double)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_float_p = ctypes.POINTER(ctypes.c_float)


class Spectrum(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("table_offset", ctypes.c_int32), ("table_count", ctypes.c_int32),
                ("pad0", ctypes.c_int32), ("a", ctypes.c_double), ("scale", ctypes.c_double)]


class Medium(ctypes.Structure):
    _fields_ = [("index_kind", ctypes.c_int32), ("n_terms", ctypes.c_int32), ("rel_air", ctypes.c_int32),
                ("opaque", ctypes.c_int32), ("coef_a", ctypes.c_double * 4), ("coef_b", ctypes.c_double * 4),
                ("absorption", ctypes.c_int32), ("scattering", ctypes.c_int32), ("index_table", ctypes.c_int32),
                ("pad0", ctypes.c_int32), ("g", ctypes.c_double)]


class Optics(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("back_absorbs", ctypes.c_int32), ("reflectance", ctypes.c_int32),
                ("conductor_n", ctypes.c_int32), ("conductor_k", ctypes.c_int32), ("texture", ctypes.c_int32),
                ("roughness", ctypes.c_double), ("texture_b", ctypes.c_int32), ("texture_c", ctypes.c_int32),
                ("texture_scale", ctypes.c_double), ("texture_param", ctypes.c_double),
                ("aim_center", ctypes.c_double * 3), ("aim_normal", ctypes.c_double * 3), ("aim_radius", ctypes.c_double),
                ("aim_share", ctypes.c_double)]


TEXTURE_NONE, TEXTURE_CHECKER, TEXTURE_NOISE, TEXTURE_RINGS, TEXTURE_TERRAIN, TEXTURE_BANDS, TEXTURE_RADIAL, \
    TEXTURE_MARBLE = range(8)


class Emission(ctypes.Structure):
    _fields_ = [("radiance", ctypes.c_int32), ("front", ctypes.c_int32), ("back", ctypes.c_int32),
                ("nee", ctypes.c_int32), ("distant", ctypes.c_int32), ("pad0", ctypes.c_int32)]


class Boundary(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int32), ("mesh", ctypes.c_int32), ("front", ctypes.c_uint32),
                ("back", ctypes.c_uint32), ("optics", ctypes.c_uint32), ("emission", ctypes.c_int32),
                ("to_world", ctypes.c_double * 12), ("params", ctypes.c_double * 4),
                ("data_offset", ctypes.c_uint32), ("data_count", ctypes.c_uint32)]


class Mesh(ctypes.Structure):
    _fields_ = [("vertex_offset", ctypes.c_uint64), ("vertex_count", ctypes.c_uint64),
                ("tri_offset", ctypes.c_uint64), ("tri_count", ctypes.c_uint64)]


class Environment(ctypes.Structure):
    _fields_ = [("sky_model", ctypes.c_int32), ("sky_radiance", ctypes.c_int32), ("has_sun", ctypes.c_int32),
                ("sun_radiance", ctypes.c_int32), ("sun_dir", ctypes.c_double * 3),
                ("sun_angular_radius", ctypes.c_double), ("sun_nee_share", ctypes.c_double),
                ("sky_horizon", ctypes.c_int32), ("sky_ground", ctypes.c_int32), ("sky_up", ctypes.c_double * 3)]


class Detector(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("region", ctypes.c_uint32), ("position", ctypes.c_double * 3), ("look_at", ctypes.c_double * 3),
                ("up", ctypes.c_double * 3), ("fov_y", ctypes.c_double), ("pixel_sigma", ctypes.c_double),
                ("boundary", ctypes.c_uint32), ("pad0", ctypes.c_int32), ("half_x", ctypes.c_double),
                ("half_y", ctypes.c_double), ("pupil_radius", ctypes.c_double), ("focus_distance", ctypes.c_double),
                ("guide_center", ctypes.c_double * 3), ("guide_radius", ctypes.c_double),
                ("guide_share", ctypes.c_double), ("flip_x", ctypes.c_int32), ("flip_y", ctypes.c_int32),
                ("has_aim", ctypes.c_int32), ("pad1", ctypes.c_int32), ("aim_center", ctypes.c_double * 3),
                ("aim_normal", ctypes.c_double * 3), ("aim_radius", ctypes.c_double), ("aim_share", ctypes.c_double),
                ("focus_center", ctypes.c_double * 3), ("focus_radius", ctypes.c_double),
                ("focus_share", ctypes.c_double)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("abi_version", ctypes.c_uint32), ("n_spectra", ctypes.c_uint32), ("n_media", ctypes.c_uint32),
                ("n_regions", ctypes.c_uint32), ("n_optics", ctypes.c_uint32), ("n_emissions", ctypes.c_uint32),
                ("n_boundaries", ctypes.c_uint32), ("n_meshes", ctypes.c_uint32),
                ("n_spectrum_table", ctypes.c_uint64), ("n_vertices", ctypes.c_uint64),
                ("n_triangles", ctypes.c_uint64),
                ("spectra", ctypes.POINTER(Spectrum)), ("spectrum_table", c_double_p),
                ("media", ctypes.POINTER(Medium)), ("region_medium", c_u32_p),
                ("optics", ctypes.POINTER(Optics)), ("emissions", ctypes.POINTER(Emission)),
                ("boundaries", ctypes.POINTER(Boundary)), ("meshes", ctypes.POINTER(Mesh)),
                ("vertices", c_double_p), ("triangles", c_u32_p),
                ("env", Environment), ("detector", Detector),
                ("frame_origin_set", ctypes.c_int32), ("pad0", ctypes.c_int32),
                ("frame_origin", ctypes.c_double * 3),
                ("n_shape_data", ctypes.c_uint64), ("shape_data", c_double_p)]


class Settings(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("max_depth", ctypes.c_int32), ("rr_depth", ctypes.c_int32),
                ("wavelength_mode", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("lambda_min", ctypes.c_double), ("lambda_max", ctypes.c_double),
                ("fresnel_floor", ctypes.c_double), ("integrator", ctypes.c_int32), ("pad0", ctypes.c_int32)]


INTEGRATOR_PATH, INTEGRATOR_LIGHT = 0, 1
INTEGRATORS = {"path": INTEGRATOR_PATH, "light": INTEGRATOR_LIGHT}

SOURCE_POINT, SOURCE_COLLIMATED, SOURCE_COLLIMATED_SQUARE = 0, 1, 2
WALK_STOCHASTIC, WALK_PRIMARY_TRANSMISSION = 0, 1
SPLAT_NEAREST, SPLAT_BILINEAR = 0, 1


class WalkDesc(ctypes.Structure):
    _fields_ = [("source_kind", ctypes.c_int32), ("mode", ctypes.c_int32), ("max_events", ctypes.c_int32),
                ("splat", ctypes.c_int32), ("position", ctypes.c_double * 3), ("axis", ctypes.c_double * 3),
                ("extent", ctypes.c_double), ("lambda_min", ctypes.c_double), ("lambda_max", ctypes.c_double),
                ("region", ctypes.c_uint32), ("target", ctypes.c_uint32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("half_x", ctypes.c_double), ("half_y", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("stream", ctypes.c_uint64)]


class WalkStats(ctypes.Structure):
    _fields_ = [("walks", ctypes.c_uint64), ("binned", ctypes.c_uint64), ("escaped", ctypes.c_uint64),
                ("events", ctypes.c_uint64), ("faults", ctypes.c_uint64)]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class AdjointStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("heightfield", ctypes.c_uint64), ("dropped", ctypes.c_uint64),
                ("faults", ctypes.c_uint64), ("seconds", ctypes.c_double), ("device_bytes", ctypes.c_uint64),
                ("replay_seconds", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Stats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("segments", ctypes.c_uint64), ("inconsistencies", ctypes.c_uint64),
                ("leaks", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64), ("device_faults", ctypes.c_uint64)]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


def make_settings(seed=1, max_depth=64, rr_depth=6, wavelength_mode=WAVELENGTHS_HERO4,
                  precision=PRECISION_MIXED, lambda_min=380.0, lambda_max=780.0, fresnel_floor=0.0,
                  integrator=INTEGRATOR_PATH):
    """RenderSettings' transport fields (src/owe/scene/scene.hpp:15-49), reference defaults.
    `integrator` is INTEGRATOR_PATH or INTEGRATOR_LIGHT, or its name ("path", "light")."""
    if isinstance(integrator, str):
        if integrator not in INTEGRATORS:
            raise RuntimeError(f"unknown integrator '{integrator}' (expected {', '.join(INTEGRATORS)})")
        integrator = INTEGRATORS[integrator]
    return Settings(seed, max_depth, rr_depth, wavelength_mode, precision, lambda_min, lambda_max, fresnel_floor,
                    integrator, 0)


_LIB = None


def load_library(path=LIB_PATH):
    """The CUDA backend's shared library. Raises when it is missing: there is no CPU fallback."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"the CUDA backend library {path} is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    sigs = {
        "owec_last_error": ([], ctypes.c_char_p),
        "owec_abi_version": ([], ctypes.c_int),
        "owec_open": ([ctypes.c_int, ctypes.POINTER(P)], ctypes.c_int),
        "owec_close": ([P], ctypes.c_int),
        "owec_device_name": ([P, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "owec_upload_scene": ([P, ctypes.POINTER(SceneDesc)], ctypes.c_int),
        "owec_build_bvh": ([P], ctypes.c_int),
        "owec_bvh_info": ([P, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "owec_set_settings": ([P, ctypes.POINTER(Settings)], ctypes.c_int),
        "owec_pass": ([P, ctypes.c_int], ctypes.c_int),
        "owec_resolve": ([P, c_double_p, c_double_p], ctypes.c_int),
        "owec_read_film": ([P, c_double_p, c_double_p], ctypes.c_int),
        "owec_read_film_device": ([P, P, P], ctypes.c_int),
        "owec_set_pass_index": ([P, ctypes.c_uint64], ctypes.c_int),
        "owec_reset_film": ([P], ctypes.c_int),
        "owec_read_stats": ([P, ctypes.POINTER(Stats)], ctypes.c_int),
        "owec_last_pass_timing": ([P, c_double_p], ctypes.c_int),
        "owec_cast_rays": ([P, ctypes.c_uint64, c_double_p, c_double_p, c_u32_p, c_u32_p, c_double_p],
                           ctypes.c_int),
        "owec_cast_rays_device": ([P, ctypes.c_uint64, P, P, P, P, P, c_double_p], ctypes.c_int),
        "owec_scene_origin": ([P, c_double_p], ctypes.c_int),
        "owec_trace_counters": ([P, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "owec_trace_launch_queries": ([P, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
                                      ctypes.c_int),
        "owec_inconsistency_log": ([P, ctypes.c_int], ctypes.c_int),
        "owec_resolve_async": ([P, c_double_p, c_double_p], ctypes.c_int),
        "owec_resolve_wait": ([P], ctypes.c_int),
        "owec_read_inconsistency_log": ([P, c_double_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "owec_walk": ([P, ctypes.POINTER(WalkDesc), ctypes.c_uint64, ctypes.c_uint64], ctypes.c_int),
        "owec_walk_resolve": ([P, c_double_p, ctypes.POINTER(WalkStats)], ctypes.c_int),
        "owec_walk_reset": ([P], ctypes.c_int),
        "owec_set_heightfield": ([P, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, c_double_p], ctypes.c_int),
        "owec_walk_adjoint": ([P, ctypes.POINTER(WalkDesc), ctypes.c_uint64, ctypes.c_uint64, c_double_p, c_double_p],
                              ctypes.c_int),
        "owec_walk_adjoint_noalloc": ([P, ctypes.POINTER(WalkDesc), ctypes.c_uint64, ctypes.c_uint64, c_double_p,
                                       c_double_p], ctypes.c_int),
        "owec_walk_timing": ([P, c_double_p], ctypes.c_int),
        "owec_device_peaks": ([P, c_double_p], ctypes.c_int),
        "owec_path_adjoint": ([P, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p, c_double_p,
                               ctypes.POINTER(AdjointStats)], ctypes.c_int),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.owec_abi_version() != ABI_VERSION:
        raise RuntimeError("libowec.so ABI version mismatch")
    _LIB = lib
    return lib


def declared_symbols(header=None):
    """Every function declared in include/*.h (for the export check)."""
    import glob
    import re
    root = os.path.dirname(HERE)
    names = []
    for h in sorted(glob.glob(os.path.join(root, "include", "*.h"))) if header is None else [header]:
        text = open(h).read()
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(owec_\w+)\s*\(", text, re.M)
    return sorted(set(names))
