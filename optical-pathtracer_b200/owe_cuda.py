"""The engine's `cuda` backend seen from Python: Backend / Renderer over the C ABI (include/owec.h).

Mirrors the reference's rendering interface (src/owe/render/backend.hpp:31-52,
src/owe/render/renderer.hpp:19-79) name for name: a Backend reports its name, summary, availability,
devices and integrators and creates Renderers; a Renderer runs passes (run_pass), resolves the image,
keeps pass / sample / time counts and transport statistics. Errors raise RuntimeError, as the
reference throws std::runtime_error. There is no CPU fallback: without the CUDA library or a device,
creating a renderer raises.
"""
import ctypes
import time

import numpy as np

import owec_abi as A


def _check(lib, status, what):
    if status != A.OK:
        raise RuntimeError(f"{what}: {lib.owec_last_error().decode()} (status {status})")


class Context:
    """One device context: a scene on the device, its BVH, settings and film."""

    def __init__(self, device=-1):
        self.lib = A.load_library()
        self.handle = ctypes.c_void_p()
        _check(self.lib, self.lib.owec_open(device, ctypes.byref(self.handle)), "owec_open")

    def close(self):
        if self.handle:
            self.lib.owec_close(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def device_name(self):
        buf = ctypes.create_string_buffer(256)
        _check(self.lib, self.lib.owec_device_name(self.handle, buf, 256), "owec_device_name")
        return buf.value.decode()

    def upload(self, desc):
        self._desc = desc  # the pointed-to arrays must outlive the call only; kept for inspection
        _check(self.lib, self.lib.owec_upload_scene(self.handle, ctypes.byref(desc)), "owec_upload_scene")
        self.width, self.height = desc.detector.width, desc.detector.height
        for stale in ("_hf_n", "_hf_heights", "_hf_boundary"):  # a new scene has no heightfield yet
            self.__dict__.pop(stale, None)

    def build_bvh(self):
        _check(self.lib, self.lib.owec_build_bvh(self.handle), "owec_build_bvh")

    def bvh_info(self):
        info = (ctypes.c_uint64 * 6)()
        _check(self.lib, self.lib.owec_bvh_info(self.handle, info), "owec_bvh_info")
        keys = ("nodes", "prims", "triangles", "node_bytes", "prim_bytes", "analytic")
        return dict(zip(keys, [int(v) for v in info]))

    def set_settings(self, settings):
        _check(self.lib, self.lib.owec_set_settings(self.handle, ctypes.byref(settings)), "owec_set_settings")

    def run_pass(self, spp):
        _check(self.lib, self.lib.owec_pass(self.handle, int(spp)), "owec_pass")

    def resolve(self, samples=True, out=None):
        """(per-pixel mean XYZ (height, width, 3), per-pixel sample counts or None). `out`: a
        C-contiguous float64 array of height x width x 3 values to write the image into (pinned
        host memory reads back fastest)."""
        if not hasattr(self, "width"):
            raise RuntimeError("owec_resolve: no scene uploaded")
        n = self.width * self.height
        if out is not None:
            if not (out.dtype == np.float64 and out.flags.c_contiguous and out.size == 3 * n):
                raise ValueError("resolve: out must be a C-contiguous float64 array of height x width x 3")
            xyz = out.reshape(-1)
        else:
            xyz = np.empty(3 * n)
        cnt = np.empty(n) if samples else None
        _check(self.lib, self.lib.owec_resolve(self.handle, xyz.ctypes.data_as(A.c_double_p),
                                               cnt.ctypes.data_as(A.c_double_p) if samples else None), "owec_resolve")
        return xyz.reshape(self.height, self.width, 3), (cnt.reshape(self.height, self.width) if samples else None)

    def resolve_async(self, out, samples=None):
        """Starts the resolve of the passes run so far into `out` (a C-contiguous float64 array of
        height x width x 3, page-locked for the copy to overlap later passes) and `samples` (height x
        width, or None) without waiting (owec_resolve_async); resolve_wait() waits for the copies.
        The arrays must stay alive until then."""
        n = self.width * self.height
        if not (out.dtype == np.float64 and out.flags.c_contiguous and out.size == 3 * n):
            raise ValueError("resolve_async: out must be a C-contiguous float64 array of height x width x 3")
        if samples is not None and not (samples.dtype == np.float64 and samples.flags.c_contiguous and samples.size == n):
            raise ValueError("resolve_async: samples must be a C-contiguous float64 array of height x width")
        _check(self.lib, self.lib.owec_resolve_async(self.handle, out.ctypes.data_as(A.c_double_p),
                                                     samples.ctypes.data_as(A.c_double_p) if samples is not None else None),
               "owec_resolve_async")

    def resolve_wait(self):
        _check(self.lib, self.lib.owec_resolve_wait(self.handle), "owec_resolve_wait")

    def read_film(self):
        """(compensated XYZ sums (height, width, 3), samples per pixel (height, width))."""
        n = self.width * self.height
        sums = np.empty(3 * n)
        cnt = np.empty(n)
        _check(self.lib, self.lib.owec_read_film(self.handle, sums.ctypes.data_as(A.c_double_p),
                                                 cnt.ctypes.data_as(A.c_double_p)), "owec_read_film")
        return sums.reshape(self.height, self.width, 3), cnt.reshape(self.height, self.width)

    def read_film_device(self, sums_ptr, samples_ptr):
        """owec_read_film_device: the film's XYZ sums (3 doubles per pixel) and samples per pixel
        into device buffers at the given addresses (0: skipped), e.g. torch CUDA tensors' data_ptr()."""
        _check(self.lib, self.lib.owec_read_film_device(self.handle, ctypes.c_void_p(sums_ptr or None),
                                                        ctypes.c_void_p(samples_ptr or None)), "owec_read_film_device")

    def set_pass_index(self, index):
        """The sample stream the next pass starts at."""
        _check(self.lib, self.lib.owec_set_pass_index(self.handle, int(index)), "owec_set_pass_index")

    def reset_film(self):
        _check(self.lib, self.lib.owec_reset_film(self.handle), "owec_reset_film")

    def stats(self):
        s = A.Stats()
        _check(self.lib, self.lib.owec_read_stats(self.handle, ctypes.byref(s)), "owec_read_stats")
        return s.as_dict()

    def last_pass_timing(self):
        """(pass seconds, intersect-kernel seconds, shadow-kernel seconds, intersect launches)."""
        out = (ctypes.c_double * 4)()
        _check(self.lib, self.lib.owec_last_pass_timing(self.handle, out), "owec_last_pass_timing")
        return out[0], out[1], out[2], int(out[3])

    def cast_rays(self, origins, directions):
        o = np.ascontiguousarray(origins, np.float64)
        d = np.ascontiguousarray(directions, np.float64)
        n = len(o)
        b = np.zeros(n, np.uint32)
        p = np.zeros(n, np.uint32)
        t = np.zeros(n, np.float64)
        _check(self.lib, self.lib.owec_cast_rays(self.handle, n, o.ctypes.data_as(A.c_double_p),
                                                 d.ctypes.data_as(A.c_double_p), b.ctypes.data_as(A.c_u32_p),
                                                 p.ctypes.data_as(A.c_u32_p), t.ctypes.data_as(A.c_double_p)),
               "owec_cast_rays")
        return b, p, t

    def trace_counters(self, enable):
        """[queries, nodes, prims, shadow queries, shadow nodes, shadow prims] counted since enabled."""
        out = (ctypes.c_uint64 * 6)()
        _check(self.lib, self.lib.owec_trace_counters(self.handle, int(enable), out), "owec_trace_counters")
        return [int(v) for v in out]

    def trace_launch_queries(self):
        """The closest-hit queries of each closest-hit launch of the passes run since counting was
        enabled (owec_trace_launch_queries), in launch order."""
        out = (ctypes.c_uint64 * 256)()
        n = ctypes.c_int()
        _check(self.lib, self.lib.owec_trace_launch_queries(self.handle, out, 256, ctypes.byref(n)),
               "owec_trace_launch_queries")
        return [int(out[k]) for k in range(min(256, n.value))]

    INCONSISTENCY_FIELDS = ("boundary", "prim", "flags", "region", "met", "dep_boundary", "dep_prim", "depth", "t",
                            "ox", "oy", "oz", "dx", "dy", "dz", "err_n")

    def inconsistency_log(self, capacity):
        """Record up to `capacity` crossings that meet a region other than the ray's (0 stops)."""
        _check(self.lib, self.lib.owec_inconsistency_log(self.handle, int(capacity)), "owec_inconsistency_log")
        self._event_cap = int(capacity)

    def read_inconsistency_log(self):
        """(records as an n x 16 array, fields INCONSISTENCY_FIELDS; crossings logged in all)."""
        cap = getattr(self, "_event_cap", 0)
        out = np.zeros((max(cap, 1), 16))
        n = ctypes.c_int()
        _check(self.lib, self.lib.owec_read_inconsistency_log(self.handle, out.ctypes.data_as(A.c_double_p), cap,
                                                              ctypes.byref(n)), "owec_read_inconsistency_log")
        return out[:min(cap, n.value)], n.value

    def walk(self, desc, first, n):
        """n forward light walks (walk indices first .. first + n - 1) binned on desc.target."""
        self._walk_shape = (desc.height, desc.width)
        _check(self.lib, self.lib.owec_walk(self.handle, ctypes.byref(desc), int(first), int(n)), "owec_walk")

    def walk_resolve(self):
        h, w = self._walk_shape
        bins = np.zeros(h * w)
        st = A.WalkStats()
        _check(self.lib, self.lib.owec_walk_resolve(self.handle, bins.ctypes.data_as(A.c_double_p), ctypes.byref(st)),
               "owec_walk_resolve")
        return bins.reshape(h, w), st.as_dict()

    def set_heightfield(self, boundary, base_z, heights):
        """Moves the vertices of mesh boundary `boundary` to z = base_z + heights (one per vertex)."""
        h = np.ascontiguousarray(heights, np.float64).ravel()
        _check(self.lib, self.lib.owec_set_heightfield(self.handle, boundary, len(h), base_z,
                                                       h.ctypes.data_as(A.c_double_p)), "owec_set_heightfield")
        self._hf_n = len(h)
        self._hf_heights = h.copy()
        self._hf_boundary = boundary

    def _adjoint_args(self, desc, g, dheights=None):
        """The loss gradient (one per walk bin) and the height-gradient accumulator (one per vertex)
        as contiguous float64 vectors, checked against the sizes the library will read and write."""
        if not hasattr(self, "_hf_n"):
            raise RuntimeError("no heightfield set (set_heightfield)")
        gg = np.ascontiguousarray(g, np.float64).ravel()
        if gg.size != desc.width * desc.height:
            raise ValueError(f"g has {gg.size} values; the walk film has {desc.width} x {desc.height} bins")
        if dheights is None:
            return gg, np.zeros(self._hf_n)
        out = np.ascontiguousarray(dheights, np.float64).ravel().copy()
        if out.size != self._hf_n:
            raise ValueError(f"dheights has {out.size} values; the heightfield has {self._hf_n} vertices")
        return gg, out

    def walk_adjoint(self, desc, first, n, g):
        """d(sum_b g_b bins_b) / d heights by path replay of walks first .. first + n - 1."""
        gg, out = self._adjoint_args(desc, g)
        _check(self.lib, self.lib.owec_walk_adjoint(self.handle, ctypes.byref(desc), int(first), int(n),
                                                    gg.ctypes.data_as(A.c_double_p), out.ctypes.data_as(A.c_double_p)),
               "owec_walk_adjoint")
        return out

    def walk_adjoint_noalloc(self, desc, first, n, g, dheights=None):
        """walk_adjoint through owec_walk_adjoint_noalloc, which allocates no device memory: its
        scratch is a fixed array in the library (at most 512 x 512 bins, 2^20 vertices). The
        gradient is added to `dheights` (zeros when not given) and returned."""
        gg, out = self._adjoint_args(desc, g, dheights)
        _check(self.lib, self.lib.owec_walk_adjoint_noalloc(self.handle, ctypes.byref(desc), int(first), int(n),
                                                            gg.ctypes.data_as(A.c_double_p),
                                                            out.ctypes.data_as(A.c_double_p)),
               "owec_walk_adjoint_noalloc")
        return out

    def path_adjoint(self, first_pass, spp, g, dheights=None, replay=False, with_stats=False, fixed_decisions=False):
        """d(sum_p g_p . film_p) / d heights by path replay of the camera paths of samples first_pass
        .. first_pass + spp - 1 (owec_path_adjoint). g: dLoss/dFilm, height x width x 3. Returns the
        gradient (added to `dheights` when given); with with_stats, (gradient, stats dict, replayed
        image or None). replay: every path replayed from its camera ray and the replayed image
        returned. fixed_decisions: the derivative at fixed random numbers (what central differences
        with common random numbers measure) instead of the gradient of the expected film."""
        if not hasattr(self, "_hf_n"):
            raise RuntimeError("no heightfield set (set_heightfield)")
        gg = np.ascontiguousarray(g, np.float64).ravel()
        if gg.size != 3 * self.width * self.height:
            raise ValueError(f"g has {gg.size} values; the film has {self.width} x {self.height} x 3")
        out = np.zeros(self._hf_n) if dheights is None else np.ascontiguousarray(dheights, np.float64).ravel().copy()
        if out.size != self._hf_n:
            raise ValueError(f"dheights has {out.size} values; the heightfield has {self._hf_n} vertices")
        rep = np.zeros(3 * self.width * self.height) if replay else None
        st = A.AdjointStats()
        flags = A.ADJOINT_FIXED_DECISIONS if fixed_decisions else 0
        _check(self.lib, self.lib.owec_path_adjoint(self.handle, int(first_pass), int(spp), flags, gg.ctypes.data_as(A.c_double_p),
                                                    out.ctypes.data_as(A.c_double_p),
                                                    rep.ctypes.data_as(A.c_double_p) if replay else None,
                                                    ctypes.byref(st)), "owec_path_adjoint")
        self._last_adjoint = st.as_dict()
        if not with_stats:
            return out
        return out, self._last_adjoint, (rep.reshape(self.height, self.width, 3) if replay else None)

    def last_path_adjoint_seconds(self):
        """Device seconds of the last path_adjoint call (both phases)."""
        return self._last_adjoint["seconds"]

    def device_peaks(self):
        """{"fp32_flops", "fp64_flops", "l2_read_bytes_per_s"}: the device's FMA rates and L2 read
        bandwidth, measured by owec_device_peaks."""
        out = (ctypes.c_double * 3)()
        _check(self.lib, self.lib.owec_device_peaks(self.handle, out), "owec_device_peaks")
        return {"fp32_flops": out[0], "fp64_flops": out[1], "l2_read_bytes_per_s": out[2]}

    def walk_timing(self):
        out = (ctypes.c_double * 2)()
        _check(self.lib, self.lib.owec_walk_timing(self.handle, out), "owec_walk_timing")
        return out[0], out[1]

    def walk_reset(self):
        _check(self.lib, self.lib.owec_walk_reset(self.handle), "owec_walk_reset")

    def scene_origin(self):
        o = (ctypes.c_double * 3)()
        _check(self.lib, self.lib.owec_scene_origin(self.handle, o), "owec_scene_origin")
        return np.array(list(o))


class Renderer:
    """A progressive estimator of one detector's image (owe::Renderer)."""

    def __init__(self, backend, desc, settings, integrator=None, device=-1):
        if integrator is None:  # RenderSettings::integrator
            names = {v: k for k, v in A.INTEGRATORS.items()}
            integrator = names.get(settings.integrator, str(settings.integrator))
        if integrator not in backend.integrators():
            known = ", ".join(backend.integrators())
            raise RuntimeError(f"unknown integrator '{integrator}' (expected {known})")
        self._backend = backend
        self.ctx = Context(device)
        self.ctx.upload(desc)
        self.ctx.build_bvh()
        # the integrator chosen by name, as RenderSettings::integrator (src/owe/scene/scene.hpp:19)
        settings = A.Settings.from_buffer_copy(settings)
        settings.integrator = A.INTEGRATORS[integrator]
        self.ctx.set_settings(settings)
        self.settings = settings
        self.integrator = integrator
        self._passes = 0
        self._spp = 0
        self._seconds = 0.0

    def run_pass(self, spp):
        """Adds a pass of `spp` samples per pixel (Renderer::runPass)."""
        if spp <= 0:
            return
        t0 = time.perf_counter()
        self.ctx.run_pass(spp)
        self._seconds += time.perf_counter() - t0
        self._passes += 1
        self._spp += spp

    def resolve(self, out=None):
        """Per-pixel mean XYZ, shape (height, width, 3) (Renderer::resolve), written into `out` when
        given."""
        return self.ctx.resolve(samples=False, out=out)[0]

    def resolve_async(self, out):
        """Renderer::resolve into `out` (page-locked, height x width x 3 float64) without waiting: the
        copy overlaps the passes run next; resolve_wait() waits for it."""
        self.ctx.resolve_async(out)

    def resolve_wait(self):
        self.ctx.resolve_wait()

    def passes(self):
        return self._passes

    def samples_per_pixel(self):
        return self._spp

    def seconds(self):
        return self._seconds

    def stats(self):
        return self.ctx.stats()

    def backend(self):
        name = self.ctx.device_name()
        mode = {A.PRECISION_MIXED: "float32 camera-relative + selective float64",
                A.PRECISION_FP32: "float32", A.PRECISION_FP64: "float64"}[self.settings.precision]
        kind = "wavefront" if self.integrator == "path" else "particles"
        return f"cuda: {name} (sm_100a {kind}; {mode})"

    def reset_observer(self):
        self.ctx.reset_film()
        self._passes = self._spp = 0
        self._seconds = 0.0
        return True

    def close(self):
        self.ctx.close()


class CudaBackend:
    """The `cuda` backend (owe::Backend)."""

    def name(self):
        return "cuda"

    def summary(self):
        return "NVIDIA B200 (sm_100a) wavefront path tracer; float32 camera-relative with selective float64"

    def available(self):
        try:
            c = Context()
            c.close()
            return True, ""
        except Exception as e:  # the reason, as Backend::available(why) reports it
            return False, str(e)

    def devices(self):
        ok, _ = self.available()
        if not ok:
            return []
        c = Context()
        try:
            return [{"index": 0, "name": c.device_name(), "type": "discrete", "driver": "CUDA"}]
        finally:
            c.close()

    def integrators(self):
        return ["path", "light"]

    def supports(self, integrator):
        return integrator in self.integrators()

    def create_renderer(self, desc, settings, integrator=None, device=-1):
        return Renderer(self, desc, settings, integrator, device)


def cuda_backend():
    return CudaBackend()
