"""Scene descriptions for the CUDA backend: a small builder over include/owec.h's owec_scene_desc,
and the procedural workloads the backend is measured on.

The builder mirrors the reference's world model (Medium -> Region -> Boundary, src/owe/scene/world.hpp)
and its builders (buildSphere, buildSheet, buildMesh, buildLens; src/owe/scene/builders.hpp:26-114):
region 0 is the ambient region, filled with air (Ciddor), as World's constructor makes it
(src/owe/scene/world.cpp:165-170).
"""
import ctypes
import math

import numpy as np

import owec_abi as A


def _arr(ctype, values):
    values = list(values)
    return (ctype * max(1, len(values)))(*values)


def translate(x, y, z):
    m = np.eye(3, 4)
    m[:, 3] = (x, y, z)
    return m


def rotate_to(frm, to):
    """Rigid rotation taking unit `frm` to unit `to` (Transform::rotateTo, src/owe/core/math.hpp:130-138)."""
    frm = np.asarray(frm, float) / np.linalg.norm(frm)
    to = np.asarray(to, float) / np.linalg.norm(to)
    axis = np.cross(frm, to)
    s = np.linalg.norm(axis)
    c = float(np.dot(frm, to))
    if s < 1e-12:
        if c > 0:
            return np.eye(3)
        a = np.array([1.0, 0, 0]) if abs(to[0]) < 0.9 else np.array([0, 1.0, 0])
        a = a - to * np.dot(a, to)
        axis, angle = a / np.linalg.norm(a), math.pi
    else:
        axis, angle = axis / s, math.atan2(s, c)
    x, y, z = axis
    K = np.array([[0, -z, y], [z, 0, -x], [-y, x, 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * K @ K


_M64 = (1 << 64) - 1


class Pcg32:
    """O'Neill's PCG32 as the reference's Rng (src/owe/core/sampling.hpp:11-30,
    src/owe/core/shared/warps.hpp:24-30): a stream per (seed, stream id), 53-bit uniforms from two
    outputs."""

    def __init__(self, seed, stream):
        self.state, self.inc = 0, ((stream << 1) | 1) & _M64
        self.next_u32()
        self.state = (self.state + seed) & _M64
        self.next_u32()

    def next_u32(self):
        old = self.state
        self.state = (old * 6364136223846793005 + self.inc) & _M64
        x = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        r = old >> 59
        return ((x >> r) | (x << ((-r) & 31))) & 0xFFFFFFFF

    def uniform(self):
        a, b = self.next_u32() >> 5, self.next_u32() >> 6
        return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0)


def align_z(axis, up=(0.0, 1.0, 0.0)):
    """The rotation whose z column is `axis` and whose y column lies toward `up` (Transform::alignZ,
    src/owe/core/math.hpp:123-132)."""
    z = np.asarray(axis, float) / np.linalg.norm(axis)
    u = np.asarray(up, float)
    if abs(np.dot(u / np.linalg.norm(u), z)) > 0.999:
        u = np.array([1.0, 0, 0]) if abs(z[0]) < 0.9 else np.array([0, 0, 1.0])
    x = np.cross(u, z)
    x /= np.linalg.norm(x)
    return np.column_stack([x, np.cross(z, x), z])


def wave_nodes(half_x, half_y, waves, spacing=-1.0):
    """The node counts of a wave surface (WaveSurface's constructor, src/owe/scene/geometry.cpp:190-207):
    (0, 0), the analytic sum, for spacing 0 or, by default, for up to six waves; otherwise nodes about
    `spacing` apart (by default a twelfth of the shortest wavelength), 2 to 4096 per axis."""
    k_max = max((math.hypot(w[1], w[2]) for w in waves), default=0.0)
    if spacing < 0:
        spacing = 0.0 if len(waves) <= 6 or k_max == 0 else (2 * math.pi / k_max) / 12
    if not spacing > 0:
        return 0, 0
    return (min(max(math.ceil(2 * half_x / spacing) + 1, 2), 4096), min(max(math.ceil(2 * half_y / spacing) + 1, 2), 4096))


def plane_wave(amplitude, wavelength, direction=0.0, phase=0.0):
    """(amplitude, kx, ky, phase) of a wave(...) in a waves body (Loader::wavesBody,
    src/owe/loader/loader_bodies.cpp:357-366)."""
    k = 2 * math.pi / wavelength
    return (amplitude, k * math.cos(direction), k * math.sin(direction), phase)


def ripple_field(count, seed, min_wavelength, max_wavelength, slope=0.1, direction=0.0, spread=math.radians(90)):
    """rippleField (src/owe/scene/builders.cpp:445-461): `count` waves with log-uniform wavelengths,
    directions spread about `direction` and amplitudes slope / (k sqrt(count)), drawn from the
    reference's PCG32 stream (seed, 0x7269707063)."""
    rng = Pcg32(seed, 0x7269707063)
    waves = []
    for _ in range(count):
        u1, u2, u3 = rng.uniform(), rng.uniform(), rng.uniform()
        lam = min_wavelength * (max_wavelength / min_wavelength) ** u1
        k = 2 * math.pi / lam
        theta = direction + (u2 - 0.5) * spread
        waves.append((slope / (k * math.sqrt(count)), k * math.cos(theta), k * math.sin(theta), 2 * math.pi * u3))
    return waves


def pose(R=None, t=(0, 0, 0)):
    m = np.zeros((3, 4))
    m[:, :3] = np.eye(3) if R is None else R
    m[:, 3] = t
    return m


class SceneBuilder:
    """Accumulates a world and produces the owec_scene_desc that describes it."""

    def __init__(self):
        self.spectra, self.table = [], []
        self.media, self.region_medium = [], []
        self.optics, self.emissions, self.boundaries, self.meshes = [], [], [], []
        self.vertices, self.triangles = [], []
        self.n_vertices = self.n_triangles = 0
        self.shape_data = []
        self.env = A.Environment(A.SKY_NONE, -1, 0, -1, (0, 0, 1), math.radians(0.2665), 0.0)
        self.detector = None
        air = self.medium_ciddor_air()
        self.region_medium.append(air)  # region 0: the ambient region

    # ---------------------------------------------------------- spectra and media
    def spectrum_constant(self, v):
        self.spectra.append(A.Spectrum(A.SPEC_CONSTANT, 0, 0, 0, float(v), 1.0))
        return len(self.spectra) - 1

    def spectrum_tabulated(self, lambdas, values, scale=1.0):
        off = len(self.table) // 2
        for l, v in zip(lambdas, values):
            self.table += [float(l), float(v)]
        self.spectra.append(A.Spectrum(A.SPEC_TABULATED, off, len(lambdas), 0, 0.0, float(scale)))
        return len(self.spectra) - 1

    def spectrum_blackbody(self, kelvin, scale):
        self.spectra.append(A.Spectrum(A.SPEC_BLACKBODY, 0, 0, 0, float(kelvin), float(scale)))
        return len(self.spectra) - 1

    def _medium(self, kind, a=(), b=(), rel_air=False, absorption=-1, scattering=-1, g=0.0, opaque=False,
                index_table=-1):
        ca = list(a) + [0.0] * (4 - len(a))
        cb = list(b) + [0.0] * (4 - len(b))
        self.media.append(A.Medium(kind, len(a), int(rel_air), int(opaque), (ctypes.c_double * 4)(*ca),
                                   (ctypes.c_double * 4)(*cb), absorption, scattering, index_table, 0, float(g)))
        return len(self.media) - 1

    def medium_ciddor_air(self, **kw):
        return self._medium(A.INDEX_CIDDOR, **kw)

    def medium_constant(self, n, **kw):
        return self._medium(A.INDEX_CONSTANT, (n,), **kw)

    def medium_sellmeier(self, B, C, rel_air=False, **kw):
        return self._medium(A.INDEX_SELLMEIER, tuple(B), tuple(C), rel_air=rel_air, **kw)

    def medium_opaque(self):
        return self._medium(A.INDEX_CONSTANT, (1.0,), opaque=True)

    def region(self, medium):
        self.region_medium.append(medium)
        return len(self.region_medium) - 1

    # ---------------------------------------------------------- optics and emission
    def optics_(self, type_, reflectance=-1, roughness=0.0, back_absorbs=False, cond_n=-1, cond_k=-1):
        self.optics.append(A.Optics(type_, int(back_absorbs), reflectance, cond_n, cond_k, 0, float(roughness)))
        return len(self.optics) - 1

    def diffuse(self, albedo, **kw):
        return self.optics_(A.SURF_DIFFUSE, self.spectrum_constant(albedo), **kw)

    def textured(self, kind, a, b, c=0.9, scale=1.0, param=0.0, **kw):
        """A Lambertian surface whose albedo mixes the constants a, b, c by a procedural texture."""
        o = self.optics_(A.SURF_DIFFUSE, self.spectrum_constant(a), **kw)
        opt = self.optics[o]
        opt.texture, opt.texture_b, opt.texture_c = kind, self.spectrum_constant(b), self.spectrum_constant(c)
        opt.texture_scale, opt.texture_param = float(scale), float(param)
        return o

    def aim_guide(self, optics, center, normal, radius, share):
        """Guide a Lambertian surface's scattering: `share` of its directions toward the disk of
        `radius` at `center` facing `normal` (SurfaceOptics::sampleAim*)."""
        o = self.optics[optics]
        o.aim_center = (ctypes.c_double * 3)(*center)
        o.aim_normal = (ctypes.c_double * 3)(*normal)
        o.aim_radius, o.aim_share = float(radius), float(share)
        return optics

    def dielectric(self, roughness=0.0):
        return self.optics_(A.SURF_DIELECTRIC, roughness=roughness)

    def absorber(self):
        return self.optics_(A.SURF_ABSORBER)

    def emission(self, radiance, front=True, back=False, nee=True, distant=False):
        self.emissions.append(A.Emission(radiance, int(front), int(back), int(nee), int(distant), 0))
        return len(self.emissions) - 1

    # ---------------------------------------------------------- boundaries
    def boundary(self, shape, params, xf, front, back, optics, emission=-1, mesh=-1, data=()):
        """A boundary; `data`: the shape's run of shape data (asphere terms, a torus arc's end,
        wall openings, a hole's centre)."""
        xf = np.asarray(xf, float).reshape(3, 4)
        p = list(params) + [0.0] * (4 - len(params))
        offset = len(self.shape_data)
        self.shape_data += [float(v) for v in data]
        self.boundaries.append(A.Boundary(shape, mesh, front, back, optics, emission,
                                          (ctypes.c_double * 12)(*xf.ravel()), (ctypes.c_double * 4)(*p),
                                          offset, len(data)))
        return len(self.boundaries) - 1

    def wave_surface(self, half_x, half_y, margin, waves, xf, front, back, optics, spacing=-1.0):
        """A WaveSurface boundary: waves as (amplitude, kx, ky, phase); sampled at nodes as the
        reference samples it (wave_nodes)."""
        nx, ny = wave_nodes(half_x, half_y, waves, spacing)
        data = [nx, ny] + [float(v) for w in waves for v in w]
        return self.boundary(A.SHAPE_WAVES, [half_x, half_y, margin], xf, front, back, optics, data=data)

    def water_pool(self, half_x, half_y, depth, margin, waves, medium, spacing=-1.0, bottom=None, walls=None, rim=None,
                   base=None):
        """buildWater (src/owe/scene/builders.cpp:402-443): a liquid region under a wave surface, closed by
        a floor and four walls facing the liquid. Without `bottom` and `walls` (optics) those are smooth
        dielectric interfaces to the ambient region; with them they are that matter, the basin an
        opaque region cut into a block whose rim (default a quarter of the larger half size wide),
        outer sides and underside (`base`, default a quarter of the depth, below the floor) face the
        air. Returns the liquid's region."""
        liquid = self.region(medium)
        iface = self.dielectric()
        basin = self.region(self.medium_opaque()) if bottom is not None or walls is not None else 0
        self.wave_surface(half_x, half_y, margin, waves, pose(), 0, liquid, iface, spacing)
        side = (lambda o: (basin, o) if o is not None else (0, iface))
        floor_back, floor_optics = side(bottom)
        self.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, half_x, half_y], translate(0.0, 0.0, -depth), liquid, floor_back,
                      floor_optics)
        wall_back, wall_optics = side(walls)
        hz = depth / 2
        for at, inward, half in (((half_x, 0.0, -hz), (-1, 0, 0), half_y), ((-half_x, 0.0, -hz), (1, 0, 0), half_y),
                                 ((0.0, half_y, -hz), (0, -1, 0), half_x), ((0.0, -half_y, -hz), (0, 1, 0), half_x)):
            self.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, half, hz], pose(align_z(inward, (0, 0, 1)), at), liquid,
                          wall_back, wall_optics)
        if basin:
            ground = walls if walls is not None else bottom
            rim = 0.25 * max(half_x, half_y) if rim is None else rim
            base = 0.25 * depth if base is None else base
            ox, oy, zb = half_x + rim, half_y + rim, -depth - base
            oz = -zb / 2
            for cx, cy, hx, hy in ((0.0, (oy + half_y) / 2, ox, (oy - half_y) / 2), (0.0, -(oy + half_y) / 2, ox, (oy - half_y) / 2),
                                   ((ox + half_x) / 2, 0.0, (ox - half_x) / 2, half_y),
                                   (-(ox + half_x) / 2, 0.0, (ox - half_x) / 2, half_y)):
                self.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, hx, hy], translate(cx, cy, 0.0), 0, basin, ground)
            for at, outward, half in (((ox, 0.0, zb / 2), (1, 0, 0), oy), ((-ox, 0.0, zb / 2), (-1, 0, 0), oy),
                                      ((0.0, oy, zb / 2), (0, 1, 0), ox), ((0.0, -oy, zb / 2), (0, -1, 0), ox)):
                self.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, half, oz], pose(align_z(outward, (0, 0, 1)), at), 0, basin,
                              ground)
            self.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, ox, oy], pose(align_z((0, 0, -1)), (0.0, 0.0, zb)), 0, basin,
                          ground)
        return liquid

    def medium_water(self):
        """The catalogue's water (src/owe/core/medium.cpp:136-142): Daimon and Masumura's Sellmeier
        index at 20 C, absorption after Pope and Fry (1/m)."""
        absorption = self.spectrum_tabulated([380, 400, 450, 500, 550, 600, 650, 700, 750, 800],
                                             [0.0114, 0.00663, 0.0092, 0.0204, 0.0565, 0.2224, 0.34, 0.65, 2.47, 2.07])
        return self.medium_sellmeier((5.684027565e-1, 1.726177391e-1, 2.086189578e-2, 1.130748688e-1),
                                     (5.101829712e-3, 1.821153936e-2, 2.620722293e-2, 1.069792721e1),
                                     absorption=absorption)

    def mesh(self, vertices, triangles):
        v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        self.meshes.append(A.Mesh(self.n_vertices, len(v), self.n_triangles, len(t)))
        self.vertices.append(v)
        self.triangles.append(t)
        self.n_vertices += len(v)
        self.n_triangles += len(t)
        return len(self.meshes) - 1

    def sphere_body(self, radius, center, interior_medium, optics, emission=-1):
        """buildSphere (src/owe/scene/builders.cpp:155-161): outside in front, interior behind."""
        inside = self.region(interior_medium)
        return self.boundary(A.SHAPE_SPHERE, [radius], translate(*center), 0, inside, optics, emission), inside

    def sheet(self, half_x, half_y, xf, optics, emission=-1, disk=False):
        """buildSheet: a two-sided plane with the ambient region on both sides."""
        if disk:
            return self.boundary(A.SHAPE_PLANE, [A.APERTURE_DISK, half_x, 0.0], xf, 0, 0, optics, emission)
        return self.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, half_x, half_y], xf, 0, 0, optics, emission)

    def mesh_body(self, vertices, triangles, interior_medium, optics, xf=None, emission=-1):
        """buildMesh (src/owe/scene/builders.cpp:174-181): a closed mesh, interior behind its faces."""
        inside = self.region(interior_medium)
        m = self.mesh(vertices, triangles)
        return self.boundary(A.SHAPE_MESH, [], pose() if xf is None else xf, 0, inside, optics, emission, m), inside

    # ---------------------------------------------------------- environment and detector
    def sun(self, direction, radiance, angular_radius=math.radians(0.2665), nee_share=0.0):
        d = np.asarray(direction, float)
        d = d / np.linalg.norm(d)
        self.env.has_sun = 1
        self.env.sun_dir = (ctypes.c_double * 3)(*d)
        self.env.sun_radiance = self.spectrum_constant(radiance)
        self.env.sun_angular_radius = angular_radius
        self.env.sun_nee_share = nee_share

    def uniform_sky(self, radiance):
        self.env.sky_model = A.SKY_UNIFORM
        self.env.sky_radiance = self.spectrum_constant(radiance)

    def gradient_sky(self, zenith, horizon, ground, up=(0.0, 0.0, 1.0)):
        """Environment::sky's gradient: ground below the horizon, horizon blending into zenith above."""
        self.env.sky_model = A.SKY_GRADIENT
        self.env.sky_radiance = self.spectrum_constant(zenith)
        self.env.sky_horizon = self.spectrum_constant(horizon)
        self.env.sky_ground = self.spectrum_constant(ground)
        u = np.asarray(up, float)
        self.env.sky_up = (ctypes.c_double * 3)(*(u / np.linalg.norm(u)))

    def observer(self, width, height, position, look_at, up=(0, 0, 1), fov_y_deg=40.0, pixel_sigma=0.0, region=0,
                 pupil=0.0, focus=0.0, guide=None):
        """An IdealObserver; pupil > 0 makes it a thin lens focused at `focus` (0: at infinity);
        guide = (centre, radius, share) draws that share of the pupil samples from a disk."""
        d = A.Detector(A.DETECTOR_OBSERVER, width, height, region, (ctypes.c_double * 3)(*position),
                       (ctypes.c_double * 3)(*look_at), (ctypes.c_double * 3)(*up),
                       math.radians(fov_y_deg), float(pixel_sigma), 0, 0, 0.0, 0.0)
        d.pupil_radius, d.focus_distance = float(pupil), float(focus)
        if guide is not None:
            d.guide_center = (ctypes.c_double * 3)(*guide[0])
            d.guide_radius, d.guide_share = float(guide[1]), float(guide[2])
        self.detector = d

    def frame_origin(self, point):
        """Put the origin of the device's camera-relative FP32 frame at `point` (default: the
        observer's position)."""
        self.origin = tuple(float(x) for x in point)

    def sensor(self, width, height, boundary, half_x, half_y, pixel_sigma=0.0, flip=(False, False), aim=None,
               focus=None):
        """A SurfaceSensor; aim = (centre, normal, radius, share) samples that share of the directions
        toward a disk, focus = (centre, radius, share) a share of those toward a second disk."""
        d = A.Detector(A.DETECTOR_SENSOR, width, height, A.REGION_OUTSIDE, (ctypes.c_double * 3)(),
                       (ctypes.c_double * 3)(), (ctypes.c_double * 3)(), 0.0, float(pixel_sigma),
                       boundary, 0, float(half_x), float(half_y))
        d.flip_x, d.flip_y = int(flip[0]), int(flip[1])
        if aim is not None:
            d.has_aim = 1
            d.aim_center = (ctypes.c_double * 3)(*aim[0])
            n = np.asarray(aim[1], float)
            d.aim_normal = (ctypes.c_double * 3)(*(n / np.linalg.norm(n)))
            d.aim_radius, d.aim_share = float(aim[2]), float(aim[3])
            if focus is not None:
                d.focus_center = (ctypes.c_double * 3)(*focus[0])
                d.focus_radius, d.focus_share = float(focus[1]), float(focus[2])
        self.detector = d

    # ---------------------------------------------------------- the description
    def desc(self):
        """An owec_scene_desc; the arrays it points into live as long as the returned object."""
        if self.detector is None:
            raise ValueError("the scene needs a detector")
        verts = np.concatenate(self.vertices) if self.vertices else np.zeros((1, 3))
        tris = np.concatenate(self.triangles) if self.triangles else np.zeros((1, 3), np.uint32)
        verts = np.ascontiguousarray(verts, np.float64)
        tris = np.ascontiguousarray(tris, np.uint32)
        keep = {
            "spectra": _arr(A.Spectrum, self.spectra),
            "table": _arr(ctypes.c_double, self.table),
            "media": _arr(A.Medium, self.media),
            "regions": _arr(ctypes.c_uint32, self.region_medium),
            "optics": _arr(A.Optics, self.optics),
            "emissions": _arr(A.Emission, self.emissions),
            "boundaries": _arr(A.Boundary, self.boundaries),
            "meshes": _arr(A.Mesh, self.meshes),
            "verts": verts,
            "tris": tris,
            "shape_data": _arr(ctypes.c_double, self.shape_data),
        }
        d = A.SceneDesc()
        d.abi_version = A.ABI_VERSION
        if getattr(self, "origin", None) is not None:
            d.frame_origin_set = 1
            d.frame_origin = (ctypes.c_double * 3)(*self.origin)
        d.n_spectra, d.n_media, d.n_regions = len(self.spectra), len(self.media), len(self.region_medium)
        d.n_optics, d.n_emissions, d.n_boundaries = len(self.optics), len(self.emissions), len(self.boundaries)
        d.n_meshes, d.n_spectrum_table = len(self.meshes), len(self.table) // 2
        d.n_vertices, d.n_triangles = self.n_vertices, self.n_triangles
        d.spectra, d.spectrum_table = keep["spectra"], keep["table"]
        d.media, d.region_medium, d.optics = keep["media"], keep["regions"], keep["optics"]
        d.emissions, d.boundaries, d.meshes = keep["emissions"], keep["boundaries"], keep["meshes"]
        d.vertices = verts.ctypes.data_as(A.c_double_p)
        d.triangles = tris.ctypes.data_as(A.c_u32_p)
        d.env = self.env
        d.detector = self.detector
        d.n_shape_data = len(self.shape_data)
        d.shape_data = keep["shape_data"]
        d._keep = keep  # the pointed-to arrays live as long as the description
        return d


# ------------------------------------------------------------------ glasses
# Schott N-BK7, relative to air (src/owe/core/medium.cpp:119).
NBK7 = ((1.03961212, 0.231792344, 1.01046945), (0.00600069867, 0.0200179144, 103.560653))
# Schott N-SF5, relative to air.
SF5 = ((1.52481889, 0.187085527, 1.42729015), (0.011254756, 0.0588995392, 129.141675))
# PMMA, three-term Sellmeier (lambda in um).
PMMA = ((0.99654, 0.18964, 0.00411), (0.00787, 0.02191, 3.85727))


# ------------------------------------------------------------------ seeded noise
def _pcg_hash(x):
    """A 32-bit integer hash (PCG output permutation) used to seed lattice gradients."""
    x = (x.astype(np.uint64) * np.uint64(747796405) + np.uint64(2891336453)) & np.uint64(0xFFFFFFFF)
    shift = ((x >> np.uint64(28)) + np.uint64(4)) & np.uint64(31)
    word = (((x >> shift) ^ x) * np.uint64(277803737)) & np.uint64(0xFFFFFFFF)
    return ((word >> np.uint64(22)) ^ word) & np.uint64(0xFFFFFFFF)


def gradient_noise3(p, seed):
    """Seeded 3-D gradient noise (Perlin's construction: random unit gradients on the integer lattice,
    quintic fade, trilinear blend of the corner ramps). Values in about [-1, 1]."""
    p = np.asarray(p, np.float64)
    i0 = np.floor(p).astype(np.int64)
    f = p - i0
    w = f * f * f * (f * (f * 6 - 15) + 10)
    out = np.zeros(len(p))
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                c = i0 + np.array([dx, dy, dz])
                h = _pcg_hash((c[:, 0] * 73856093 ^ c[:, 1] * 19349663 ^ c[:, 2] * 83492791 ^ seed * 2654435761)
                              & 0xFFFFFFFF)
                # gradient: a direction from the hash (uniform on the sphere)
                u = (h & np.uint64(0xFFFF)).astype(np.float64) / 65535.0
                v = (h >> np.uint64(16)).astype(np.float64) / 65535.0
                z = 1 - 2 * u
                r = np.sqrt(np.maximum(0, 1 - z * z))
                phi = 2 * math.pi * v
                g = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
                d = f - np.array([dx, dy, dz])
                ramp = (g * d).sum(1)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += wx * wy * wz * ramp
    return out * 1.6


def uv_sphere(n_lon=1024, n_lat=512, radius=1.0, amplitude=0.05, frequency=4.0, seed=7):
    """A UV sphere of n_lon meridians and n_lat rings between its poles: n_lon * n_lat * 2 triangles
    (2^20 at 1024 x 512). Vertices are displaced radially by seeded gradient noise of amplitude
    `amplitude * radius`; faces are counter-clockwise seen from outside."""
    rings = n_lat
    j = np.arange(1, n_lat + 1)
    theta = math.pi * j / (n_lat + 1)
    phi = 2 * math.pi * np.arange(n_lon) / n_lon
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    ring = np.stack([st * np.cos(phi)[None, :], st * np.sin(phi)[None, :], np.broadcast_to(ct, (rings, n_lon))], -1)
    dirs = np.concatenate([np.array([[0, 0, 1.0]]), ring.reshape(-1, 3), np.array([[0, 0, -1.0]])])
    n = gradient_noise3(dirs * frequency, seed)
    n = np.clip(n, -1, 1)
    verts = dirs * (radius * (1 + amplitude * n))[:, None]
    north, south = 0, 1 + rings * n_lon
    idx = lambda r, c: 1 + r * n_lon + (c % n_lon)  # noqa: E731
    c = np.arange(n_lon)
    tris = [np.stack([np.full(n_lon, north), idx(0, c), idx(0, c + 1)], 1)]
    for r in range(rings - 1):
        a, b = idx(r, c), idx(r, c + 1)
        a2, b2 = idx(r + 1, c), idx(r + 1, c + 1)
        tris.append(np.stack([a, a2, b2], 1))
        tris.append(np.stack([a, b2, b], 1))
    tris.append(np.stack([np.full(n_lon, south), idx(rings - 1, c + 1), idx(rings - 1, c)], 1))
    tris = np.concatenate(tris).astype(np.uint32)
    return verts, tris


# ------------------------------------------------------------------ the workloads
def glass_sphere_on_floor(width=256, height=256, pixel_sigma=0.0, sun_radiance=1.0e4):
    """An N-BK7 sphere of radius 1 on a Lambertian floor (albedo 0.8) under the sun at 45 degrees
    elevation; pinhole camera. The small plain-method workload."""
    sb = SceneBuilder()
    bk7 = sb.medium_sellmeier(*NBK7, rel_air=True)
    sb.sphere_body(1.0, (0, 0, 1.0), bk7, sb.dielectric())
    sb.sheet(20.0, 20.0, pose(), sb.diffuse(0.8))
    el = math.radians(45.0)
    az = math.atan2(0.35, 0.94)  # the sun stands behind the camera's right shoulder
    sb.sun((math.sin(az) * math.cos(el), -math.cos(az) * math.cos(el), math.sin(el)), sun_radiance)
    sb.observer(width, height, (0.0, -5.5, 2.6), (0.0, 0.0, 0.8), fov_y_deg=40.0, pixel_sigma=pixel_sigma)
    return sb


def bvh_stress_room(width=1920, height=1080, n_lon=1024, n_lat=512, pixel_sigma=0.0):
    """A 2^20-triangle displaced UV sphere (radius 1, noise amplitude 5 %) inside a closed Lambertian
    box with one area light on the ceiling. The BVH-stress workload."""
    sb = SceneBuilder()
    opaque = sb.medium_opaque()
    verts, tris = uv_sphere(n_lon, n_lat)
    sb.mesh_body(verts, tris, opaque, sb.diffuse(0.6), xf=translate(0, 0, 1.2))
    wall = sb.diffuse(0.7)
    h = 3.0  # box [-3, 3] x [-3, 3] x [0, 4]: five walls facing in, floor at z = 0
    sb.sheet(h, h, pose(), wall)  # floor (front +z)
    sb.sheet(h, h, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0, 0, 4.0)), wall)  # ceiling
    sb.sheet(2.0, h, pose(rotate_to((0, 0, 1), (1, 0, 0)), (-h, 0, 2.0)), wall)
    sb.sheet(2.0, h, pose(rotate_to((0, 0, 1), (-1, 0, 0)), (h, 0, 2.0)), wall)
    sb.sheet(h, 2.0, pose(rotate_to((0, 0, 1), (0, -1, 0)), (0, h, 2.0)), wall)
    sb.sheet(h, 2.0, pose(rotate_to((0, 0, 1), (0, 1, 0)), (0, -h, 2.0)), wall)
    lamp = sb.emission(sb.spectrum_constant(8.0))
    sb.sheet(0.8, 0.8, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0.0, 0.0, 3.98)), sb.absorber(), emission=lamp)
    sb.observer(width, height, (0.3, -2.7, 1.6), (0.0, 0.0, 1.0), fov_y_deg=55.0, pixel_sigma=pixel_sigma)
    return sb


def fog_room(width=64, height=48, n_lon=128, n_lat=64, panel_n=16, sigma_s=0.5, sigma_a=0.05, g=0.8, seed=3):
    """The participating-medium configuration at a reduced size: the closed Lambertian box of
    bvh_stress_room filled with a homogeneous medium (scattering sigma_s, absorption sigma_a per
    metre, Henyey-Greenstein g), a displaced-sphere prop, and a PMMA panel whose top face is a
    panel_n x panel_n heightfield of seeded heights, under one area light."""
    sb = SceneBuilder()
    fog = sb._medium(A.INDEX_CONSTANT, (1.0,), absorption=sb.spectrum_constant(sigma_a),
                     scattering=sb.spectrum_constant(sigma_s), g=g)
    sb.region_medium[0] = fog  # the ambient region, where the camera is, holds the medium
    opaque = sb.medium_opaque()
    verts, tris = uv_sphere(n_lon, n_lat, radius=0.6, seed=seed)
    sb.mesh_body(verts, tris, opaque, sb.diffuse(0.6), xf=translate(-1.0, 0.5, 0.8))
    pmma = sb.medium_sellmeier(*PMMA, rel_air=False)
    rng = np.random.Generator(np.random.PCG64(seed))
    h = rng.uniform(-2e-3, 2e-3, (panel_n, panel_n))
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = 0
    inside = sb.region(pmma)
    half, thick = 0.4, 0.05
    top_v, top_t = heightfield_grid(panel_n, panel_n, half, half, thick, h)
    top_v = np.asarray(top_v, float).reshape(-1, 3) + (0.8, -0.4, 0.6)
    glass = sb.dielectric()
    sb.boundary(A.SHAPE_MESH, [], pose(), 0, inside, glass, -1, sb.mesh(top_v, top_t))
    rest_v, rest_t = slab_rest(panel_n, panel_n, half, half, lambda i, j: thick + h[j, i])
    rest_v = np.asarray(rest_v, float).reshape(-1, 3) + (0.8, -0.4, 0.6)
    sb.boundary(A.SHAPE_MESH, [], pose(), 0, inside, glass, -1, sb.mesh(rest_v, rest_t))
    wall = sb.diffuse(0.7)
    w = 3.0
    sb.sheet(w, w, pose(), wall)
    sb.sheet(w, w, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0, 0, 4.0)), wall)
    sb.sheet(2.0, w, pose(rotate_to((0, 0, 1), (1, 0, 0)), (-w, 0, 2.0)), wall)
    sb.sheet(2.0, w, pose(rotate_to((0, 0, 1), (-1, 0, 0)), (w, 0, 2.0)), wall)
    sb.sheet(w, 2.0, pose(rotate_to((0, 0, 1), (0, -1, 0)), (0, w, 2.0)), wall)
    sb.sheet(w, 2.0, pose(rotate_to((0, 0, 1), (0, 1, 0)), (0, -w, 2.0)), wall)
    lamp = sb.emission(sb.spectrum_constant(8.0))
    sb.sheet(0.8, 0.8, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0.0, 0.0, 3.98)), sb.absorber(), emission=lamp)
    sb.observer(width, height, (0.3, -2.7, 1.6), (0.0, 0.0, 1.0), fov_y_deg=55.0)
    return sb


def heightfield_panel(sb, n, heights, half, thickness, offset, inside):
    """A closed slab of `inside`'s medium whose top face is an n x n heightfield over
    [-half, half]^2 at z = thickness + heights, bottom at z = 0, moved by `offset`; both faces smooth
    dielectric boundaries with the ambient region outside. Returns (heightfield boundary, base z of
    its heights in its frame)."""
    h = np.asarray(heights, np.float64).reshape(n, n)
    off = np.asarray(offset, float)
    glass = sb.dielectric()
    top_v, top_t = heightfield_grid(n, n, half, half, thickness, h)
    hf = sb.boundary(A.SHAPE_MESH, [], pose(), 0, inside, glass, -1, sb.mesh(np.asarray(top_v) + off, top_t))
    rest_v, rest_t = slab_rest(n, n, half, half, lambda i, j: thickness + h[j, i])
    sb.boundary(A.SHAPE_MESH, [], pose(), 0, inside, glass, -1, sb.mesh(np.asarray(rest_v) + off, rest_t))
    return hf, thickness + off[2]


def refraction_panel(n=16, heights=None, width=32, height=32, size=0.2, thickness=0.02, elevation=0.3,
                     fog=None, sky=0.05, lamp=20.0):
    """The camera-path adjoint's check scene: a PMMA panel whose top face is an n x n heightfield,
    held `elevation` above a Lambertian floor and seen from 4 m above by a narrow pinhole, so that the
    image is the floor seen through the refracting heights. A rectangular lamp standing low at the
    side lights the floor beneath the panel with a strong falloff; a dim uniform sky lights the rest.
    fog = (sigma_s, sigma_a, g) fills the ambient region with a homogeneous medium."""
    sb = SceneBuilder()
    if fog is not None:
        sb.region_medium[0] = sb._medium(A.INDEX_CONSTANT, (1.0,), absorption=sb.spectrum_constant(fog[1]),
                                         scattering=sb.spectrum_constant(fog[0]), g=fog[2])
    pmma = sb.medium_sellmeier(*PMMA, rel_air=False)
    inside = sb.region(pmma)
    h = np.zeros((n, n)) if heights is None else np.asarray(heights, np.float64).reshape(n, n)
    hf, base_z = heightfield_panel(sb, n, h, size / 2, thickness, (0.0, 0.0, elevation), inside)
    sb.sheet(2.0, 2.0, pose(), sb.diffuse(0.7))
    light = sb.emission(sb.spectrum_constant(lamp))
    sb.sheet(0.1, 0.15, pose(rotate_to((0, 0, 1), (1, 0, 0)), (-0.5, 0.0, 0.15)), sb.absorber(), emission=light)
    if sky > 0:
        sb.uniform_sky(sky)
    sb.observer(width, height, (0.0, 0.0, 4.0), (0.0, 0.0, 0.0), up=(0, 1, 0), fov_y_deg=2.5)
    return sb, {"heightfield": hf, "base_z": base_z, "n": n, "half": size / 2}


def caustic_room(width=1920, height=1080, n_lon=1024, n_lat=512, panel_n=1024, heights=None, sigma_s=0.5,
                 sigma_a=0.05, g=0.8, seed=3, panel_half=0.4, panel_thickness=0.05):
    """The large-adjoint configuration: the closed Lambertian box of bvh_stress_room filled with a
    homogeneous medium (scattering sigma_s, absorption sigma_a per metre, Henyey-Greenstein g), two
    displaced-sphere props of n_lon x n_lat each (2^21 triangles at 1024 x 512), a PMMA panel whose
    top face is a panel_n x panel_n heightfield (heights 0 unless given) standing in the camera's view,
    one area light on the ceiling and a small lamp standing low beside the panel, whose steep falloff
    across the floor beneath the panel is what the camera sees move when the heights refract it;
    1920 x 1080 pinhole camera."""
    sb = SceneBuilder()
    fog = sb._medium(A.INDEX_CONSTANT, (1.0,), absorption=sb.spectrum_constant(sigma_a),
                     scattering=sb.spectrum_constant(sigma_s), g=g)
    sb.region_medium[0] = fog
    opaque = sb.medium_opaque()
    for k, (c, r) in enumerate((((-1.2, 0.8, 0.9), 0.7), ((1.4, 1.2, 0.7), 0.55))):
        verts, tris = uv_sphere(n_lon, n_lat, radius=r, seed=seed + k)
        sb.mesh_body(verts, tris, opaque, sb.diffuse(0.6), xf=translate(*c))
    pmma = sb.medium_sellmeier(*PMMA, rel_air=False)
    inside = sb.region(pmma)
    h = np.zeros((panel_n, panel_n)) if heights is None else np.asarray(heights, np.float64).reshape(panel_n, panel_n)
    hf, base_z = heightfield_panel(sb, panel_n, h, panel_half, panel_thickness, (0.3, -0.6, 0.5), inside)
    wall = sb.diffuse(0.7)
    w = 3.0
    sb.sheet(w, w, pose(), wall)
    sb.sheet(w, w, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0, 0, 4.0)), wall)
    sb.sheet(2.0, w, pose(rotate_to((0, 0, 1), (1, 0, 0)), (-w, 0, 2.0)), wall)
    sb.sheet(2.0, w, pose(rotate_to((0, 0, 1), (-1, 0, 0)), (w, 0, 2.0)), wall)
    sb.sheet(w, 2.0, pose(rotate_to((0, 0, 1), (0, -1, 0)), (0, w, 2.0)), wall)
    sb.sheet(w, 2.0, pose(rotate_to((0, 0, 1), (0, 1, 0)), (0, -w, 2.0)), wall)
    lamp = sb.emission(sb.spectrum_constant(8.0))
    sb.sheet(0.8, 0.8, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0.0, 0.0, 3.98)), sb.absorber(), emission=lamp)
    side = sb.emission(sb.spectrum_constant(40.0))
    sb.sheet(0.15, 0.2, pose(rotate_to((0, 0, 1), (1, 0, 0)), (-0.45, -0.6, 0.15)), sb.absorber(), emission=side)
    sb.observer(width, height, (0.3, -2.7, 1.6), (0.2, -0.2, 0.6), fov_y_deg=50.0)
    return sb, {"heightfield": hf, "base_z": base_z, "n": panel_n, "half": panel_half, "centre": (0.3, -0.6, 0.5),
                "thickness": panel_thickness, "view": ((0.3, -2.7, 1.6), (0.2, -0.2, 0.6), (0, 0, 1), 50.0)}


def planetary_ground(width=64, height=64, radius=6371000.0):
    """The reference's planetary-surface regression (benchmarks/regressions/planetary_ground.owe):
    the ground is a sphere of the Earth's radius whose top lies 0.2 m below the origin, a 5 cm marker
    sphere stands near the origin, the sun at 45 degrees elevation behind the camera and a dim
    uniform sky; a pinhole looks down at the marker. A ray leaving the ground starts |o| = R from the
    sphere's centre, where single precision cannot tell the surface from a metre off it."""
    sb = SceneBuilder()
    sb.uniform_sky(0.1)
    sb.sun((0.0, -math.sqrt(0.5), math.sqrt(0.5)), 1.0e4)
    opaque = sb.medium_opaque()
    sb.sphere_body(radius, (0.0, 0.0, -radius - 0.2), opaque, sb.diffuse(0.3))
    sb.sphere_body(0.05, (0.0, 0.0, 0.05), opaque, sb.diffuse(0.4))
    sb.observer(width, height, (0.0, -0.7, 0.4), (0.0, 0.0, -0.1), fov_y_deg=35.0)
    return sb


def far_nee_visibility(blocker="blocked", width=16, height=16):
    """The reference's far next-event regression (benchmarks/regressions/far_nee_visibility.owe): a
    white 0.4 m receiver at the origin lit only by a 0.1 m emitting sheet (radiance 1e12) 1e6 m
    overhead, facing down, and a black 0.4 m screen 5 cm below the emitter that blocks all of its
    light. blocker = "side" moves the screen 1 m aside, "beyond" to 5 cm above the emitter: both
    leave the receiver lit alike. A segment shortened by a fraction of its length skips the 5 cm."""
    sb = SceneBuilder()
    down = np.diag([1.0, -1.0, -1.0])  # a half turn about x: the sheet's front faces down
    sb.sheet(0.2, 0.2, pose(), sb.diffuse(0.8))
    sb.sheet(0.05, 0.05, pose(down, (0.0, 0.0, 1.0e6)), sb.absorber(), sb.emission(sb.spectrum_constant(1.0e12)))
    at = {"blocked": (0.0, 0.0, 1.0e6 - 0.05), "side": (1.0, 0.0, 1.0e6 - 0.05), "beyond": (0.0, 0.0, 1.0e6 + 0.05)}
    sb.sheet(0.2, 0.2, pose(down, at[blocker]), sb.absorber())
    sb.observer(width, height, (0.0, -0.1, 0.3), (0.0, 0.0, 0.0), fov_y_deg=20.0)
    return sb


def reflected_moonlight(width=16, height=16):
    """The reference's conformance check of light reflected by a distant body (tests/test_backends.cpp:
    69-97): a white two-sided Lambertian floor lit only by a full-phase Lambertian moon (albedo 0.3,
    radius 1e6 m, 1e9 m overhead) under a sun shining up from below (radiance 1e5), the floor's
    scattering guided toward the moon's disk (Scene::indirectGuide: half the samples, radius x 1.001);
    a narrow pinhole looks at the floor. Expected luminance (2/3) 0.3 E_sun (1e6 / 1e9)^2 / pi."""
    sb = SceneBuilder()
    white = sb.diffuse(1.0)
    sb.aim_guide(white, (0.0, 0.0, 1e9), (0.0, 0.0, -1.0), 1e6 * 1.001, 0.5)
    sb.sheet(4.0, 4.0, pose(), white, disk=True)
    sb.sphere_body(1e6, (0.0, 0.0, 1e9), sb.medium_opaque(), sb.diffuse(0.3))
    sb.sun((0.0, 0.0, -1.0), 1e5)
    sb.observer(width, height, (0.0, -1.0, 1.0), (0.0, 0.0, 0.0), fov_y_deg=0.01)
    return sb


def reflected_moonlight_expected(angular_radius=math.radians(0.2665)):
    solar = 1e5 * math.pi * math.sin(angular_radius) ** 2
    return (2.0 / 3.0) * 0.3 * solar * (1e6 / 1e9) ** 2 / math.pi


def furnace_sphere(rho, width=16, height=16):
    """Inside a closed diffuse sphere of albedo rho emitting Le = 1 inward: L = Le / (1 - rho)
    (tests/test_backends.cpp:349-378)."""
    sb = SceneBuilder()
    air = sb.medium_ciddor_air()
    e = sb.emission(sb.spectrum_constant(1.0), front=False, back=True)
    inside = sb.region(air)
    sb.boundary(A.SHAPE_SPHERE, [1.0], pose(), 0, inside, sb.diffuse(rho), e)
    sb.observer(width, height, (0.2, 0.1, -0.3), (1, 0.3, 0), fov_y_deg=70.0, region=inside)
    return sb


def invisible_sphere(width=24, height=24):
    """A lossless N-SF11 sphere in a uniform radiance field is invisible (tests/test_backends.cpp:380-407)."""
    sb = SceneBuilder()
    sb.uniform_sky(1.0)
    sf11 = sb.medium_sellmeier((1.73759695, 0.313747346, 1.89878101), (0.013188707, 0.0623068142, 155.23629),
                               rel_air=True)
    sb.sphere_body(1.0, (0, 0, 0), sf11, sb.dielectric())
    sb.observer(width, height, (0, -4, 0), (0, 0, 0), fov_y_deg=30.0)
    return sb


def _planck(l_nm, kelvin):
    """Planck spectral radiance, lambda in nm evaluated in micrometres (the kernels' planck)."""
    l = np.asarray(l_nm, float) * 1e-3
    return 1e6 * 1.191042972e8 / (l ** 5 * (np.exp(1.438776877e4 / (l * kelvin)) - 1))


def _cie_y(l):
    """The CIE y-bar multi-lobe fit (the kernels' cieY)."""
    l = np.asarray(l, float)

    def lobe(mu, s1, s2):
        t = (l - mu) / np.where(l < mu, s1, s2)
        return np.exp(-0.5 * t * t)
    return 0.821 * lobe(568.8, 46.9, 40.5) + 0.286 * lobe(530.9, 16.3, 31.1)


def blackbody_scale(kelvin, luminance):
    """The scale that gives a blackbody spectrum the luminance (Y) `luminance`."""
    l = np.linspace(360.0, 830.0, 941)
    y = _cie_y(l)
    return luminance * np.trapezoid(y, l) / np.trapezoid(_planck(l, kelvin) * y, l)


def lamp_over_floor(width=24, height=18):
    """A 4000 K lamp sphere (luminance 5, black body) over a 4 x 4 m Lambertian floor whose
    reflectance rises from 0.3 (blue) to 0.9 (red), seen through a pinhole: the scene on which the
    reference's conformance suite checks light tracing against path tracing
    (tests/test_backends.cpp:597-614; the floor's rgb(0.9, 0.6, 0.3) is a tabulated ramp here)."""
    sb = SceneBuilder()
    floor = sb.optics_(A.SURF_DIFFUSE, sb.spectrum_tabulated([400.0, 500.0, 600.0, 700.0], [0.3, 0.5, 0.75, 0.9]))
    sb.sheet(2.0, 2.0, pose(), floor)
    lamp = sb.emission(sb.spectrum_blackbody(4000.0, blackbody_scale(4000.0, 5.0)))
    sb.sphere_body(0.25, (0.4, -0.2, 1.2), sb.medium_opaque(), sb.absorber(), lamp)
    sb.observer(width, height, (0.0, -2.2, 1.4), (0.0, 0.0, 0.0), fov_y_deg=40.0)
    return sb


def disk_irradiance(a=0.3, h=0.5, radiance=2.0, half=0.15, screen=False):
    """A Lambertian disk emitter of radius a (absorbing, emitting downward) at height h over an
    upward-facing square sensor of half-size `half` with 2 x 2 pixels; with `screen` the sensor is a
    diffuse screen of reflectance 0.7 that records the incident flux and scatters the rest
    (tests/analytic.hpp:26-60)."""
    sb = SceneBuilder()
    flip = np.diag([1.0, -1.0, -1.0])  # a half turn about x: the disk's front faces down
    sb.sheet(a, a, pose(flip, (0.0, 0.0, h)), sb.absorber(), sb.emission(sb.spectrum_constant(radiance)), disk=True)
    optics = sb.diffuse(0.7) if screen else sb.optics_(A.SURF_DETECTOR)
    b = sb.sheet(half, half, pose(), optics)
    sb.sensor(2, 2, b, half, half)
    return sb


def disk_irradiance_mean(radiance, a, h, half, n=200):
    """The mean over the centred square of half-size `half` of the irradiance a Lambertian disk of
    radius a and radiance L casts on a parallel plane at distance h below its centre:
    E(r) = pi L / 2 (1 - (h^2 + r^2 - a^2) / sqrt((h^2 + r^2 + a^2)^2 - 4 r^2 a^2))."""
    x = -half + (np.arange(n) + 0.5) * 2 * half / n
    r2 = x[:, None] ** 2 + x[None, :] ** 2
    s = h * h + r2 + a * a
    e = math.pi * radiance / 2 * (1 - (h * h + r2 - a * a) / np.sqrt(s * s - 4 * r2 * a * a))
    return float(e.mean())


def shape_gallery(width=48, height=36, sun=True):
    """One of every trimmed and lathe shape beside the conic ones, as two-sided Lambertian sheets on a
    floor under the sun and a uniform sky: a cone frustum, a torus patch (a vessel's fillet), a round
    wall with two openings, an observatory dome with its slit, a disk with an off-centre hole and an
    even asphere (src/owe/scene/geometry.hpp:51-300)."""
    sb = SceneBuilder()
    sb.sheet(3.0, 3.0, pose(), sb.diffuse(0.5))
    grey, white = sb.diffuse(0.6), sb.diffuse(0.85)
    sb.boundary(A.SHAPE_CONE, [0.35, 0.0, 0.1, 0.6], translate(-1.1, 0.2, 0.0), 0, 0, white)
    sb.boundary(A.SHAPE_TORUS, [0.3, 0.25, 0.2, -math.pi / 2], translate(1.1, 0.2, 0.0), 0, 0, grey,
                data=[math.pi / 2])
    sb.boundary(A.SHAPE_ROUND_WALL, [0.45, 0.7], translate(0.0, 1.2, 0.0), 0, 0, white,
                data=[0.0, 0.35, 0.1, 0.45, math.pi, 0.25, 0.2, 0.6])
    sb.boundary(A.SHAPE_DOME, [0.5, 0.6, 0.25, 1.2], translate(0.0, -0.4, 0.0), 0, 0, grey)
    sb.boundary(A.SHAPE_PLANE, [A.APERTURE_DISK_HOLE, 0.4, 0.12], pose(rotate_to((0, 0, 1), (0, -1, 0.3)), (1.2, -1.0, 0.5)),
                0, 0, white, data=[0.12, 0.05])
    sb.boundary(A.SHAPE_SAG, [1 / 0.6, -0.6, 0.35, 0.0], pose(rotate_to((0, 0, 1), (0.2, -1, 0.4)), (-1.2, -1.0, 0.45)),
                0, 0, white, data=[0.4, -0.6, 0.3])
    if sun:
        sb.sun((0.4, -0.5, 0.75), 3.0e4)
    sb.uniform_sky(0.4)
    sb.observer(width, height, (0.0, -4.2, 2.6), (0.0, 0.1, 0.3), fov_y_deg=42.0)
    return sb


def texture_gallery(width=64, height=40):
    """Every procedural texture on Lambertian albedos: a checker floor and six spheres (noise,
    rings, terrain, bands, radial, marble) under the sun and a uniform sky
    (src/owe/core/shared/textures.hpp:93-138)."""
    sb = SceneBuilder()
    sb.sheet(10.0, 10.0, pose(), sb.textured(A.TEXTURE_CHECKER, 0.8, 0.15, scale=0.4))
    opaque = sb.medium_opaque()
    kinds = [(A.TEXTURE_NOISE, 0.15, 0.0), (A.TEXTURE_RINGS, 0.1, 0.8), (A.TEXTURE_TERRAIN, 0.2, 0.25),
             (A.TEXTURE_BANDS, 0.12, 0.6), (A.TEXTURE_RADIAL, 0.3, 0.0), (A.TEXTURE_MARBLE, 0.25, 0.7)]
    for i, (kind, scale, param) in enumerate(kinds):
        x, y = -1.0 + 1.0 * (i % 3), -0.5 + 1.0 * (i // 3)
        sb.sphere_body(0.35, (x, y, 0.35), opaque, sb.textured(kind, 0.85, 0.1, 0.5, scale=scale, param=param))
    sb.sun((0.3, -0.4, 0.85), 2.0e4)
    sb.uniform_sky(0.5)
    sb.observer(width, height, (0.0, -2.6, 3.2), (0.0, 0.2, 0.2), fov_y_deg=45.0)  # sees no sky
    return sb


def gradient_sky_scene(width=48, height=36):
    """A glass sphere and a Lambertian block on a floor under a gradient sky (ground, horizon,
    zenith; Environment::Sky::Gradient) tilted off the z axis, no sun: the sky seen directly,
    through the glass, and as the only light."""
    sb = SceneBuilder()
    bk7 = sb.medium_sellmeier(*NBK7, rel_air=True)
    sb.sphere_body(0.5, (-0.4, 0.3, 0.5), bk7, sb.dielectric())
    sb.sphere_body(0.35, (0.7, -0.2, 0.35), sb.medium_opaque(), sb.diffuse(0.7))
    sb.sheet(2.5, 2.5, pose(), sb.diffuse(0.6))
    sb.gradient_sky(1.2, 0.4, 0.1, up=(0.1, 0.0, 1.0))
    sb.observer(width, height, (0.0, -3.5, 1.6), (0.0, 0.0, 0.4), fov_y_deg=45.0)
    return sb


def box_mesh(lo, hi):
    """An axis-aligned box as a closed triangle mesh, counter-clockwise seen from outside."""
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = np.array([(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
                  (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)], float)
    t = np.array([(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
                  (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6), (3, 0, 4), (3, 4, 7)], np.uint32)
    return v, t


def touching_glass(width=48, height=36, thickness=0.2, gap=0.0):
    """Two N-BK7 blocks side by side (touching when gap = 0: coincident faces of two boundaries) and
    a thin glass plate of the given thickness over a Lambertian floor under the sun: contacts the
    reference resolves by its region rule (src/owe/scene/world.cpp:440-582)."""
    sb = SceneBuilder()
    bk7 = sb.medium_sellmeier(*NBK7, rel_air=True)
    glass = sb.dielectric()
    v, t = box_mesh((-0.6, -0.3, 0.0), (0.0, 0.3, 0.5))
    sb.mesh_body(v, t, bk7, glass)
    v, t = box_mesh((gap, -0.3, 0.0), (0.6, 0.3, 0.5))
    sb.mesh_body(v, t, bk7, glass)
    v, t = box_mesh((-0.5, -0.9, 0.3), (0.5, -0.45, 0.3 + thickness))
    sb.mesh_body(v, t, bk7, glass)
    sb.sheet(3.0, 3.0, pose(), sb.diffuse(0.7))
    sb.sun((0.35, -0.3, 0.9), 2.0e4)
    sb.uniform_sky(0.3)
    sb.observer(width, height, (0.2, -2.8, 1.9), (0.0, -0.2, 0.25), fov_y_deg=40.0)
    return sb


GALLERY = ("cauchy", "tabulated", "gold", "rough_gold", "rough_glass")


def materials_gallery(width=48, height=36, fog_box=True, sun=True, objects=GALLERY):
    """The optics the configurations do not use, side by side on a Lambertian floor before a wall,
    under a rectangular lamp (and the sun): spheres of Cauchy glass and of glass with a tabulated
    index (both dispersive), a smooth and a rough gold conductor (tabulated n + ik), a rough N-BK7
    dielectric (`objects` picks some; one alone fills the view). With fog_box, a box of scattering fog
    bounded by null boundaries stands between the camera and the spheres, so that camera paths cross
    null boundaries and next-event shadow rays walk through them (Tracer::transmittance,
    src/owe/transport/transport.cpp:237-321)."""
    sb = SceneBuilder()
    sb.sheet(3.0, 3.0, pose(), sb.diffuse(0.6))
    sb.sheet(3.0, 1.5, pose(rotate_to((0, 0, 1), (0, -1, 0)), (0.0, 1.2, 1.5)), sb.diffuse(0.5))
    lam = np.linspace(380.0, 780.0, 11)
    gold_n = sb.spectrum_tabulated([400, 500, 600, 700, 780], [1.47, 0.97, 0.25, 0.16, 0.17])
    gold_k = sb.spectrum_tabulated([400, 500, 600, 700, 780], [1.95, 1.87, 2.98, 3.95, 4.70])
    opaque = sb.medium_opaque()
    places = {"cauchy": (-1.2, 0.2, 0.3), "tabulated": (-0.4, 0.2, 0.3), "gold": (0.4, 0.2, 0.3),
              "rough_gold": (1.2, 0.2, 0.3), "rough_glass": (0.0, -0.5, 0.25)}
    for name in objects:
        c = places[name]
        if name == "cauchy":
            sb.sphere_body(0.3, c, sb._medium(A.INDEX_CAUCHY, (1.5046, 0.00420, 0.0)), sb.dielectric())
        elif name == "tabulated":
            table = sb.spectrum_tabulated(lam, 1.60 + 0.0135 / (lam / 1000) ** 2)
            sb.sphere_body(0.3, c, sb._medium(A.INDEX_TABULATED, index_table=table), sb.dielectric())
        elif name == "gold":
            sb.sphere_body(0.3, c, opaque, sb.optics_(A.SURF_CONDUCTOR, cond_n=gold_n, cond_k=gold_k))
        elif name == "rough_gold":
            sb.sphere_body(0.3, c, opaque, sb.optics_(A.SURF_CONDUCTOR, roughness=0.25, cond_n=gold_n, cond_k=gold_k))
        else:
            sb.sphere_body(0.25, c, sb.medium_sellmeier(*NBK7, rel_air=True), sb.dielectric(roughness=0.2))
    if fog_box:
        fog = sb._medium(A.INDEX_CONSTANT, (1.0,), absorption=sb.spectrum_constant(0.2),
                         scattering=sb.spectrum_constant(1.5), g=0.3)
        v, t = box_mesh((-1.8, -1.6, 0.05), (1.8, -1.0, 1.1))
        sb.boundary(A.SHAPE_MESH, [], pose(), 0, sb.region(fog), sb.optics_(A.SURF_NULL), -1, sb.mesh(v, t))
    lamp = sb.emission(sb.spectrum_constant(6.0))
    sb.sheet(0.6, 0.4, pose(rotate_to((0, 0, 1), (0, 0, -1)), (0.3, -0.3, 2.6)), sb.absorber(), emission=lamp)
    if sun:
        sb.sun((-0.4, -0.5, 0.75), 1.0e4)
    if len(objects) == 1:
        c = places[objects[0]]
        sb.observer(width, height, (c[0], c[1] - 1.6, c[2] + 0.5), c, fov_y_deg=24.0)
    else:
        sb.observer(width, height, (0.0, -3.6, 1.3), (0.0, 0.0, 0.35), fov_y_deg=42.0)
    return sb


def asphere_lens(width=48, height=48):
    """A biconvex N-BK7 lens with even-aspheric faces (A4, A6) and a cylindrical rim over a
    Lambertian floor under the sun: light through two numerically crossed surfaces."""
    sb = SceneBuilder()
    bk7 = sb.medium_sellmeier(*NBK7, rel_air=True)
    glass = sb.region(bk7)
    opt = sb.dielectric()
    r, t = 0.3, 0.12
    # front face: vertex at z = t / 2, bulging up (+z normal outward)
    sb.boundary(A.SHAPE_SAG, [-1 / 0.9, -1.2, r, 0.0], translate(0, 0, 1.0 + t / 2), 0, glass, opt, data=[-0.08, 0.02])
    # back face: vertex at z = -t / 2, bulging down; its +z normal points into the glass
    sb.boundary(A.SHAPE_SAG, [-1 / 0.9, -1.2, r, 0.0], pose(np.diag([1.0, -1.0, -1.0]), (0, 0, 1.0 - t / 2)), 0, glass,
                opt, data=[-0.08, 0.02])
    sag_edge = float(-(1 / 0.9) * r * r / (1 + math.sqrt(1 - (1 - 1.2) * (1 / 0.9) ** 2 * r * r))
                     - 0.08 * r ** 4 + 0.02 * r ** 6)
    sb.boundary(A.SHAPE_CYLINDER, [r, -(t / 2 + sag_edge), t / 2 + sag_edge], translate(0, 0, 1.0), 0, glass, sb.absorber())
    sb.sheet(4.0, 4.0, pose(), sb.diffuse(0.8))
    sb.sun((0.1, -0.15, 1.0), 2.0e4)
    sb.observer(width, height, (0.0, -2.6, 2.4), (0.0, 0.0, 0.6), fov_y_deg=40.0)
    return sb


def ripple_caustics(amplitude=0.0005, wavelength=0.02, depth=0.08, gap=0.001):
    """Sunlight through water rippled by one plane wave h = a sin(k x) onto the flat bottom of a layer,
    and out into a 160 x 4-pixel sensor just below it (tests/test_references.cpp:322-345): an
    overhead sun of unit radiance, a 0.24 m pool with a 0.03 m margin and dielectric floor and walls."""
    sb = SceneBuilder()
    sb.sun((0.0, 0.0, 1.0), 1.0)
    sb.water_pool(0.06, 0.06, depth, 0.03, [plane_wave(amplitude, wavelength)], sb.medium_water())
    b = sb.sheet(0.02, 0.01, translate(0.0, 0.0, -depth - gap), sb.optics_(A.SURF_DETECTOR))
    sb.sensor(160, 4, b, 0.02, 0.01)
    return sb


def wave_pool(width=48, height=32, sampled=False, sun_radius_deg=4.0):
    """A pool of water in a Lambertian basin (benchmarks/caustic_water_surface.owe's body, smaller and
    shallower waves): three analytic plane waves, or 24 ripples sampled as a bicubic spline, under a
    sun widened to `sun_radius_deg` and a uniform sky, seen obliquely through a pinhole."""
    sb = SceneBuilder()
    if sampled:
        waves = ripple_field(24, 3, 0.01, 0.05, slope=0.15)
    else:
        waves = [plane_wave(0.002, 0.03, 0.3), plane_wave(0.0012, 0.021, 1.9, 1.0), plane_wave(0.0008, 0.013, -0.7, 2.0)]
    tile = sb.diffuse(0.8)
    sb.water_pool(0.15, 0.15, 0.08, 0.05, waves, sb.medium_water(), bottom=tile, walls=tile)
    sb.sun((0.3, -0.2, 1.0), 150.0, angular_radius=math.radians(sun_radius_deg))
    sb.uniform_sky(0.3)
    sb.observer(width, height, (0.0, -0.26, 0.26), (0.0, 0.0, -0.06), fov_y_deg=45.0)
    return sb


def random_rays(n, seed, lo, hi, target_lo, target_hi):
    """n rays from uniform points of box [lo, hi] toward uniform points of [target_lo, target_hi]
    (seeded numpy PCG64). Unit directions."""
    rng = np.random.Generator(np.random.PCG64(seed))
    o = rng.uniform(lo, hi, size=(n, 3))
    t = rng.uniform(target_lo, target_hi, size=(n, 3))
    d = t - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.ascontiguousarray(o), np.ascontiguousarray(d)


# ------------------------------------------------------------------ lenses and forward walks
def sag_z(c, k, r):
    """The conic sag at radius r (conicSag, src/owe/core/shared/surfaces.hpp:162)."""
    return c * r * r / (1 + math.sqrt(max(0.0, 1 - (1 + k) * c * c * r * r)))


def ciddor_air(lam_nm):
    l2 = (lam_nm * 1e-3) ** 2
    s2 = 1 / l2
    return 1 + 0.05792105 / (238.0185 - s2) + 0.00167917 / (57.362 - s2)


def sellmeier_index(coefs, lam_nm, rel_air=True):
    l2 = (lam_nm * 1e-3) ** 2
    n = math.sqrt(1 + sum(b * l2 / (l2 - c) for b, c in zip(*coefs)))
    return n * ciddor_air(lam_nm) if rel_air else n


def paraxial_image_distance(radii, thicknesses, indices, object_distance):
    """Distance behind the last vertex where a paraxial ray from an on-axis point `object_distance`
    in front of the first vertex crosses the axis (y-nu trace). indices: the media before, between
    and after the surfaces, relative to the surrounding air."""
    y, nu = 1e-6, 1e-6 / object_distance  # nu = n u
    for i, R in enumerate(radii):
        c = 0.0 if math.isinf(R) else 1.0 / R
        nu = nu - y * c * (indices[i + 1] - indices[i])
        if i < len(thicknesses):
            y = y + thicknesses[i] * nu / indices[i + 1]
    u = nu / indices[-1]
    return -y / u


def lens_body(sb, surfaces, media, thickness, z0=0.0, rim="ground"):
    """buildLens (src/owe/scene/builders.cpp:24-70): conic surfaces S1..Sn+1 along +z from z0, the
    media between them, cylindrical rims between the surfaces' edges. Cemented surfaces are one
    boundary between two glasses. surfaces: (R, semi_diameter)."""
    n = len(media)
    edge = max(sd for _, sd in surfaces)
    regions = [sb.region(m) for m in media]
    dielectric = sb.dielectric()
    rim_optics = sb.absorber() if rim == "black" else sb.dielectric(0.35 if rim == "ground" else 0.0)
    zv = [z0]
    for t in thickness:
        zv.append(zv[-1] + t)
    z_edge = []
    for i, (R, sd) in enumerate(surfaces):
        c = 0.0 if math.isinf(R) else 1.0 / R
        front = regions[i] if i < n else 0
        back = regions[i - 1] if i > 0 else 0
        sb.boundary(A.SHAPE_SAG, [c, 0.0, sd, 0.0], translate(0, 0, zv[i]), front, back, dielectric)
        z_edge.append(zv[i] + sag_z(c, 0.0, sd))
        if sd < edge:
            sb.boundary(A.SHAPE_PLANE, [A.APERTURE_DISK, edge, sd], translate(0, 0, z_edge[i]), front, back, rim_optics)
    for i in range(n):
        assert z_edge[i + 1] > z_edge[i], "non-positive edge thickness"
        sb.boundary(A.SHAPE_CYLINDER, [edge, z_edge[i], z_edge[i + 1]], pose(), 0, regions[i], rim_optics)
    return regions, zv


def achromat_scene(film=1024, half_size=2.5e-4, wavelength=587.5618):
    """A cemented achromat: N-BK7 crown (R1 = 61.5 mm, R2 = -44.6 mm, 6 mm) and N-SF5 flint
    (R3 = -129 mm, 2.5 mm), 25 mm diameter, with a point source 10 m in front on its axis and a
    detector sheet at the paraxial focus (at `wavelength`). Returns (builder, walk description
    fields: detector boundary, source position, focus z)."""
    sb = SceneBuilder()
    bk7 = sb.medium_sellmeier(*NBK7, rel_air=True)
    sf5 = sb.medium_sellmeier(*SF5, rel_air=True)
    radii = [0.0615, -0.0446, -0.129]
    lens_body(sb, [(r, 0.0125) for r in radii], [bk7, sf5], [0.006, 0.0025])
    na = ciddor_air(wavelength)
    idx = [1.0, sellmeier_index(NBK7, wavelength) / na, sellmeier_index(SF5, wavelength) / na, 1.0]
    back_focus = paraxial_image_distance(radii, [0.006, 0.0025], idx, 10.0)
    z_focus = 0.0085 + back_focus
    det = sb.optics_(A.SURF_DETECTOR)
    target = sb.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, half_size, half_size], translate(0, 0, z_focus), 0, 0, det)
    sb.observer(8, 8, (0, 0, -1.0), (0, 0, 0), fov_y_deg=5.0)  # a camera for the renderer's origin; walks bin on the sheet
    return sb, {"target": target, "source": (0.0, 0.0, -10.0), "z_focus": z_focus, "half": half_size, "film": film}


def achromat_walk(info, seed=0, mode=A.WALK_STOCHASTIC, splat=A.SPLAT_NEAREST, lambda_range=(380.0, 780.0),
                  max_events=32):
    """Walks from the point source into the cone that just covers the lens (13 mm at 10 m)."""
    w = A.WalkDesc()
    w.source_kind = A.SOURCE_POINT
    w.mode = mode
    w.max_events = max_events
    w.splat = splat
    w.position = (ctypes.c_double * 3)(*info["source"])
    w.axis = (ctypes.c_double * 3)(0.0, 0.0, 1.0)
    w.extent = math.atan(0.013 / 10.0)
    w.lambda_min, w.lambda_max = lambda_range
    w.region = 0
    w.target = info["target"]
    w.width = w.height = info["film"]
    w.half_x = w.half_y = info["half"]
    w.seed = seed
    w.stream = 0
    return w


# ------------------------------------------------------------------ the differentiable caustic slab
def heightfield_grid(nx, ny, half_x, half_y, base_z, heights):
    """Vertices and triangles of an nx x ny heightfield over [-half_x, half_x] x [-half_y, half_y]:
    vertex j * nx + i at (x_i, y_j, base_z + heights[j, i]); cell (i, j) is split into
    (v00, v10, v11) and (v00, v11, v01), counter-clockwise seen from +z (front: +z)."""
    h = np.asarray(heights, np.float64).reshape(ny, nx)
    x = np.linspace(-half_x, half_x, nx)
    y = np.linspace(-half_y, half_y, ny)
    X, Y = np.meshgrid(x, y)
    v = np.stack([X.ravel(), Y.ravel(), base_z + h.ravel()], 1)
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1))
    v00 = (j * nx + i).ravel()
    v10, v01, v11 = v00 + 1, v00 + nx, v00 + nx + 1
    tris = np.empty((2 * len(v00), 3), np.uint32)
    tris[0::2] = np.stack([v00, v10, v11], 1)
    tris[1::2] = np.stack([v00, v11, v01], 1)
    return v, tris


def slab_rest(nx, ny, half_x, half_y, top_z_edges):
    """The bottom (z = 0) and the four sides of a slab whose top is a heightfield: the sides follow
    the heightfield's edge vertices exactly (the same coordinates), so the body is closed and
    watertight. top_z_edges(i, j) gives the top z at edge vertex (i, j). Faces point outward."""
    x = np.linspace(-half_x, half_x, nx)
    y = np.linspace(-half_y, half_y, ny)
    # bottom as a grid with the same edge vertices (no T-junctions with the sides), facing -z: one
    # quad (x_i, y_j), (x_i, y_j+1), (x_i+1, y_j+1), (x_i+1, y_j) per cell, four vertices each
    I, J = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1))
    I, J = I.ravel(), J.ravel()
    zeros = np.zeros(len(I))
    q = np.stack([np.stack([x[I], y[J], zeros], 1), np.stack([x[I], y[J + 1], zeros], 1),
                  np.stack([x[I + 1], y[J + 1], zeros], 1), np.stack([x[I + 1], y[J], zeros], 1)], 1)
    verts = [q.reshape(-1, 3)]
    base = 4 * np.arange(len(I), dtype=np.int64)
    tris = [np.stack([np.stack([base, base + 1, base + 2], 1), np.stack([base, base + 2, base + 3], 1)], 1).reshape(-1, 3)]
    side_v, side_t = [], []

    def quad(a, b, c, d):  # counter-clockwise seen from outside
        k = len(side_v)
        side_v.extend([a, b, c, d])
        side_t.append((k, k + 1, k + 2))
        side_t.append((k, k + 2, k + 3))

    for i in range(nx - 1):  # side y = -half (normal -y) and y = +half (normal +y)
        quad((x[i], y[0], 0.0), (x[i + 1], y[0], 0.0), (x[i + 1], y[0], top_z_edges(i + 1, 0)), (x[i], y[0], top_z_edges(i, 0)))
        quad((x[i + 1], y[-1], 0.0), (x[i], y[-1], 0.0), (x[i], y[-1], top_z_edges(i, ny - 1)),
             (x[i + 1], y[-1], top_z_edges(i + 1, ny - 1)))
    for j in range(ny - 1):  # side x = -half (normal -x) and x = +half (normal +x)
        quad((x[0], y[j + 1], 0.0), (x[0], y[j], 0.0), (x[0], y[j], top_z_edges(0, j)), (x[0], y[j + 1], top_z_edges(0, j + 1)))
        quad((x[-1], y[j], 0.0), (x[-1], y[j + 1], 0.0), (x[-1], y[j + 1], top_z_edges(nx - 1, j + 1)),
             (x[-1], y[j], top_z_edges(nx - 1, j)))
    off = len(verts[0])
    verts.append(np.array(side_v, float))
    tris.append(np.array(side_t, np.int64) + off)
    return np.concatenate(verts), np.concatenate(tris).astype(np.uint32)


def caustic_slab_scene(n=256, heights=None, wall_bins=512, wall_half=0.075, size=0.1, thickness=0.01,
                       wall_distance=1.0):
    """A PMMA slab (size x size x thickness) whose exit face (+z) is an n x n heightfield, lit by a
    collimated beam along +z; a Lambertian wall `wall_distance` behind the exit face records the
    irradiance in wall_bins^2 bins. The heightfield is boundary `info['heightfield']`, a mesh whose
    vertex j * n + i has height heights[j, i] over z = thickness."""
    sb = SceneBuilder()
    pmma = sb.medium_sellmeier(*PMMA, rel_air=False)
    h = np.zeros((n, n)) if heights is None else np.asarray(heights, np.float64).reshape(n, n)
    half = size / 2
    inside = sb.region(pmma)
    top_v, top_t = heightfield_grid(n, n, half, half, thickness, h)
    glass = sb.dielectric()
    m_top = sb.mesh(top_v, top_t)
    hf = sb.boundary(A.SHAPE_MESH, [], pose(), 0, inside, glass, -1, m_top)
    rest_v, rest_t = slab_rest(n, n, half, half, lambda i, j: thickness + h[j, i])
    m_rest = sb.mesh(rest_v, rest_t)
    sb.boundary(A.SHAPE_MESH, [], pose(), 0, inside, glass, -1, m_rest)
    wall_z = thickness + wall_distance
    wall = sb.boundary(A.SHAPE_PLANE, [A.APERTURE_RECT, 0.5, 0.5], pose(rotate_to((0, 0, 1), (0, 0, -1)), (0, 0, wall_z)),
                       0, 0, sb.diffuse(0.8))
    sb.observer(8, 8, (0.0, 0.0, -1.0), (0, 0, 0), fov_y_deg=10.0)
    sb.frame_origin((0.0, 0.0, thickness))  # FP32 precision where the heights are
    info = {"heightfield": hf, "wall": wall, "n": n, "half": half, "thickness": thickness, "wall_half": wall_half,
            "bins": wall_bins, "wall_z": wall_z}
    return sb, info


def caustic_walk(info, seed=0, splat=A.SPLAT_BILINEAR, wavelength=550.0):
    """The collimated sun beam over the slab's entry face, primary transmission (deterministic
    Fresnel weights), binned on the wall."""
    w = A.WalkDesc()
    w.source_kind = A.SOURCE_COLLIMATED_SQUARE
    w.mode = A.WALK_PRIMARY_TRANSMISSION
    w.max_events = 32
    w.splat = splat
    w.position = (ctypes.c_double * 3)(0.0, 0.0, -0.05)
    w.axis = (ctypes.c_double * 3)(0.0, 0.0, 1.0)
    w.extent = info["half"] * 0.999
    w.lambda_min = w.lambda_max = wavelength
    w.region = 0
    w.target = info["wall"]
    w.width = w.height = info["bins"]
    w.half_x = w.half_y = info["wall_half"]
    w.seed = seed
    w.stream = 0
    return w


def gaussian_blobs(bins, count=64, seed=0, sigma_range=(5.0, 20.0)):
    """A seeded target image: `count` Gaussian blobs of sigma in sigma_range bins, normalised to
    unit mean."""
    rng = np.random.Generator(np.random.PCG64(seed))
    yy, xx = np.mgrid[0:bins, 0:bins] + 0.5
    img = np.zeros((bins, bins))
    for _ in range(count):
        cx, cy = rng.uniform(0.15 * bins, 0.85 * bins, 2)
        s = rng.uniform(*sigma_range)
        img += rng.uniform(0.5, 1.0) * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    return img / img.mean()
