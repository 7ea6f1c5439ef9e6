/*
 * owec.h — the C ABI of the B200 path-tracing backend ("cuda") of the Optical World Engine.
 *
 * The engine's hot path is its unidirectional spectral path tracer: the reference runs it as
 * `Tracer::radiance` over `World::intersect` behind the `owe::Backend` / `owe::Renderer` pair
 * (src/owe/render/backend.hpp:31-52, src/owe/render/renderer.hpp:19-79). This library replaces
 * everything below `Renderer::pass()` and `Renderer::resolve()` with sm_100a kernels. The engine
 * binds it through a thin C++ adapter (a `CudaBackend : owe::Backend` that flattens `owe::Scene`
 * into `owec_scene_desc`), so the world model, scenes and front ends stay unchanged.
 *
 * Conventions
 *   - Every function returns an `int` status: OWEC_OK (0) or a negative OWEC_E_* code. The
 *     message of the last failure on the calling thread is returned by owec_last_error().
 *     The engine's adapter turns a non-zero status into std::runtime_error, which is how the
 *     reference reports an unusable backend (src/owe/render/backend.hpp:44).
 *   - Lengths are metres, wavelengths nanometres, angles radians, as in the reference.
 *   - All pointers are host pointers unless a name ends in `_dev` (device pointers).
 *   - One context serves one thread at a time (the reference drives a Renderer from one thread,
 *     src/owe/render/renderer.hpp:38-47). Calls are synchronous at return unless noted.
 */
#ifndef OWEC_H
#define OWEC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OWEC_ABI_VERSION 5

/* ------------------------------------------------------------------ status codes */
#define OWEC_OK 0
#define OWEC_E_INVALID (-1)      /* a bad argument or scene description                         */
#define OWEC_E_CUDA (-2)         /* a CUDA runtime failure (no device, launch error, ...)       */
#define OWEC_E_NOMEM (-3)        /* device or host allocation failed                            */
#define OWEC_E_STATE (-4)        /* the call needs a step that has not been taken (no scene, ...) */
#define OWEC_E_DEVICE_FAULT (-5) /* a kernel reported a bounded-loop overrun or queue overflow   */
#define OWEC_E_UNSUPPORTED (-6)  /* a feature this backend does not implement                   */

/* ------------------------------------------------------------------ scene description
 * A flattened owe::World (src/owe/scene/world.hpp:1-7): media, regions, optics, emissions and
 * boundaries in world coordinates (IEEE double), plus the environment and one detector. Indices
 * refer to the arrays of the same description. Mirrors the reference's types field by field.
 */

/* Spectrum kinds (src/owe/core/spectrum.hpp:28-78). */
#define OWEC_SPEC_CONSTANT 0  /* value a                                                        */
#define OWEC_SPEC_TABULATED 1 /* piecewise linear over (lambda, value) pairs, clamped at the ends */
#define OWEC_SPEC_BLACKBODY 2 /* Planck at a kelvin, times scale                                 */

typedef struct owec_spectrum {
    int32_t kind;
    int32_t table_offset; /* first (lambda, value) pair in owec_scene_desc.spectrum_table */
    int32_t table_count;  /* number of pairs                                             */
    int32_t pad0;
    double a;     /* constant value, or blackbody temperature in kelvin */
    double scale; /* multiplier of tabulated and blackbody spectra (1 when unused) */
} owec_spectrum;

/* Refractive-index models (src/owe/core/medium.hpp:12-40). */
#define OWEC_INDEX_CONSTANT 0  /* n = coef_a[0]                                        */
#define OWEC_INDEX_CAUCHY 1    /* n = A + B/l^2 + C/l^4, (A,B,C) = coef_a[0..2], l in um */
#define OWEC_INDEX_SELLMEIER 2 /* n^2 = 1 + sum B_i l^2/(l^2 - C_i), B = coef_a, C = coef_b */
#define OWEC_INDEX_CIDDOR 3    /* standard dry air (Ciddor 1996 two-term form)          */
#define OWEC_INDEX_TABULATED 4 /* n = spectrum `index_table`                            */

#define OWEC_MAX_SELLMEIER_TERMS 4

typedef struct owec_medium {
    int32_t index_kind;
    int32_t n_terms;      /* Sellmeier terms used (1..4) */
    int32_t rel_air;      /* 1: the model is relative to air and is multiplied by n_air(l) */
    int32_t opaque;       /* 1: never entered by light (interiors of opaque bodies) */
    double coef_a[OWEC_MAX_SELLMEIER_TERMS];
    double coef_b[OWEC_MAX_SELLMEIER_TERMS];
    int32_t absorption;   /* spectrum index of sigma_a (1/m), -1 = none */
    int32_t scattering;   /* spectrum index of sigma_s (1/m), -1 = none */
    int32_t index_table;  /* spectrum index for OWEC_INDEX_TABULATED, else -1 */
    int32_t pad0;
    double g;             /* Henyey-Greenstein anisotropy */
} owec_medium;

/* Surface types (src/owe/scene/world.hpp:52-61), same order. */
#define OWEC_SURF_NULL 0
#define OWEC_SURF_DIELECTRIC 1
#define OWEC_SURF_DIFFUSE 2
#define OWEC_SURF_CONDUCTOR 3
#define OWEC_SURF_MIRROR 4
#define OWEC_SURF_ABSORBER 5
#define OWEC_SURF_DETECTOR 6

/* Procedural textures of a Lambertian surface's albedo (Texture::Kind, src/owe/scene/world.hpp:29-49,
 * and their patterns, src/owe/core/shared/textures.hpp): mixing weights of the spectra a (the
 * optics' reflectance), b and c at the boundary-local hit point and normal. */
#define OWEC_TEXTURE_NONE 0
#define OWEC_TEXTURE_CHECKER 1
#define OWEC_TEXTURE_NOISE 2
#define OWEC_TEXTURE_RINGS 3
#define OWEC_TEXTURE_TERRAIN 4
#define OWEC_TEXTURE_BANDS 5
#define OWEC_TEXTURE_RADIAL 6
#define OWEC_TEXTURE_MARBLE 7

typedef struct owec_optics {
    int32_t type;
    int32_t back_absorbs;  /* thin opaque sheet with a black back */
    int32_t reflectance;   /* spectrum index (diffuse albedo / mirror reflectance / conductor tint), -1 = 1 */
    int32_t conductor_n;   /* spectrum index of the metal's n, -1 = none */
    int32_t conductor_k;   /* spectrum index of the metal's k, -1 = none */
    int32_t texture;       /* OWEC_TEXTURE_* of a diffuse albedo */
    double roughness;      /* GGX alpha; below 1e-3 the surface is smooth (a delta) */
    int32_t texture_b;     /* spectrum indices of the texture's second and third spectra */
    int32_t texture_c;
    double texture_scale;  /* cell or feature size, metres */
    double texture_param;  /* terrain: snow line height; rings, bands, marble: turbulence */
    /* A Lambertian surface's aim guide (SurfaceOptics::sampleAim*, src/owe/scene/world.hpp:113-114):
     * in radiance transport from the front, aim_share of the scattered directions are drawn toward
     * the disk (aim_center, aim_normal, aim_radius), world coordinates; 0 = none */
    double aim_center[3];
    double aim_normal[3];
    double aim_radius;
    double aim_share;
} owec_optics;

typedef struct owec_emission {
    int32_t radiance; /* spectrum index (Lambertian spectral radiance) */
    int32_t front;
    int32_t back;
    int32_t nee;      /* 0: only seen when hit, never sampled by next-event estimation */
    int32_t distant;  /* sampling hint for astronomical emitters */
    int32_t pad0;
} owec_emission;

/* Shapes (src/owe/scene/geometry.hpp), in their own frames. "Data" is the boundary's run of
 * owec_scene_desc.shape_data (data_offset, data_count). */
#define OWEC_SHAPE_SPHERE 0   /* params: R                                        */
#define OWEC_SHAPE_SAG 1      /* params: c (1/R), k (conic), rMax, rMin; vertex at 0, +z normal. Data: the even
                               * asphere terms A4, A6, ... (none: a conic, solved as a quadric; otherwise the
                               * sag is crossed numerically, SagSurface::intersectNumeric) */
#define OWEC_SHAPE_PLANE 2    /* params: aperture (OWEC_APERTURE_*), a, b         */
#define OWEC_SHAPE_CYLINDER 3 /* params: R, z0, z1                                */
#define OWEC_SHAPE_MESH 4     /* mesh: index into owec_scene_desc.meshes           */
#define OWEC_SHAPE_CONE 5     /* params: r0, z0, r1, z1: the frustum revolving the segment (r0, z0)-(r1, z1)
                               * about z (ConeShape; z0 != z1), normal away from the axis */
#define OWEC_SHAPE_TORUS 6    /* params: R, zc, rho, a0; data: a1. The arc of radius rho about (R, zc) in the
                               * (r, z) half-plane for angles a0..a1, revolved about z (TorusPatchShape) */
#define OWEC_SHAPE_ROUND_WALL 7 /* params: R, H; data: openings as (azimuth, width, sill, top) quadruples: an
                                 * open cylinder from z = 0 to H with rectangular openings (RoundWallShape) */
#define OWEC_SHAPE_DOME 8     /* params: R, slit azimuth, slit width, slit top elevation: the hemisphere
                               * z >= 0 with an observing slit (DomeShape) */
#define OWEC_SHAPE_WAVES 9    /* params: halfX, halfY, margin; data: nodes_x, nodes_y, then the plane waves as
                               * (amplitude, kx, ky, phase): the liquid surface z = w(x) w(y) sum a sin(kx x + ky y
                               * + phase) over the rectangle, tapered to 0 within margin of its edges, +z normal
                               * (WaveSurface). nodes_x = nodes_y = 0: the analytic sum; otherwise the sum
                               * sampled at nodes_x x nodes_y nodes (2..4096 each) as a bicubic Hermite spline */

#define OWEC_APERTURE_DISK 0 /* a = rMax, b = rMin */
#define OWEC_APERTURE_RECT 1 /* a = halfX, b = halfY */
#define OWEC_APERTURE_ELLIPSE 2
#define OWEC_APERTURE_DISK_HOLE 3 /* a = rMax, b = the hole's radius; data: the hole's centre (hx, hy) */

#define OWEC_REGION_OUTSIDE 0xFFFFFFFFu /* placeholder resolved by the engine before flattening */

typedef struct owec_boundary {
    int32_t shape;
    int32_t mesh;       /* OWEC_SHAPE_MESH: mesh index; else -1 */
    uint32_t front;     /* region on the +normal side */
    uint32_t back;      /* region on the -normal side */
    uint32_t optics;
    int32_t emission;   /* -1 = none */
    double to_world[12];/* rigid transform shape -> world: row-major [R | t], 3 rows of 4 */
    double params[4];
    uint32_t data_offset; /* first value of the shape's data in owec_scene_desc.shape_data */
    uint32_t data_count;  /* its number of values (0: none) */
} owec_boundary;

typedef struct owec_mesh {
    uint64_t vertex_offset; /* first vertex in owec_scene_desc.vertices (xyz triples) */
    uint64_t vertex_count;
    uint64_t tri_offset;    /* first triangle in owec_scene_desc.triangles (index triples, mesh-local) */
    uint64_t tri_count;
} owec_mesh;

#define OWEC_SKY_NONE 0
#define OWEC_SKY_UNIFORM 1   /* sky_radiance in every direction */
#define OWEC_SKY_GRADIENT 2  /* Environment::sky's gradient (src/owe/scene/world.cpp:60-65): below the
                              * horizon sky_ground, above it horizon (1 - t) + zenith t, t = cos^0.45
                              * from sky_up; sky_radiance is the zenith */

typedef struct owec_environment {
    int32_t sky_model;
    int32_t sky_radiance;     /* spectrum index of the uniform sky, -1 = none */
    int32_t has_sun;
    int32_t sun_radiance;     /* spectrum index */
    double sun_dir[3];        /* unit vector toward the sun */
    double sun_angular_radius;/* radians; the reference default is 0.2665 degrees */
    double sun_nee_share;     /* fraction of NEE light selections given to the sun (0 = by power) */
    int32_t sky_horizon;      /* OWEC_SKY_GRADIENT: spectrum indices of the horizon and the ground */
    int32_t sky_ground;
    double sky_up[3];         /* OWEC_SKY_GRADIENT: the zenith direction */
} owec_environment;

#define OWEC_DETECTOR_OBSERVER 0 /* IdealObserver: pinhole or thin lens (src/owe/scene/detector.hpp:75-123) */
#define OWEC_DETECTOR_SENSOR 1   /* SurfaceSensor: hemispherical or aimed (src/owe/scene/detector.hpp:125-158) */

typedef struct owec_detector {
    int32_t kind;
    int32_t width;
    int32_t height;
    uint32_t region;          /* region in which camera paths start */
    double position[3];       /* observer */
    double look_at[3];
    double up[3];
    double fov_y;
    double pixel_sigma;       /* Gaussian pixel response in pixels; 0 = the square alone */
    uint32_t boundary;        /* sensor: its detector boundary */
    int32_t pad0;
    double half_x, half_y;    /* sensor: half sizes in the boundary's plane */
    /* Observer: a thin lens (IdealObserver::pupilRadius, focusDistance; pupil 0: a pinhole; focus 0
     * or infinite: focused at infinity) and its pupil guide toward an instrument's exit pupil
     * (IdealObserver::guide; radius 0: none). */
    double pupil_radius, focus_distance;
    double guide_center[3];
    double guide_radius, guide_share;
    /* Sensor: the readout flips and the aimed direction sampling (SurfaceSensor flipX, flipY,
     * hasAim, aimCenter, aimNormal, aimRadius, aimShare, focusCenter, focusRadius, focusShare). */
    int32_t flip_x, flip_y;
    int32_t has_aim, pad1;
    double aim_center[3], aim_normal[3];
    double aim_radius, aim_share;
    double focus_center[3];
    double focus_radius, focus_share;
} owec_detector;

typedef struct owec_scene_desc {
    uint32_t abi_version;     /* OWEC_ABI_VERSION */
    uint32_t n_spectra, n_media, n_regions, n_optics, n_emissions, n_boundaries, n_meshes;
    uint64_t n_spectrum_table, n_vertices, n_triangles;
    const owec_spectrum* spectra;
    const double* spectrum_table;  /* (lambda, value) pairs */
    const owec_medium* media;
    const uint32_t* region_medium; /* medium of each region; region 0 is the ambient region */
    const owec_optics* optics;
    const owec_emission* emissions;
    const owec_boundary* boundaries;
    const owec_mesh* meshes;
    const double* vertices;        /* xyz triples, shape frame of their boundary */
    const uint32_t* triangles;     /* index triples, counter-clockwise = front */
    owec_environment env;
    owec_detector detector;
    /* The origin of the camera-relative FP32 frame. 0: the observer's position (the sensor's
     * centre). 1: frame_origin, for work that measures somewhere else than at the detector: forward
     * walks onto a heightfield want the FP32 precision at the heightfield, not at the camera. */
    int32_t frame_origin_set;
    int32_t pad0;
    double frame_origin[3];
    uint64_t n_shape_data;
    const double* shape_data;      /* the shapes' data (asphere terms, wall openings, ...) */
} owec_scene_desc;

/* ------------------------------------------------------------------ pass settings */

#define OWEC_WAVELENGTHS_HERO4 0      /* four stratified hero wavelengths (src/owe/core/wavelengths.hpp:32-44) */
#define OWEC_WAVELENGTHS_UNIFORM1 1   /* one wavelength per path, uniform in [lambda_min, lambda_max] */

#define OWEC_PRECISION_MIXED 0  /* FP32 camera-relative + FP64 root refinement, re-offset, film sums */
#define OWEC_PRECISION_FP32 1   /* plain FP32 everywhere (the baseline the mixed mode is measured against) */
#define OWEC_PRECISION_FP64 2   /* all-FP64 instantiation of the same kernels */

/* Integrators (RenderSettings::integrator, src/owe/scene/scene.hpp:19). */
#define OWEC_INTEGRATOR_PATH 0   /* "path": camera paths with next-event estimation (Tracer::radiance) */
#define OWEC_INTEGRATOR_LIGHT 1  /* "light": particles from the emitters, connected to the pinhole at every
                                  * non-specular vertex, or recorded where they reach a surface sensor (the
                                  * reference's GPU particle pass, src/owe/backends/gpu/shaders/particle.slang) */

typedef struct owec_settings {
    uint64_t seed;          /* RenderSettings::seed (src/owe/scene/scene.hpp:15-49) */
    int32_t max_depth;      /* RenderSettings::maxDepth */
    int32_t rr_depth;       /* RenderSettings::rrDepth */
    int32_t wavelength_mode;
    int32_t precision;
    double lambda_min;      /* OWEC_WAVELENGTHS_UNIFORM1 range, nm */
    double lambda_max;
    double fresnel_floor;   /* RenderSettings::fresnelFloor */
    int32_t integrator;     /* OWEC_INTEGRATOR_* */
    int32_t pad0;
} owec_settings;

/* Transport statistics (src/owe/scene/transport_stats.hpp:12-31) plus device counters. */
typedef struct owec_stats {
    uint64_t paths, segments, inconsistencies, leaks;
    uint64_t shadow_rays;   /* next-event visibility queries traced */
    uint64_t device_faults; /* bounded loops that ran out (traversal stack, shadow walk guard) */
} owec_stats;

/* ------------------------------------------------------------------ context */

typedef struct owec_ctx owec_ctx;

/* Message of the last failure on this thread (never NULL). */
const char* owec_last_error(void);
/* OWEC_ABI_VERSION of the loaded library. */
int owec_abi_version(void);

/* Opens device `device` (-1: the current one). Replaces Backend::available/createRenderer's
 * device selection (src/owe/render/backend.hpp:38-51). */
int owec_open(int device, owec_ctx** out);
int owec_close(owec_ctx* ctx);
/* Name of the opened device, e.g. "NVIDIA B200". */
int owec_device_name(owec_ctx* ctx, char* buf, size_t len);

/* Copies a scene to the device: the camera-relative FP32 geometry, FP64 shape frames, media,
 * optics and the next-event light table (World::build's buildLightTable,
 * src/owe/scene/world.cpp:285-350). Discards the film. Replaces the scene half of
 * CpuRenderer's constructor (src/owe/backends/cpu/cpu_backend.cpp:37-44). */
int owec_upload_scene(owec_ctx* ctx, const owec_scene_desc* scene);
/* Builds the wide BVH over every primitive on the device (World::build's Bvh::build and each
 * MeshShape's, src/owe/scene/world.cpp:280, src/owe/scene/mesh.cpp:40). */
int owec_build_bvh(owec_ctx* ctx);
/* Node, leaf and primitive counts of the built BVH; bytes of its node and primitive arrays. */
int owec_bvh_info(owec_ctx* ctx, uint64_t info[6]);

/* Render settings used by the next passes; resets the film when they change the estimator. */
int owec_set_settings(owec_ctx* ctx, const owec_settings* settings);
/* One pass of `spp` samples per pixel (Renderer::pass, src/owe/render/renderer.hpp:63;
 * CpuRenderer::pass, src/owe/backends/cpu/cpu_backend.cpp:52-94). Sample s of the pass draws
 * from the PCG32 stream (hashCombine(seed, pixel), pass_index + s): a 1-spp pass reproduces the
 * reference's per-pixel stream exactly. With OWEC_INTEGRATOR_LIGHT a pass emits width x height x
 * spp particles (the reference GPU renderer's passParticles, gpu_renderer_passes.cpp:303-311),
 * particle i drawing from the stream (hashCombine(seed ^ 0x5bd1e995, i), pass_index).
 * Synchronous at return. */
int owec_pass(owec_ctx* ctx, int spp);
/* Resolved image: XYZ per pixel (3 doubles, row-major) and samples per pixel
 * (CpuRenderer::resolve, src/owe/backends/cpu/cpu_backend.cpp:96-107). Either pointer may be NULL.
 * With OWEC_INTEGRATOR_LIGHT the image is the particle splats over the particles emitted
 * (GpuRenderer::resolve, gpu_renderer_film.cpp:17-21) and `samples` is spp summed over the passes. */
int owec_resolve(owec_ctx* ctx, double* xyz, double* samples);
/* owec_resolve without the wait: the image of the passes run so far is formed on the device at once
 * (later passes do not change it) and copied into xyz / samples by a second stream while the caller
 * runs the next passes; owec_resolve_wait returns when every copy started has landed. The buffers
 * must stay valid until then and be page-locked for the copy to overlap (cudaHostAlloc). Two images
 * are kept on the device, so a render loop can start a resolve after every pass: a call waits for
 * the copy it would overwrite, started two calls before (in such a loop it ended during the pass in
 * between). No counterpart in the reference, whose Renderer::resolve returns the image. */
int owec_resolve_async(owec_ctx* ctx, double* xyz, double* samples);
int owec_resolve_wait(owec_ctx* ctx);
/* The film as sums: the compensated per-pixel XYZ sums (3 doubles, row-major) and the samples per
 * pixel, which the ranks of a multi-GPU render add up before dividing. No counterpart in the
 * reference, which renders on one device. Either pointer may be NULL. With OWEC_INTEGRATOR_LIGHT the
 * sums are the particle splats over width x height and the samples spp summed over the passes, so
 * that sums / samples is the resolved image there too. */
int owec_read_film(owec_ctx* ctx, double* xyz_sums, double* samples);
/* owec_read_film into device memory of the context's device (xyz_sums_dev: 3 doubles per pixel,
 * samples_dev: 1 per pixel; either may be NULL): the film's sums stay on the device, for a
 * device-side all-reduce of the ranks' films (NCCL). Path integrator only. No counterpart in the
 * reference. */
int owec_read_film_device(owec_ctx* ctx, double* xyz_sums_dev, double* samples_dev);
/* Sets the index of the next pass's first sample stream (the pass index of owec_pass): each rank
 * of a multi-GPU render starts its share of the streams there, so that the ranks together draw
 * exactly the streams one device would. */
int owec_set_pass_index(owec_ctx* ctx, uint64_t pass_index);
/* Discards the film and the pass count (Renderer::resetObserver, src/owe/render/renderer.hpp:60). */
int owec_reset_film(owec_ctx* ctx);
int owec_read_stats(owec_ctx* ctx, owec_stats* stats);
/* Timing of the last owec_pass, measured with CUDA events on the context's stream:
 * out[0] device seconds of the whole pass, out[1] of its closest-hit (intersect) kernels,
 * out[2] of its shadow-ray kernels, out[3] the number of intersect launches. */
int owec_last_pass_timing(owec_ctx* ctx, double out[4]);

/* Closest hits of n rays given in world coordinates (World::intersect,
 * src/owe/scene/world.cpp:553-582, with no departure anchor). Outputs per ray: boundary index
 * (0xFFFFFFFE on a miss, the reference's kNone), primitive (mesh triangle index, 0 for analytic
 * shapes) and distance. Host buffers; copies are part of the call. */
int owec_cast_rays(owec_ctx* ctx, uint64_t n, const double* origins, const double* directions,
                   uint32_t* boundary, uint32_t* prim, double* t);
/* The same on device buffers already resident in HBM (float32 camera-relative origins, unit
 * float32 directions, packed xyz). Asynchronous on the context's stream; *seconds (may be NULL)
 * receives the kernel's CUDA-event time after an implicit synchronisation when non-NULL. */
int owec_cast_rays_device(owec_ctx* ctx, uint64_t n, const float* origins_dev, const float* directions_dev,
                          uint32_t* boundary_dev, uint32_t* prim_dev, float* t_dev, double* seconds);
/* Traversal counters for the algorithmic traffic of a pass. enable = 1 zeroes and starts them,
 * 0 stops them; out (may be NULL) receives [closest-hit queries, wide nodes visited, primitives
 * tested, shadow queries, their nodes, their primitives] counted while enabled. Counting adds
 * atomics to the traversal kernels: never enable it in a timed pass. */
int owec_trace_counters(owec_ctx* ctx, int enable, uint64_t out[6]);
/* The closest-hit queries of each closest-hit kernel launch, in launch order, of the camera passes
 * run since counting was last enabled (owec_trace_counters with enable = 1), up to 256 launches:
 * out[0 .. min(capacity, *count) - 1]; *count = the launches logged. For dividing a profiler's
 * per-launch counters by the work each launch did. */
int owec_trace_launch_queries(owec_ctx* ctx, uint64_t* out, int capacity, int* count);
/* A log of the crossings whose met region differs from the ray's (TransportStats::inconsistencies),
 * for scenes with contacts (touching bodies, thin plates): capacity > 0 records up to that many
 * (at most 2^20) from the next pass on, 0 stops. Each record is 16 doubles: boundary, triangle,
 * hit flags (1 met from the front, 2 undecided contact), the ray's region, the region met, the
 * boundary and triangle the ray left, the path's depth, the distance, the camera-relative origin
 * (3), the direction (3) and the anchor's error. Scenes without contacts record nothing. */
int owec_inconsistency_log(owec_ctx* ctx, int capacity);
/* Copies min(capacity, *count) records into out (16 doubles each); *count = the crossings logged
 * since the log was enabled (it may exceed the log's capacity). */
int owec_read_inconsistency_log(owec_ctx* ctx, double* out, int capacity, int* count);
/* The camera-relative origin the device geometry is stored against (world = stored + origin). */
int owec_scene_origin(owec_ctx* ctx, double origin[3]);

/* ------------------------------------------------------------------ forward light walks
 * Walks from an emitter through the world to a detector surface, binned where they end on it:
 * the reference's Tracer::walk (src/owe/transport/transport.cpp:531-595) for every walk of a
 * batch, with the emitter sampling of the lens analyser and the inspector's emission probes
 * (src/owe/analysis/analysis.cpp:50-52, src/owe/analysis/inspect.cpp:250-262). Walk i of a batch
 * draws from the PCG32 stream (hashCombine(seed, first_walk + i), stream): first a uniform for its
 * wavelength (uniform in [lambda_min, lambda_max]), then a Draw2 for its emission, then the walk's
 * own draws in the reference's order. */

#define OWEC_SOURCE_POINT 0       /* a point emitting uniformly into a cone about `axis` */
#define OWEC_SOURCE_COLLIMATED 1  /* a parallel beam along `axis` over a disk of radius `extent` */
#define OWEC_SOURCE_COLLIMATED_SQUARE 2 /* the same over a square of half-size `extent` */

#define OWEC_WALK_STOCHASTIC 0            /* WalkMode::Stochastic: Monte-Carlo branching */
#define OWEC_WALK_PRIMARY_TRANSMISSION 1  /* WalkMode::PrimaryTransmission: refract with weight T */

#define OWEC_SPLAT_NEAREST 0   /* each walk adds to the bin it lands in */
#define OWEC_SPLAT_BILINEAR 1  /* a tent one bin wide: smooth in the landing point (differentiable) */

typedef struct owec_walk_desc {
    int32_t source_kind;
    int32_t mode;
    int32_t max_events;      /* the reference's maxEvents (256) */
    int32_t splat;
    double position[3];      /* point source position, or the beam's centre */
    double axis[3];          /* cone axis / beam direction (unit) */
    double extent;           /* point: cone half-angle (radians); collimated: beam radius or half-size */
    double lambda_min, lambda_max;
    uint32_t region;         /* region the walks start in */
    uint32_t target;         /* boundary whose walk endings are binned */
    int32_t width, height;   /* bins over the target's rectangle [-half_x, half_x] x [-half_y, half_y] */
    double half_x, half_y;   /* in the target shape's frame (x, y) */
    uint64_t seed;
    uint64_t stream;
} owec_walk_desc;

typedef struct owec_walk_stats {
    uint64_t walks, binned, escaped, events, faults;
} owec_walk_stats;

/* Adds n walks (first_walk .. first_walk + n - 1) to the walk film of `walk` (one film per
 * context; a different walk description starts it over). Synchronous. */
int owec_walk(owec_ctx* ctx, const owec_walk_desc* walk, uint64_t first_walk, uint64_t n);
/* The walk film: per bin, the sum of the binned walks' throughput times (source measure) /
 * (walks * bin area), where the source measure is the cone's solid angle (point source) or the
 * beam's area (collimated): irradiance per unit source intensity or irradiance. */
int owec_walk_resolve(owec_ctx* ctx, double* bins, owec_walk_stats* stats);
int owec_walk_reset(owec_ctx* ctx);

/* ------------------------------------------------------------------ heightfields and the adjoint
 * A refractive heightfield is a mesh boundary whose vertices move along the z axis of its frame:
 * vertex k of its mesh sits at (x_k, y_k, base_z + h[k]) (x_k, y_k as uploaded). The reference has
 * no heightfield shape; it is a MeshShape (src/owe/scene/mesh.cpp) whose vertices the optimiser
 * moves. */

/* Sets the heights (one per vertex of the boundary's mesh) of mesh boundary `boundary`, makes it the
 * heightfield the adjoint differentiates, and rebuilds the BVH on the device. The caller keeps the
 * vertices shared with other boundaries (a slab's sides) where those boundaries have them. */
int owec_set_heightfield(owec_ctx* ctx, uint32_t boundary, uint64_t n_vertices, double base_z, const double* heights);
/* Path-replay adjoint of the walk film: the gradient of sum_b g[b] * bins[b] (bins as
 * owec_walk_resolve gives them for walks first .. first + n - 1 of `walk`, which must use
 * OWEC_WALK_PRIMARY_TRANSMISSION and OWEC_SPLAT_BILINEAR) with respect to the heights set by
 * owec_set_heightfield, accumulated into dheights (one per vertex). Each walk is recomputed from its seed
 * and differentiated through its crossings; nothing of the forward pass is stored. */
int owec_walk_adjoint(owec_ctx* ctx, const owec_walk_desc* walk, uint64_t first, uint64_t n, const double* g,
                      double* dheights);
/* owec_walk_adjoint for callers that must not allocate device memory once they are running, such
 * as an optimiser loop inside a host application that fixed its GPU memory at start-up, or that
 * shares the device with a framework whose allocator already holds the free memory: there a
 * cudaMalloc can fail, and every cudaMalloc / cudaFree pair stalls the whole device. It has no
 * counterpart in the reference. Its scratch (loss gradient, height-gradient accumulator,
 * counters) is a fixed array in the library image, 10.5 MB on every GPU that loads the library,
 * so the walk film may have at most 512 x 512 bins and the heightfield at most 1048576 vertices;
 * larger calls return OWEC_E_INVALID. The scene must be uploaded and its BVH built, after the
 * settings, beforehand, since those steps allocate. Every call looks up the array's device address
 * (so a device reset between calls is harmless); the first call on a device also loads the array
 * onto it: make that first call before any stream capture. Calls share the array, so two calls that overlap on the
 * GPU (from two threads, or two contexts on one device) race and corrupt each other's results.
 * Same arguments and result as owec_walk_adjoint. */
int owec_walk_adjoint_noalloc(owec_ctx* ctx, const owec_walk_desc* walk, uint64_t first, uint64_t n,
                              const double* g, double* dheights);
/* The path-replay adjoint of the camera film: the gradient of sum_p g[p] . film[p] with respect to the
 * heights set by owec_set_heightfield, added into dheights (one per vertex). film is the resolved image
 * (XYZ per pixel, owec_resolve) of the samples first_pass .. first_pass + spp - 1 of every pixel, as
 * owec_set_pass_index(first_pass) followed by owec_pass(spp) after owec_reset_film renders it; g holds
 * 3 doubles per pixel, row-major. The camera paths are regenerated from their streams and walked again
 * with the forward pass's arithmetic, in two phases per batch: the wavefront kernels run them and stop
 * each at its first surface event on the heightfield, keeping its state there (one checkpoint per path
 * that reaches the heightfield), and a replay kernel resumes from those checkpoints, carrying the
 * derivatives of the path's vertices, directions and throughput with respect to the heights of the
 * heightfield triangles it crosses. This is the backward half of the camera film's forward/backward
 * pair (the forward half is owec_pass); the reference has no differentiable transport. With
 * replay_xyz (may be NULL) every path is instead replayed from its camera ray by the replay kernel,
 * and replay_xyz receives their mean XYZ per pixel, which equals the forward film of the same
 * samples. Needs the path integrator and a scene without null boundaries (OWEC_E_UNSUPPORTED
 * otherwise). */
typedef struct owec_adjoint_stats {
    uint64_t paths;       /* camera paths replayed */
    uint64_t heightfield; /* of them, the paths that crossed the heightfield */
    uint64_t dropped;     /* of those, the paths whose derivative was not followed (an event beyond the
                           * adjoint's model: rough or conductor lobes, textures, shapes other than planes,
                           * spheres and meshes, more than 12 heights): left out of the gradient */
    uint64_t faults;      /* bounded loops that ran out */
    double seconds;       /* device time of the call */
    uint64_t device_bytes;/* device memory the call held beyond what the context held before it: its
                           * buffers (loss gradient, height gradient, checkpoints, replayed film) and the
                           * replay kernel's per-thread stacks */
    double replay_seconds;/* of seconds, the device time of the derivative replay alone (the rest is the
                           * wavefront phase that runs the paths to their first heightfield crossing) */
} owec_adjoint_stats;
/* flags: 0, the unbiased gradient of the expected film (sampling detached: the Fresnel branch and
 * roulette probabilities and the drawn scattering directions held fixed, their weights' values
 * differentiated); OWEC_ADJOINT_FIXED_DECISIONS, the derivative of the estimator at fixed random
 * numbers (those probabilities and frames moving with the path), which central differences with
 * common random numbers measure but which leaves out the branches' boundary terms. */
#define OWEC_ADJOINT_FIXED_DECISIONS 1
int owec_path_adjoint(owec_ctx* ctx, uint64_t first_pass, int spp, int flags, const double* g, double* dheights,
                      double* replay_xyz, owec_adjoint_stats* stats);

/* Throughput probes of the opened device, for rooflines that no driver-measured peak covers: out[0] the
 * FP32 and out[1] the FP64 fused multiply-add rate (flop/s, eight independent chains per thread on
 * every multiprocessor), out[2] the L2 read bandwidth (bytes/s, 128-bit loads that bypass L1 over a
 * buffer a quarter of the L2's size, read repeatedly). Each is one CUDA-event-timed kernel after a
 * warm-up; the call allocates a scratch buffer of a quarter of the L2 for the last. No counterpart
 * in the reference. */
int owec_device_peaks(owec_ctx* ctx, double out[3]);

/* Device seconds of the last owec_walk and owec_walk_adjoint calls. */
int owec_walk_timing(owec_ctx* ctx, double out[2]);

#ifdef __cplusplus
}
#endif

#endif /* OWEC_H */
