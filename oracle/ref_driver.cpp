// Oracle harness over the reference engine itself (test infrastructure, never shipped or timed as
// the product). Compiled together with the reference's own sources into oracle/_ref/liboweref.so by
// oracle/Makefile. It turns an owec_scene_desc (include/owec.h) into an owe::Scene with the
// reference's public API and exposes, as a C ABI for the tests and the CPU-baseline leg of the
// benchmark:
//   - oweref_render: the reference's camera-path pass (CpuRenderer::pass,
//     src/owe/backends/cpu/cpu_backend.cpp:52-94) over Tracer::radiance, with the hero-4 wavelength
//     sampling of the reference, or with one wavelength uniform in [lambda_min, lambda_max], the
//     mode the reference lacks (the pattern of tests/test_transport.cpp:185-186);
//   - oweref_render_backend: the same through the reference's own `cpu` Backend, unchanged;
//   - oweref_cast_rays: World::intersect (src/owe/scene/world.cpp:553-582) for hit-ID parity.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "owe/backends/cpu/cpu_backend.hpp"
#include "owe/core/parallel.hpp"
#include "owe/scene/builders.hpp"
#include "owe/scene/prescription.hpp"
#include "owe/scene/scene.hpp"
#include "owe/transport/transport.hpp"
#include "owec.h"

using namespace owe;

namespace {

thread_local std::string g_error;

struct RefScene {
    Scene scene;
    std::vector<uint32_t> regionMap;  // desc region -> world region
};

Spectrum makeSpectrum(const owec_scene_desc& d, int32_t index) {
    if (index < 0) return Spectrum::constant(0);
    if (uint32_t(index) >= d.n_spectra) throw std::runtime_error("spectrum index out of range");
    const owec_spectrum& s = d.spectra[index];
    switch (s.kind) {
        case OWEC_SPEC_CONSTANT: return Spectrum::constant(s.a);
        case OWEC_SPEC_TABULATED: {
            std::vector<double> l, v;
            for (int32_t i = 0; i < s.table_count; ++i) {
                l.push_back(d.spectrum_table[2 * (s.table_offset + i)]);
                v.push_back(d.spectrum_table[2 * (s.table_offset + i) + 1]);
            }
            return Spectrum::tabulated(l, v).scaled(s.scale);
        }
        case OWEC_SPEC_BLACKBODY: {
            Spectrum b = Spectrum::blackbody(s.a, 1.0);
            return b.scaled(s.scale / b.paramScale());
        }
    }
    throw std::runtime_error("unknown spectrum kind");
}

IndexModel makeIndex(const owec_scene_desc& d, const owec_medium& m) {
    IndexModel idx;
    switch (m.index_kind) {
        case OWEC_INDEX_CONSTANT: idx = IndexModel::constant(m.coef_a[0]); break;
        case OWEC_INDEX_CAUCHY: idx = IndexModel::cauchy(m.coef_a[0], m.coef_a[1], m.coef_a[2]); break;
        case OWEC_INDEX_SELLMEIER: {
            std::vector<double> B(m.coef_a, m.coef_a + m.n_terms), C(m.coef_b, m.coef_b + m.n_terms);
            idx = IndexModel::sellmeier(B, C);
            break;
        }
        case OWEC_INDEX_CIDDOR: idx = IndexModel::ciddorAir(); break;
        case OWEC_INDEX_TABULATED: {
            const owec_spectrum& s = d.spectra[m.index_table];
            std::vector<double> l, v;
            for (int32_t i = 0; i < s.table_count; ++i) {
                l.push_back(d.spectrum_table[2 * (s.table_offset + i)]);
                v.push_back(d.spectrum_table[2 * (s.table_offset + i) + 1] * s.scale);
            }
            idx = IndexModel::tabulated(l, v);
            break;
        }
        default: throw std::runtime_error("unknown index model");
    }
    return m.rel_air ? idx.relativeToAir() : idx;
}

std::shared_ptr<const Shape> makeShape(const owec_scene_desc& d, const owec_boundary& b) {
    const double* p = b.params;
    if (b.data_count && (!d.shape_data || uint64_t(b.data_offset) + b.data_count > d.n_shape_data))
        throw std::runtime_error("shape data out of range");
    const double* data = b.data_count ? d.shape_data + b.data_offset : nullptr;
    switch (b.shape) {
        case OWEC_SHAPE_SPHERE: return std::make_shared<SphereShape>(p[0]);
        case OWEC_SHAPE_SAG:
            return std::make_shared<SagSurface>(p[0], p[1], std::vector<double>(data, data + b.data_count), p[2], p[3]);
        case OWEC_SHAPE_PLANE:
            if (int(p[0]) == OWEC_APERTURE_DISK) return PlaneShape::disk(p[1], p[2]);
            if (int(p[0]) == OWEC_APERTURE_RECT) return PlaneShape::rect(p[1], p[2]);
            if (int(p[0]) == OWEC_APERTURE_DISK_HOLE) {
                if (b.data_count != 2) throw std::runtime_error("disk with hole: its data is the hole's centre");
                return PlaneShape::diskWithHole(p[1], p[2], data[0], data[1]);
            }
            return PlaneShape::ellipse(p[1], p[2]);
        case OWEC_SHAPE_CYLINDER: return std::make_shared<CylinderShape>(p[0], p[1], p[2]);
        case OWEC_SHAPE_CONE: return std::make_shared<ConeShape>(p[0], p[1], p[2], p[3]);
        case OWEC_SHAPE_TORUS:
            if (b.data_count != 1) throw std::runtime_error("torus patch: its data is the arc's end angle");
            return std::make_shared<TorusPatchShape>(p[0], p[1], p[2], p[3], data[0]);
        case OWEC_SHAPE_ROUND_WALL: {
            std::vector<RoundWallShape::Opening> open;
            for (uint32_t i = 0; i + 3 < b.data_count; i += 4)
                open.push_back({data[i], data[i + 1], data[i + 2], data[i + 3]});
            return std::make_shared<RoundWallShape>(p[0], p[1], std::move(open));
        }
        case OWEC_SHAPE_DOME: return std::make_shared<DomeShape>(p[0], p[1], p[2], p[3]);
        case OWEC_SHAPE_WAVES: {
            if (b.data_count < 2 || (b.data_count - 2) % 4)
                throw std::runtime_error("wave surface: its data is the node counts and four values per wave");
            std::vector<PlaneWave> waves;
            for (uint32_t i = 2; i + 3 < b.data_count; i += 4) waves.push_back({data[i], data[i + 1], data[i + 2], data[i + 3]});
            const int nx = int(data[0]), ny = int(data[1]);
            // WaveSurface takes a node spacing: find one that its constructor turns into these counts
            double spacing = 0;
            if (nx > 0) {
                auto count = [](double half, double s) { return std::clamp(int(std::ceil(2 * half / s)) + 1, 2, 4096); };
                spacing = std::max(2 * p[0] / (nx - 1), 2 * p[1] / (ny - 1));
                for (int k = 0; k < 8 && (count(p[0], spacing) != nx || count(p[1], spacing) != ny); ++k)
                    spacing = std::nextafter(spacing, INFINITY);
                if (count(p[0], spacing) != nx || count(p[1], spacing) != ny)
                    throw std::runtime_error("wave surface: no node spacing gives these node counts");
            }
            return std::make_shared<WaveSurface>(std::move(waves), p[0], p[1], p[2], spacing);
        }
        case OWEC_SHAPE_MESH: {
            if (b.mesh < 0 || uint32_t(b.mesh) >= d.n_meshes) throw std::runtime_error("mesh index out of range");
            const owec_mesh& m = d.meshes[b.mesh];
            std::vector<Vec3> pos(m.vertex_count);
            for (uint64_t i = 0; i < m.vertex_count; ++i) {
                const double* v = d.vertices + 3 * (m.vertex_offset + i);
                pos[i] = {v[0], v[1], v[2]};
            }
            std::vector<std::array<uint32_t, 3>> tris(m.tri_count);
            for (uint64_t i = 0; i < m.tri_count; ++i) {
                const uint32_t* t = d.triangles + 3 * (m.tri_offset + i);
                tris[i] = {t[0], t[1], t[2]};
            }
            return std::make_shared<MeshShape>(std::move(pos), std::move(tris), "mesh");
        }
    }
    throw std::runtime_error("unknown shape kind");
}

Transform makeTransform(const double* m) {
    Transform xf;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) xf.R.m[i][j] = m[4 * i + j];
        xf.t[i] = m[4 * i + 3];
    }
    return xf;
}

std::unique_ptr<RefScene> buildScene(const owec_scene_desc& d) {
    auto rs = std::make_unique<RefScene>();
    World& w = rs->scene.world;
    std::vector<uint32_t> mediumMap(d.n_media);
    for (uint32_t i = 0; i < d.n_media; ++i) {
        const owec_medium& m = d.media[i];
        Medium med;
        med.name = "desc-medium-" + std::to_string(i);
        med.index = makeIndex(d, m);
        med.absorption = makeSpectrum(d, m.absorption);
        med.scattering = makeSpectrum(d, m.scattering);
        med.g = m.g;
        med.opaque = m.opaque != 0;
        mediumMap[i] = w.addMedium(med);
    }
    if (d.n_regions == 0) throw std::runtime_error("a scene needs its ambient region");
    rs->regionMap.resize(d.n_regions);
    w.setAmbientMedium(mediumMap.at(d.region_medium[0]));
    rs->regionMap[0] = 0;
    for (uint32_t r = 1; r < d.n_regions; ++r)
        rs->regionMap[r] = w.addRegion("desc-region-" + std::to_string(r), mediumMap.at(d.region_medium[r]));
    std::vector<uint32_t> opticsMap(d.n_optics);
    for (uint32_t i = 0; i < d.n_optics; ++i) {
        const owec_optics& o = d.optics[i];
        SurfaceOptics so;
        so.name = "desc-optics-" + std::to_string(i);
        so.type = SurfaceType(o.type);
        so.roughness = o.roughness;
        so.backAbsorbs = o.back_absorbs != 0;
        so.reflectance = o.reflectance >= 0 ? makeSpectrum(d, o.reflectance) : Spectrum::constant(1.0);
        if (o.conductor_n >= 0) so.conductor.n = makeSpectrum(d, o.conductor_n);
        if (o.conductor_k >= 0) so.conductor.k = makeSpectrum(d, o.conductor_k);
        if (o.texture != OWEC_TEXTURE_NONE) {
            so.texture.kind = Texture::Kind(o.texture);
            so.texture.a = so.reflectance;
            so.texture.b = makeSpectrum(d, o.texture_b);
            so.texture.c = makeSpectrum(d, o.texture_c);
            so.texture.scale = o.texture_scale;
            so.texture.param = o.texture_param;
        }
        if (o.aim_share > 0) {
            const Vec3 n{o.aim_normal[0], o.aim_normal[1], o.aim_normal[2]};
            so.sampleAimCenter = {o.aim_center[0], o.aim_center[1], o.aim_center[2]};
            so.sampleAimNormal = normalize(n);
            so.sampleAimRadius = o.aim_radius;
            so.sampleAimShare = o.aim_share;
        }
        if (so.type == SurfaceType::Detector) so.detector = 0;
        // a diffuse measurement screen: the sensor's own boundary with Lambertian optics
        if (so.type == SurfaceType::Diffuse && d.detector.kind == OWEC_DETECTOR_SENSOR &&
            d.detector.boundary < d.n_boundaries && d.boundaries[d.detector.boundary].optics == i)
            so.detector = 0;
        opticsMap[i] = w.addOptics(so);
    }
    std::vector<int> emissionMap(d.n_emissions);
    for (uint32_t i = 0; i < d.n_emissions; ++i) {
        const owec_emission& e = d.emissions[i];
        Emission em;
        em.radiance = makeSpectrum(d, e.radiance);
        em.front = e.front != 0;
        em.back = e.back != 0;
        em.nee = e.nee != 0;
        em.distant = e.distant != 0;
        emissionMap[i] = w.addEmission(em);
    }
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        w.addBoundary(-1, "desc-boundary-" + std::to_string(i), makeShape(d, b), makeTransform(b.to_world),
                      rs->regionMap.at(b.front), rs->regionMap.at(b.back), opticsMap.at(b.optics),
                      b.emission >= 0 ? emissionMap.at(b.emission) : -1);
    }
    Environment& env = w.env;
    env.skyModel = d.env.sky_model == OWEC_SKY_UNIFORM    ? Environment::Sky::Uniform
                   : d.env.sky_model == OWEC_SKY_GRADIENT ? Environment::Sky::Gradient
                                                          : Environment::Sky::None;
    if (d.env.sky_radiance >= 0) env.zenith = makeSpectrum(d, d.env.sky_radiance);
    if (d.env.sky_model == OWEC_SKY_GRADIENT) {
        env.horizon = makeSpectrum(d, d.env.sky_horizon);
        env.ground = makeSpectrum(d, d.env.sky_ground);
        env.up = normalize(Vec3(d.env.sky_up[0], d.env.sky_up[1], d.env.sky_up[2]));
    }
    env.hasSun = d.env.has_sun != 0;
    env.sunDir = normalize(Vec3(d.env.sun_dir[0], d.env.sun_dir[1], d.env.sun_dir[2]));
    env.sunAngularRadius = d.env.sun_angular_radius;
    if (d.env.sun_radiance >= 0) env.sunRadiance = makeSpectrum(d, d.env.sun_radiance);
    env.sunNeeShare = d.env.sun_nee_share;

    const owec_detector& dd = d.detector;
    if (dd.kind == OWEC_DETECTOR_OBSERVER) {
        auto eye = std::make_unique<IdealObserver>();
        eye->name = "eye";
        eye->width = dd.width;
        eye->height = dd.height;
        eye->position = {dd.position[0], dd.position[1], dd.position[2]};
        eye->lookAt = {dd.look_at[0], dd.look_at[1], dd.look_at[2]};
        eye->up = {dd.up[0], dd.up[1], dd.up[2]};
        eye->fovY = dd.fov_y;
        eye->pixelSigma = dd.pixel_sigma;
        eye->pupilRadius = dd.pupil_radius;
        eye->focusDistance = dd.focus_distance > 0 && std::isfinite(dd.focus_distance) ? dd.focus_distance : Inf;
        rs->scene.detectors.push_back(std::move(eye));
    } else {
        auto s = std::make_unique<SurfaceSensor>();
        s->name = "sensor";
        s->width = dd.width;
        s->height = dd.height;
        s->boundaryIndex = dd.boundary;
        s->halfX = dd.half_x;
        s->halfY = dd.half_y;
        s->pixelSigma = dd.pixel_sigma;
        s->flipX = dd.flip_x != 0;
        s->flipY = dd.flip_y != 0;
        s->hasAim = dd.has_aim != 0;
        s->aimCenter = {dd.aim_center[0], dd.aim_center[1], dd.aim_center[2]};
        s->aimNormal = {dd.aim_normal[0], dd.aim_normal[1], dd.aim_normal[2]};
        s->aimRadius = dd.aim_radius;
        s->aimShare = dd.aim_share;
        s->focusCenter = {dd.focus_center[0], dd.focus_center[1], dd.focus_center[2]};
        s->focusRadius = dd.focus_radius;
        s->focusShare = dd.focus_share;
        rs->scene.detectors.push_back(std::move(s));
    }
    rs->scene.build();
    if (dd.kind == OWEC_DETECTOR_OBSERVER && dd.region != OWEC_REGION_OUTSIDE)
        rs->scene.detectors[0]->region = rs->regionMap.at(dd.region);
    if (dd.kind == OWEC_DETECTOR_OBSERVER && dd.guide_radius > 0) {
        // a pupil guide as IdealObserver::prepare would set for an instrument's exit pupil
        auto* eye = static_cast<IdealObserver*>(rs->scene.detectors[0].get());
        eye->guide.center = {dd.guide_center[0], dd.guide_center[1], dd.guide_center[2]};
        eye->guide.radius = dd.guide_radius;
        eye->guide.share = dd.guide_share;
    }
    return rs;
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
    } catch (...) {
        g_error = "unknown exception";
    }
    return -1;
}

// One camera-path pass of `spp` samples per pixel with the reference's stream layout
// (CpuRenderer::pass, src/owe/backends/cpu/cpu_backend.cpp:52-94). Pixels [first, last) only
// (a bounded sample for timing); xyz/samples are whole-film arrays and are accumulated into.
void pass(const RefScene& rs, const owec_settings& s, int spp, int passIndex, int threads, uint64_t first,
          uint64_t last, double* xyz, double* samples, TransportStats& total) {
    const Scene& sc = rs.scene;
    const Detector& det = *sc.detectors[0];
    Tracer tracer(sc, s.max_depth, s.rr_depth);
    tracer.setFresnelFloor(s.fresnel_floor);
    const int W = det.width;
    const uint64_t n = last - first;
    threads = threads > 0 ? threads : int(hardwareThreads());
    std::atomic<uint64_t> next{0};
    std::vector<TransportStats> stats(static_cast<size_t>(threads));
    const uint64_t chunk = 64;
    parallelWorkers(size_t(threads), [&](size_t tid) {
        for (;;) {
            uint64_t c0 = next.fetch_add(chunk);
            if (c0 >= n) break;
            for (uint64_t k = c0; k < std::min(n, c0 + chunk); ++k) {
                const uint64_t pixel = first + k;
                const int x = int(pixel % uint64_t(W)), y = int(pixel / uint64_t(W));
                Rng rng(hashCombine(s.seed, pixel), uint64_t(passIndex));
                double acc[3] = {0, 0, 0};
                double rot = rng.uniform();
                for (int si = 0; si < spp; ++si) {
                    double u = (si + rng.uniform()) / spp + rot;
                    u -= std::floor(u);
                    Wavelengths wl;
                    if (s.wavelength_mode == OWEC_WAVELENGTHS_UNIFORM1) {
                        const double lam = s.lambda_min + (s.lambda_max - s.lambda_min) * u;
                        wl.lambda.fill(lam);
                        wl.pdf.fill(0);
                        wl.pdf[0] = 1.0 / ((s.lambda_max - s.lambda_min) * NW);
                    } else {
                        wl = Wavelengths::sample(u);
                    }
                    Ray ray;
                    double weight;
                    double px = x + rng.uniform(), py = y + rng.uniform();
                    Vec2 f = det.filterOffset(rng);
                    if (!det.generate(px + f.x, py + f.y, rng, ray, weight) || weight <= 0) continue;
                    Spec4 L = tracer.radiance(ray, det.region, wl, rng, stats[tid]);
                    if (L.isZero()) continue;
                    XYZ c = wl.toXYZ(L * weight);
                    if (!std::isfinite(c.x + c.y + c.z)) continue;
                    acc[0] += c.x;
                    acc[1] += c.y;
                    acc[2] += c.z;
                }
                for (int ch = 0; ch < 3; ++ch) xyz[3 * pixel + ch] += acc[ch];
                if (samples) samples[pixel] += spp;
            }
        }
    });
    for (auto& st : stats) total.add(st);
}

void toStats(const TransportStats& t, owec_stats* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->paths = t.paths;
    out->segments = t.segments;
    out->inconsistencies = t.inconsistencies;
    out->leaks = t.leaks;
}

}  // namespace

extern "C" {

const char* oweref_last_error(void) { return g_error.c_str(); }

void* oweref_scene_create(const owec_scene_desc* desc) {
    std::unique_ptr<RefScene> rs;
    if (guarded([&] { rs = buildScene(*desc); }) != 0) return nullptr;
    return rs.release();
}

void oweref_scene_destroy(void* scene) { delete static_cast<RefScene*>(scene); }

// `passes` passes of `spp` samples per pixel, pass indices first_pass .. first_pass + passes - 1,
// over pixels [pixel_begin, pixel_end) (pixel_end = 0: the whole film). xyz (3 per pixel) and
// samples (1 per pixel, may be NULL) receive the raw sums (not divided by the sample count).
int oweref_render(void* scene, const owec_settings* s, int spp, int passes, int first_pass, int threads,
                  uint64_t pixel_begin, uint64_t pixel_end, double* xyz, double* samples, owec_stats* stats) {
    return guarded([&] {
        const RefScene& rs = *static_cast<const RefScene*>(scene);
        const Detector& det = *rs.scene.detectors[0];
        const uint64_t npix = uint64_t(det.width) * uint64_t(det.height);
        const uint64_t end = pixel_end == 0 ? npix : std::min(pixel_end, npix);
        TransportStats total;
        for (int p = 0; p < passes; ++p)
            pass(rs, *s, spp, first_pass + p, threads, pixel_begin, end, xyz, samples, total);
        toStats(total, stats);
    });
}

// The reference's own cpu backend, unchanged (hero-4 wavelengths only): `passes` passes of `spp`
// through Renderer::runPass, then Renderer::resolve (per-pixel means).
int oweref_render_backend(void* scene, const owec_settings* s, int spp, int passes, int threads, double* xyz,
                          owec_stats* stats, double* seconds) {
    return guarded([&] {
        const RefScene& rs = *static_cast<const RefScene*>(scene);
        RenderSettings st;
        st.backend = "cpu";
        st.seed = s->seed;
        st.maxDepth = s->max_depth;
        st.rrDepth = s->rr_depth;
        st.threads = threads;
        st.fresnelFloor = s->fresnel_floor;
        st.spp = spp;
        auto r = cpuBackend().createRenderer(rs.scene, 0, st);
        for (int p = 0; p < passes; ++p) r->runPass(spp);
        Image img = r->resolve();
        std::memcpy(xyz, img.xyz.data(), img.xyz.size() * sizeof(double));
        toStats(r->stats(), stats);
        if (seconds) *seconds = r->seconds();
    });
}

// World::intersect for n rays without departure anchors. boundary = kNone (0xFFFFFFFE) on a miss.
int oweref_cast_rays(void* scene, uint64_t n, const double* o, const double* d, int threads, uint32_t* boundary,
                     uint32_t* prim, double* t) {
    return guarded([&] {
        const World& w = static_cast<const RefScene*>(scene)->scene.world;
        const size_t parts = size_t(threads > 0 ? threads : int(hardwareThreads()));
        parallelParts(size_t(n), parts * 8, [&](size_t, size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) {
                Ray r{{o[3 * i], o[3 * i + 1], o[3 * i + 2]}, {d[3 * i], d[3 * i + 1], d[3 * i + 2]}};
                SurfaceHit h;
                if (w.intersect(r, Inf, h)) {
                    boundary[i] = h.boundary;
                    prim[i] = h.prim;
                    t[i] = h.t;
                } else {
                    boundary[i] = kNone;
                    prim[i] = 0;
                    t[i] = Inf;
                }
            }
        });
    });
}

// Forward light walks through Tracer::walk (src/owe/transport/transport.cpp:531-595), emitted and
// binned as owec_walk describes (include/owec.h): walk i draws from the stream
// (hashCombine(seed, first + i), stream): its wavelength, its emission (Draw2), then the walk's own
// draws. bins (width * height) receive the sum of the binned walks' throughput times their splat
// weights; stats: [walks, binned, escaped, events].
namespace {

// Tracer::walk for walks first .. first + n - 1 binned as owec_walk bins them; with a box (xmin, xmax,
// ymin, ymax, zmin, zmax, world coordinates), only the walks whose emission point lies in it run.
int walkRange(void* scene, const owec_walk_desc* w, uint64_t first, uint64_t n, int threads, double* bins,
              uint64_t* stats, const double* box) {
    return guarded([&] {
        const RefScene& rs = *static_cast<const RefScene*>(scene);
        const World& world = rs.scene.world;
        Tracer tracer(rs.scene, 64, 6);
        const Vec3 axis = normalize(Vec3(w->axis[0], w->axis[1], w->axis[2]));
        Vec3 S, T;
        orthonormalBasis(axis, S, T);
        const double cosMax = std::cos(w->extent);
        const Boundary& target = world.boundaries().at(w->target);
        const WalkMode mode = w->mode == OWEC_WALK_PRIMARY_TRANSMISSION ? WalkMode::PrimaryTransmission : WalkMode::Stochastic;
        const int nt = threads > 0 ? threads : int(hardwareThreads());
        const size_t nb = size_t(w->width) * w->height;
        std::vector<std::vector<double>> part(size_t(nt), std::vector<double>(nb, 0.0));
        std::vector<std::array<uint64_t, 4>> st(size_t(nt), {0, 0, 0, 0});
        parallelParts(size_t(n), size_t(nt), [&](size_t t, size_t b, size_t e) {
            for (size_t k = b; k < e; ++k) {
                Rng rng(hashCombine(w->seed, first + k), w->stream);
                const double lambda = w->lambda_min + (w->lambda_max - w->lambda_min) * rng.uniform();
                const Draw2 u(rng);
                Vec3 o(w->position[0], w->position[1], w->position[2]), d;
                if (w->source_kind == OWEC_SOURCE_POINT) {
                    const double cosT = (1 - u.u1) + u.u1 * cosMax, sinT = safeSqrt(1 - cosT * cosT), phi = 2 * Pi * u.u2;
                    d = S * (std::cos(phi) * sinT) + T * (std::sin(phi) * sinT) + axis * cosT;
                } else if (w->source_kind == OWEC_SOURCE_COLLIMATED) {
                    const Vec2 q = sampleUniformDiskConcentric(u.u1, u.u2);
                    o = o + (S * q.x + T * q.y) * w->extent;
                    d = axis;
                } else {
                    o = o + (S * (2 * u.u1 - 1) + T * (2 * u.u2 - 1)) * w->extent;
                    d = axis;
                }
                if (box && !(o.x >= box[0] && o.x <= box[1] && o.y >= box[2] && o.y <= box[3] && o.z >= box[4] &&
                             o.z <= box[5]))
                    continue;
                const PathRecord rec = tracer.walk(Ray{o, d}, rs.regionMap.at(w->region), lambda, mode, rng, w->max_events);
                st[t][0]++;
                st[t][3] += rec.v.size() - 1;
                const PathVertex& last = rec.v.back();
                if (last.event == EventKind::Escape) { st[t][2]++; continue; }
                if (last.boundary != w->target) continue;
                if (last.event != EventKind::Detect && last.event != EventKind::Diffuse && last.event != EventKind::Absorb)
                    continue;
                const Vec3 pl = target.toLocal.point(last.p);
                const double fx = (pl.x / w->half_x + 1) * 0.5 * w->width, fy = (1 - pl.y / w->half_y) * 0.5 * w->height;
                bool any = false;
                if (w->splat == OWEC_SPLAT_NEAREST) {
                    if (fx >= 0 && fy >= 0 && fx < w->width && fy < w->height) {
                        part[t][size_t(int(fy)) * w->width + size_t(int(fx))] += last.beta;
                        any = true;
                    }
                } else {
                    const double gx = fx - 0.5, gy = fy - 0.5;
                    const int x0 = int(std::floor(gx)), y0 = int(std::floor(gy));
                    const double ax = gx - x0, ay = gy - y0;
                    for (int j = 0; j < 2; ++j)
                        for (int i = 0; i < 2; ++i) {
                            const int xi = x0 + i, yj = y0 + j;
                            if (xi < 0 || yj < 0 || xi >= w->width || yj >= w->height) continue;
                            part[t][size_t(yj) * w->width + size_t(xi)] += last.beta * (i ? ax : 1 - ax) * (j ? ay : 1 - ay);
                            any = true;
                        }
                }
                if (any) st[t][1]++;
            }
        });
        for (size_t i = 0; i < nb; ++i) {
            double acc = 0;
            for (int t = 0; t < nt; ++t) acc += part[size_t(t)][i];
            bins[i] += acc;
        }
        for (int k = 0; k < 4; ++k) {
            stats[k] = 0;
            for (int t = 0; t < nt; ++t) stats[k] += st[size_t(t)][size_t(k)];
        }
    });
}

}  // namespace

int oweref_walk(void* scene, const owec_walk_desc* w, uint64_t first, uint64_t n, int threads, double* bins,
                uint64_t* stats) {
    return walkRange(scene, w, first, n, threads, bins, stats, nullptr);
}

// The walks of first .. first + n - 1 whose emission point lies in box (xmin, xmax, ymin, ymax, zmin,
// zmax, world coordinates), binned as oweref_walk bins them (raw throughput sums). A finite
// difference of the binned film with common random numbers needs only the walks that can meet the
// moved geometry: the others repeat the same arithmetic on both sides and cancel exactly.
int oweref_walk_in_box(void* scene, const owec_walk_desc* w, uint64_t first, uint64_t n, const double* box,
                       int threads, double* bins, uint64_t* stats) {
    return walkRange(scene, w, first, n, threads, bins, stats, box);
}

// World-level facts the tests pin the restatement against: the light table (selection pdfs),
// the scene radius and the detector's located region.
int oweref_scene_info(void* scene, double* light_pdfs, int max_lights, int* n_lights, double* scene_radius,
                      uint32_t* detector_region) {
    return guarded([&] {
        const RefScene& rs = *static_cast<const RefScene*>(scene);
        const World& w = rs.scene.world;
        *n_lights = int(w.lights().size());
        for (int i = 0; i < std::min(max_lights, *n_lights); ++i) light_pdfs[i] = w.lightSelectPdf(size_t(i));
        *scene_radius = w.sceneRadius();
        *detector_region = rs.scene.detectors[0]->region;
    });
}

// The reference's paraxial analysis (paraxialAnalysis, src/owe/scene/prescription.cpp) of a
// sequence of n spherical surfaces (radii, m; Inf: flat) with thicknesses n - 1 (m) between them
// and Sellmeier glasses after each of the first n - 1 surfaces (3 B and 3 C coefficients per glass,
// relative to air), in air: the image distance behind the last vertex of an on-axis object
// object_distance in front of the first, at lambda (nm).
int oweref_paraxial_image_distance(int n, const double* radii, const double* thickness, const double* sellmeier,
                                   double object_distance, double lambda, double* image_distance) {
    return guarded([&] {
        Prescription p;
        p.objectDistance = object_distance;
        p.wavelength = lambda;
        for (int i = 0; i < n; ++i) {
            PrescriptionSurface s;
            s.R = radii[i];
            s.t = i + 1 < n ? thickness[i] : 0.0;
            s.medium = i + 1 < n ? "glass" + std::to_string(i) : "air";
            s.sd = 0.0125;
            p.surfaces.push_back(s);
        }
        const IndexFn catalog = catalogIndex();
        const IndexFn index = [&](const std::string& medium, double l) {
            if (medium.rfind("glass", 0) != 0) return catalog(medium, l);
            const int g = std::stoi(medium.substr(5));
            const double* c = sellmeier + 6 * g;
            const double um2 = (l * 1e-3) * (l * 1e-3);
            double n2 = 1;
            for (int k = 0; k < 3; ++k) n2 += c[k] * um2 / (um2 - c[3 + k]);
            return std::sqrt(n2) * catalog("air", l);
        };
        *image_distance = paraxialAnalysis(p, lambda, index).imageDistance;
    });
}

// The refractive index of a desc medium at a wavelength (IndexModel::n).
int oweref_medium_index(void* scene, uint32_t region, double lambda, double* n) {
    return guarded([&] {
        const RefScene& rs = *static_cast<const RefScene*>(scene);
        *n = rs.scene.world.indexOf(rs.regionMap.at(region), lambda);
    });
}

}  // extern "C"
