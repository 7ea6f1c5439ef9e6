// The engine-side binding of the CUDA backend: `CudaBackend : owe::Backend` and
// `CudaRenderer : owe::Renderer` over the C ABI of include/owec.h.
//
// This file belongs in the engine's tree as src/owe/backends/cuda/cuda_backend.cpp, beside the cpu
// and gpu backends; the registry lists it (src/owe/backends/registry.cpp:10-13) and the layering
// rule allows it core/, scene/, render/ and backends/cuda/ (not transport/). It flattens the world
// model into owec_scene_desc: media, regions, optics, emitters, boundaries with their rigid frames
// and shape data, the sun and sky, and the detector. Scenes using features the CUDA backend does not
// implement (image albedo textures, environment maps, stained glass) are refused with
// std::runtime_error, as Backend::createRenderer does for unsupported settings
// (src/owe/render/backend.hpp:44); the material maps only the reference GPU renderer applies
// (relief, roughness maps, normal and roughness images) are left out, as its CPU transport leaves them.
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "owe/render/backend.hpp"
#include "owe/scene/geometry.hpp"
#include "owec.h"

namespace owe {

namespace {

void check(int status, const char* what) {
    if (status != OWEC_OK) throw std::runtime_error(std::string(what) + ": " + owec_last_error());
}

// The flattened arrays an owec_scene_desc points into.
struct Flat {
    std::vector<owec_spectrum> spectra;
    std::vector<double> table;
    std::vector<owec_medium> media;
    std::vector<uint32_t> regionMedium;
    std::vector<owec_optics> optics;
    std::vector<owec_emission> emissions;
    std::vector<owec_boundary> boundaries;
    std::vector<owec_mesh> meshes;
    std::vector<double> vertices;
    std::vector<uint32_t> triangles;
    std::vector<double> shapeData;
    owec_scene_desc desc{};

    // Appends a shape's data run and records it in the boundary.
    void data(owec_boundary& b, std::initializer_list<double> values) { data(b, std::vector<double>(values)); }
    void data(owec_boundary& b, const std::vector<double>& values) {
        b.data_offset = uint32_t(shapeData.size());
        b.data_count = uint32_t(values.size());
        shapeData.insert(shapeData.end(), values.begin(), values.end());
    }

    int32_t spectrum(const Spectrum& s) {
        owec_spectrum o{};
        o.scale = 1;
        switch (s.kind()) {
            case Spectrum::Kind::Constant:
                o.kind = OWEC_SPEC_CONSTANT;
                o.a = s.paramA() * s.paramScale();
                break;
            case Spectrum::Kind::Blackbody:
                o.kind = OWEC_SPEC_BLACKBODY;
                o.a = s.paramA();
                o.scale = s.paramScale();
                break;
            default: {  // tabulated, and the RGB spectra sampled every nanometre over the visible range
                o.kind = OWEC_SPEC_TABULATED;
                o.table_offset = int32_t(table.size() / 2);
                if (s.kind() == Spectrum::Kind::Tabulated) {
                    const auto& L = *s.tableLambdas();
                    const auto& V = *s.tableValues();
                    for (size_t i = 0; i < L.size(); ++i) { table.push_back(L[i]); table.push_back(V[i]); }
                    o.table_count = int32_t(L.size());
                    o.scale = s.paramScale();
                } else {
                    int n = 0;
                    for (double l = LambdaMin; l <= LambdaMax; l += 1.0, ++n) {
                        table.push_back(l);
                        table.push_back(s.eval(l));
                    }
                    o.table_count = n;
                }
            }
        }
        spectra.push_back(o);
        return int32_t(spectra.size() - 1);
    }
};

std::unique_ptr<Flat> flatten(const Scene& sc, int detectorIndex) {
    auto f = std::make_unique<Flat>();
    const World& w = sc.world;
    for (const Medium& m : w.media()) {
        owec_medium o{};
        o.absorption = o.scattering = o.index_table = -1;
        o.rel_air = m.index.isRelativeToAir();
        o.opaque = m.opaque;
        o.g = m.g;
        switch (m.index.kind()) {
            case IndexModel::Kind::Constant: o.index_kind = OWEC_INDEX_CONSTANT; o.coef_a[0] = m.index.coeffA()[0]; break;
            case IndexModel::Kind::Cauchy:
                o.index_kind = OWEC_INDEX_CAUCHY;
                for (int i = 0; i < 3; ++i) o.coef_a[i] = m.index.coeffA()[size_t(i)];
                break;
            case IndexModel::Kind::Sellmeier:
                if (m.index.coeffA().size() > OWEC_MAX_SELLMEIER_TERMS)
                    throw std::runtime_error("medium '" + m.name + "': more Sellmeier terms than the cuda backend takes");
                o.index_kind = OWEC_INDEX_SELLMEIER;
                o.n_terms = int32_t(m.index.coeffA().size());
                for (int i = 0; i < o.n_terms; ++i) {
                    o.coef_a[i] = m.index.coeffA()[size_t(i)];
                    o.coef_b[i] = m.index.coeffB()[size_t(i)];
                }
                break;
            case IndexModel::Kind::Ciddor: o.index_kind = OWEC_INDEX_CIDDOR; break;
            case IndexModel::Kind::Tabulated:
                o.index_kind = OWEC_INDEX_TABULATED;
                o.index_table = f->spectrum(m.index.table());
                break;
        }
        if (m.absorbs()) o.absorption = f->spectrum(m.absorption);
        if (m.scatters()) o.scattering = f->spectrum(m.scattering);
        f->media.push_back(o);
    }
    for (const Region& r : w.regions()) f->regionMedium.push_back(r.medium);
    for (const SurfaceOptics& so : w.optics()) {
        // A surface relief, roughness maps and normal or roughness images are the reference GPU
        // renderer's alone (SurfaceOptics, src/owe/scene/world.hpp:88-100): the CPU transport, which
        // this backend follows, renders such a material without them, and so does this backend. An
        // image albedo texture the CPU transport does render; this backend does not.
        if (so.texture.kind == Texture::Kind::Image)
            throw std::runtime_error("material '" + so.name + "' uses an image texture, which the cuda backend does not render");
        if (so.type == SurfaceType::StainedGlass) throw std::runtime_error("stained glass is not rendered by the cuda backend");
        owec_optics o{};
        o.type = int32_t(so.type);
        o.back_absorbs = so.backAbsorbs;
        o.roughness = so.roughness;
        o.reflectance = f->spectrum(so.reflectance);
        o.conductor_n = so.type == SurfaceType::Conductor ? f->spectrum(so.conductor.n) : -1;
        o.conductor_k = so.type == SurfaceType::Conductor ? f->spectrum(so.conductor.k) : -1;
        if (so.texture.kind != Texture::Kind::None && so.type == SurfaceType::Diffuse) {
            // only a Lambertian albedo reads a texture, whose spectrum a takes the reflectance's place
            // (surfaceAlbedo, scattering.cpp:190-195)
            o.texture = int32_t(so.texture.kind);
            o.reflectance = f->spectrum(so.texture.a);
            o.texture_b = f->spectrum(so.texture.b);
            o.texture_c = f->spectrum(so.texture.c);
            o.texture_scale = so.texture.scale;
            o.texture_param = so.texture.param;
        }
        if (so.sampleAimShare > 0 && so.type == SurfaceType::Diffuse) {
            // a measurement screen's or the indirect guide's aim (sampleScatter, scattering.cpp:120-131)
            for (int k = 0; k < 3; ++k) {
                o.aim_center[k] = so.sampleAimCenter[k];
                o.aim_normal[k] = so.sampleAimNormal[k];
            }
            o.aim_radius = so.sampleAimRadius;
            o.aim_share = so.sampleAimShare;
        }
        f->optics.push_back(o);
    }
    for (const Emission& e : w.emissions()) {
        owec_emission o{};
        o.radiance = f->spectrum(e.radiance);
        o.front = e.front;
        o.back = e.back;
        o.nee = e.nee;
        o.distant = e.distant;
        f->emissions.push_back(o);
    }
    for (const Boundary& b : w.boundaries()) {
        owec_boundary o{};
        o.mesh = -1;
        o.front = b.front;
        o.back = b.back;
        o.optics = b.optics;
        o.emission = b.emission;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) o.to_world[4 * i + j] = b.toWorld.R.m[i][j];
            o.to_world[4 * i + 3] = b.toWorld.t[i];
        }
        const Shape* s = b.shape.get();
        if (auto* sp = dynamic_cast<const SphereShape*>(s)) {
            o.shape = OWEC_SHAPE_SPHERE;
            o.params[0] = sp->radius();
        } else if (auto* sg = dynamic_cast<const SagSurface*>(s)) {
            o.shape = OWEC_SHAPE_SAG;
            o.params[0] = sg->curvature();
            o.params[1] = sg->conic();
            o.params[2] = sg->rMax();
            o.params[3] = sg->rMin();
            o.data_offset = uint32_t(f->shapeData.size());
            o.data_count = uint32_t(sg->asphere().size());
            f->shapeData.insert(f->shapeData.end(), sg->asphere().begin(), sg->asphere().end());
        } else if (auto* pl = dynamic_cast<const PlaneShape*>(s)) {
            o.shape = OWEC_SHAPE_PLANE;
            switch (pl->aperture()) {
                case PlaneShape::Aperture::Disk: o.params[0] = OWEC_APERTURE_DISK; break;
                case PlaneShape::Aperture::Rect: o.params[0] = OWEC_APERTURE_RECT; break;
                case PlaneShape::Aperture::Ellipse: o.params[0] = OWEC_APERTURE_ELLIPSE; break;
                case PlaneShape::Aperture::DiskHole:
                    o.params[0] = OWEC_APERTURE_DISK_HOLE;
                    f->data(o, {pl->holeX(), pl->holeY()});
                    break;
            }
            o.params[1] = pl->a();
            o.params[2] = pl->b();
        } else if (auto* cy = dynamic_cast<const CylinderShape*>(s)) {
            o.shape = OWEC_SHAPE_CYLINDER;
            o.params[0] = cy->radius();
            o.params[1] = cy->z0();
            o.params[2] = cy->z1();
        } else if (auto* co = dynamic_cast<const ConeShape*>(s)) {
            o.shape = OWEC_SHAPE_CONE;
            o.params[0] = co->r0();
            o.params[1] = co->z0();
            o.params[2] = co->r1();
            o.params[3] = co->z1();
        } else if (auto* to = dynamic_cast<const TorusPatchShape*>(s)) {
            o.shape = OWEC_SHAPE_TORUS;
            o.params[0] = to->majorRadius();
            o.params[1] = to->zc();
            o.params[2] = to->rho();
            o.params[3] = to->a0();
            f->data(o, {to->a1()});
        } else if (auto* rw = dynamic_cast<const RoundWallShape*>(s)) {
            o.shape = OWEC_SHAPE_ROUND_WALL;
            o.params[0] = rw->radius();
            o.params[1] = rw->height();
            o.data_offset = uint32_t(f->shapeData.size());
            o.data_count = uint32_t(4 * rw->openings().size());
            for (const auto& op : rw->openings())
                f->shapeData.insert(f->shapeData.end(), {op.azimuth, op.width, op.sill, op.top});
        } else if (auto* dm = dynamic_cast<const DomeShape*>(s)) {
            o.shape = OWEC_SHAPE_DOME;
            o.params[0] = dm->radius();
            o.params[1] = dm->slitAzimuth();
            o.params[2] = dm->slitWidth();
            o.params[3] = dm->slitTop();
        } else if (auto* ws = dynamic_cast<const WaveSurface*>(s)) {
            o.shape = OWEC_SHAPE_WAVES;
            o.params[0] = ws->halfX();
            o.params[1] = ws->halfY();
            o.params[2] = ws->margin();
            std::vector<double> data = {double(ws->sampled() ? ws->nodesX() : 0), double(ws->sampled() ? ws->nodesY() : 0)};
            for (const PlaneWave& w : ws->waves()) data.insert(data.end(), {w.amplitude, w.kx, w.ky, w.phase});
            f->data(o, data);
        } else if (auto* me = dynamic_cast<const MeshShape*>(s)) {
            o.shape = OWEC_SHAPE_MESH;
            o.mesh = int32_t(f->meshes.size());
            owec_mesh m{};
            m.vertex_offset = f->vertices.size() / 3;
            m.vertex_count = me->positions().size();
            m.tri_offset = f->triangles.size() / 3;
            m.tri_count = me->triangles().size();
            for (const Vec3& p : me->positions()) { f->vertices.push_back(p.x); f->vertices.push_back(p.y); f->vertices.push_back(p.z); }
            for (const auto& t : me->triangles()) for (uint32_t v : t) f->triangles.push_back(v);
            f->meshes.push_back(m);
        } else {
            throw std::runtime_error("boundary '" + b.name + "' has a shape the cuda backend does not render (" + s->describe() + ")");
        }
        f->boundaries.push_back(o);
    }
    owec_scene_desc& d = f->desc;
    d.abi_version = OWEC_ABI_VERSION;
    const Environment& env = w.env;
    if (env.skyModel == Environment::Sky::Map)
        throw std::runtime_error("the cuda backend renders uniform and gradient skies, not environment maps");
    d.env.sky_model = env.skyModel == Environment::Sky::Uniform    ? OWEC_SKY_UNIFORM
                      : env.skyModel == Environment::Sky::Gradient ? OWEC_SKY_GRADIENT
                                                                   : OWEC_SKY_NONE;
    d.env.sky_radiance = d.env.sky_model != OWEC_SKY_NONE ? f->spectrum(env.zenith) : -1;
    d.env.sky_horizon = d.env.sky_model == OWEC_SKY_GRADIENT ? f->spectrum(env.horizon) : -1;
    d.env.sky_ground = d.env.sky_model == OWEC_SKY_GRADIENT ? f->spectrum(env.ground) : -1;
    for (int k = 0; k < 3; ++k) d.env.sky_up[k] = env.up[k];
    d.env.has_sun = env.hasSun;
    d.env.sun_radiance = env.hasSun ? f->spectrum(env.sunRadiance) : -1;
    for (int k = 0; k < 3; ++k) d.env.sun_dir[k] = env.sunDir[k];
    d.env.sun_angular_radius = env.sunAngularRadius;
    d.env.sun_nee_share = env.sunNeeShare;
    const Detector& det = *sc.detectors.at(size_t(detectorIndex));
    d.detector.width = det.width;
    d.detector.height = det.height;
    d.detector.pixel_sigma = det.pixelSigma;
    d.detector.region = det.region;
    if (auto* eye = dynamic_cast<const IdealObserver*>(&det)) {
        d.detector.kind = OWEC_DETECTOR_OBSERVER;
        for (int k = 0; k < 3; ++k) {
            d.detector.position[k] = eye->position[k];
            d.detector.look_at[k] = eye->lookAt[k];
            d.detector.up[k] = eye->up[k];
            d.detector.guide_center[k] = eye->guide.center[k];
        }
        d.detector.fov_y = eye->fovY;
        d.detector.pupil_radius = eye->pupilRadius;
        d.detector.focus_distance = std::isfinite(eye->focusDistance) ? eye->focusDistance : 0;
        d.detector.guide_radius = eye->guide.radius;
        d.detector.guide_share = eye->guide.share;
    } else if (auto* sen = dynamic_cast<const SurfaceSensor*>(&det)) {
        d.detector.kind = OWEC_DETECTOR_SENSOR;
        d.detector.boundary = sen->boundaryIndex;
        d.detector.half_x = sen->halfX;
        d.detector.half_y = sen->halfY;
        d.detector.flip_x = sen->flipX;
        d.detector.flip_y = sen->flipY;
        d.detector.has_aim = sen->hasAim;
        for (int k = 0; k < 3; ++k) {
            d.detector.aim_center[k] = sen->aimCenter[k];
            d.detector.aim_normal[k] = sen->aimNormal[k];
            d.detector.focus_center[k] = sen->focusCenter[k];
        }
        d.detector.aim_radius = sen->aimRadius;
        d.detector.aim_share = sen->aimShare;
        d.detector.focus_radius = sen->focusRadius;
        d.detector.focus_share = sen->focusShare;
    } else {
        throw std::runtime_error("unknown detector type");
    }
    d.n_spectra = uint32_t(f->spectra.size());
    d.n_media = uint32_t(f->media.size());
    d.n_regions = uint32_t(f->regionMedium.size());
    d.n_optics = uint32_t(f->optics.size());
    d.n_emissions = uint32_t(f->emissions.size());
    d.n_boundaries = uint32_t(f->boundaries.size());
    d.n_meshes = uint32_t(f->meshes.size());
    d.n_spectrum_table = f->table.size() / 2;
    d.n_vertices = f->vertices.size() / 3;
    d.n_triangles = f->triangles.size() / 3;
    d.spectra = f->spectra.data();
    d.spectrum_table = f->table.data();
    d.media = f->media.data();
    d.region_medium = f->regionMedium.data();
    d.optics = f->optics.data();
    d.emissions = f->emissions.data();
    d.boundaries = f->boundaries.data();
    d.meshes = f->meshes.data();
    d.vertices = f->vertices.data();
    d.triangles = f->triangles.data();
    d.n_shape_data = f->shapeData.size();
    d.shape_data = f->shapeData.data();
    return f;
}

class CudaRenderer final : public Renderer {
public:
    CudaRenderer(const Scene& scene, int detectorIndex, const RenderSettings& settings)
        : Renderer(scene, detectorIndex, settings, {"path", "light"}), detectorIndex_(detectorIndex) {
        check(owec_open(settings.device, &ctx_), "cuda backend");
        upload();
        owec_settings s{};
        s.seed = settings.seed;
        s.max_depth = settings.maxDepth;
        s.rr_depth = settings.rrDepth;
        s.wavelength_mode = OWEC_WAVELENGTHS_HERO4;
        s.precision = OWEC_PRECISION_MIXED;
        s.lambda_min = 380;
        s.lambda_max = 780;
        s.fresnel_floor = settings.fresnelFloor;
        s.integrator = settings.integrator == "light" ? OWEC_INTEGRATOR_LIGHT : OWEC_INTEGRATOR_PATH;
        check(owec_set_settings(ctx_, &s), "cuda backend");
    }
    ~CudaRenderer() override { owec_close(ctx_); }

    Image resolve() const override {
        Image img;
        img.width = det_->width;
        img.height = det_->height;
        img.xyz.assign(size_t(img.width) * img.height * 3, 0.0);
        check(owec_resolve(ctx_, img.xyz.data(), nullptr), "cuda backend");
        return img;
    }
    std::string backend() const override {
        char name[256];
        owec_device_name(ctx_, name, sizeof name);
        return std::string("cuda: ") + name + " (sm_100a wavefront; float32 camera-relative + selective float64)";
    }
    bool resetObserver() override {
        upload();  // the pose lives in the scene description; the film starts over
        resetProgress();
        return true;
    }

private:
    void pass(int spp) override {
        check(owec_pass(ctx_, spp), "cuda backend");
        owec_stats st{};
        check(owec_read_stats(ctx_, &st), "cuda backend");
        stats_ = {};
        stats_.paths = st.paths;
        stats_.segments = st.segments;
        stats_.inconsistencies = st.inconsistencies;
        stats_.leaks = st.leaks;
    }
    void upload() {
        auto flat = flatten(scene_, detectorIndex_);
        check(owec_upload_scene(ctx_, &flat->desc), "cuda backend");
        check(owec_build_bvh(ctx_), "cuda backend");
    }

    owec_ctx* ctx_ = nullptr;
    int detectorIndex_;
};

class CudaBackend final : public Backend {
public:
    std::string name() const override { return "cuda"; }
    std::string summary() const override {
        return "NVIDIA B200 (sm_100a) wavefront path tracer; float32 camera-relative with selective float64";
    }
    bool available(std::string* why) const override {
        owec_ctx* c = nullptr;
        if (owec_open(-1, &c) != OWEC_OK) {
            if (why) *why = owec_last_error();
            return false;
        }
        owec_close(c);
        return true;
    }
    std::vector<DeviceInfo> devices() const override {
        owec_ctx* c = nullptr;
        if (owec_open(-1, &c) != OWEC_OK) return {};
        DeviceInfo d;
        char name[256];
        owec_device_name(c, name, sizeof name);
        d.name = name;
        d.type = "discrete";
        d.driver = "CUDA";
        owec_close(c);
        return {d};
    }
    std::vector<std::string> integrators() const override { return {"path", "light"}; }
    std::unique_ptr<Renderer> createRenderer(const Scene& scene, int detectorIndex,
                                             const RenderSettings& settings) const override {
        return std::make_unique<CudaRenderer>(scene, detectorIndex, settings);
    }
};

}  // namespace

const Backend& cudaBackend() {
    static const CudaBackend backend;
    return backend;
}

}  // namespace owe
