// Stand-ins for the reference's glTF model loading (src/owe/scene/gltf.cpp), whose third-party
// decoder (cgltf) is fetched by the reference's CMake at configure time and is absent here. Test
// infrastructure only: the path tracer's hot path loads no models, and a scene that names a glTF
// model fails to load with the message below. Wavefront OBJ models still load through the
// reference's own loadObj.
#include <stdexcept>
#include <string>
#include <vector>

#include "owe/scene/geometry.hpp"

namespace owe {

namespace {
bool isGltf(const std::string& path) {
    auto ends = [&](const char* s) {
        const std::string e(s);
        return path.size() >= e.size() && path.compare(path.size() - e.size(), e.size(), e) == 0;
    };
    return ends(".gltf") || ends(".glb");
}
}  // namespace

MeshData loadGltf(const std::string& path, double) {
    throw std::runtime_error("glTF models are not available in the oracle's build of the engine (no glTF decoder): " + path);
}

MeshData loadModel(const std::string& path, double scale) {
    if (isGltf(path)) return loadGltf(path, scale);
    return loadObj(path, scale);
}

MeshData selectParts(const MeshData& m, const std::vector<std::string>& names) {
    if (names.empty()) return m;
    throw std::runtime_error("selecting named model parts needs the glTF decoder, absent from the oracle's build of the engine");
}

}  // namespace owe
