// Wavefront OBJ loader (contract: WVM/src/obj_loader.cpp:49-186, tests WVM/tests/test_obj.cpp):
// `v x y z` and `f a b c ...` (1-based absolute indices, "i", "i/t", "i/t/n", "i//n"), fan
// triangulation, one grey Lambertian material, a camera looking down -z at the mesh from 1.5
// bounding-box diagonals, then finalize_scene. Other statements are ignored. Errors are
// std::runtime_error naming the file and, for a bad line, its 1-based number.
#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "wf/scene.hpp"

namespace wf {
namespace {

std::vector<std::string> fields(const std::string& line) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && (line[i] == ' ' || line[i] == '\t' || line[i] == '\r')) ++i;
        const size_t s = i;
        while (i < line.size() && line[i] != ' ' && line[i] != '\t' && line[i] != '\r') ++i;
        if (i > s) out.push_back(line.substr(s, i - s));
    }
    return out;
}

bool whole_float(const std::string& s, float* out) {
    if (s.empty()) return false;
    char* end = nullptr;
    errno = 0;
    const float v = std::strtof(s.c_str(), &end);
    if (end != s.c_str() + s.size()) return false;
    *out = v;
    return true;
}

bool whole_int(const std::string& s, long* out) {
    if (s.empty()) return false;
    char* end = nullptr;
    errno = 0;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end != s.c_str() + s.size() || errno != 0) return false;
    *out = v;
    return true;
}

}  // namespace

Scene load_obj(const std::string& path, int width, int height) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("load_obj: cannot open " + path);
    Scene s;
    s.name = path;
    s.width = width;
    s.height = height;
    auto fail = [&](int line, const std::string& what) {
        throw std::runtime_error(path + " line " + std::to_string(line) + ": " + what);
    };
    std::string line;
    int n = 0;
    while (std::getline(in, line)) {
        ++n;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        const std::vector<std::string> f = fields(line);
        if (f.empty()) continue;
        if (f[0] == "v") {
            if (f.size() != 4) fail(n, "a vertex needs exactly 3 coordinates");
            Vec3 v;
            if (!whole_float(f[1], &v.x) || !whole_float(f[2], &v.y) || !whole_float(f[3], &v.z))
                fail(n, "malformed vertex coordinate");
            s.vertices.push_back(v);
        } else if (f[0] == "f") {
            if (f.size() < 4) fail(n, "a face needs at least 3 indices");
            std::vector<int> idx;
            for (size_t k = 1; k < f.size(); ++k) {
                long v = 0;
                if (!whole_int(f[k].substr(0, f[k].find('/')), &v)) fail(n, "malformed face index '" + f[k] + "'");
                if (v < 1 || v > (long)s.vertices.size())
                    fail(n, "face index " + std::to_string(v) + " outside 1.." + std::to_string(s.vertices.size()));
                idx.push_back((int)v - 1);
            }
            for (size_t k = 1; k + 1 < idx.size(); ++k)
                s.triangles.push_back(Triangle{idx[0], idx[k], idx[k + 1], 0});
        }
    }
    if (s.triangles.empty()) throw std::runtime_error(path + ": no faces");

    Material grey{};
    grey.type = kLambert;
    grey.ior = 1.5f;
    grey.albedo = Vec3{0.7f, 0.7f, 0.7f};
    s.materials.push_back(grey);

    Vec3 lo = s.vertices[0], hi = s.vertices[0];
    for (const Vec3& v : s.vertices) {
        lo = vmin(lo, v);
        hi = vmax(hi, v);
    }
    const Vec3 centre = (lo + hi) * 0.5f;
    const float diag = length(hi - lo);
    s.camera.position = centre + Vec3{0.0f, 0.0f, diag * 1.5f};
    s.camera.look_at = centre;
    s.camera.up = Vec3{0.0f, 1.0f, 0.0f};
    s.camera.vfov_deg = 45.0f;
    finalize_scene(s);
    return s;
}

}  // namespace wf
