// Scene validation, finalisation (lights + BVH), the flat view and the canonical scene hash.
// Behaviour and messages follow WVM/src/scene.cpp:10-160 and WVM/src/scenes.cpp:7-26.
#include <stdexcept>
#include "wf/bvh.hpp"
#include "wf/scene.hpp"

namespace wf {

SceneView Scene::view() const {
    SceneView sv{};
    sv.spheres = spheres.empty() ? nullptr : spheres.data();
    sv.vertices = vertices.empty() ? nullptr : vertices.data();
    sv.triangles = triangles.empty() ? nullptr : triangles.data();
    sv.materials = materials.empty() ? nullptr : materials.data();
    sv.nodes = nodes.empty() ? nullptr : nodes.data();
    sv.prim_order = prim_order.empty() ? nullptr : prim_order.data();
    sv.lights = lights.empty() ? nullptr : lights.data();
    sv.n_spheres = (int)spheres.size();
    sv.n_triangles = (int)triangles.size();
    sv.n_materials = (int)materials.size();
    sv.n_nodes = (int)nodes.size();
    sv.n_lights = (int)lights.size();
    sv.env = env;
    sv.camera = make_camera_rig(camera, width, height);
    sv.width = width;
    sv.height = height;
    return sv;
}

std::string validate_scene(const Scene& scene) {
    if (scene.spheres.empty() && scene.triangles.empty()) return "no primitives";
    if (scene.materials.empty()) return "no materials";
    const int n_mat = (int)scene.materials.size();
    const int n_vtx = (int)scene.vertices.size();
    for (const Sphere& s : scene.spheres) {
        if (s.material < 0 || s.material >= n_mat) return "sphere material index out of range";
        if (s.radius <= 0.0f || !is_finite1(s.radius)) return "sphere has invalid radius";
        if (!is_finite3(s.center)) return "sphere centre is non-finite";
    }
    for (const Triangle& t : scene.triangles) {
        if (t.material < 0 || t.material >= n_mat) return "triangle material index out of range";
        const bool bad = t.i0 < 0 || t.i0 >= n_vtx || t.i1 < 0 || t.i1 >= n_vtx || t.i2 < 0 ||
                         t.i2 >= n_vtx;
        if (bad) return "triangle vertex index out of range";
    }
    for (const Vec3& v : scene.vertices)
        if (!is_finite3(v)) return "vertex is non-finite";
    return "";
}

static bool emits(const Material& m) {
    return m.emission.x > 0.0f || m.emission.y > 0.0f || m.emission.z > 0.0f;
}

// Lights in primitive-id order (spheres, then triangles), WVM/src/scene.cpp:69-91.
static void collect_lights(Scene& scene) {
    scene.lights.clear();
    const int ns = (int)scene.spheres.size();
    for (int i = 0; i < ns; ++i) {
        const Sphere& s = scene.spheres[i];
        if (!emits(scene.materials[s.material])) continue;
        const float area = 4.0f * 3.14159265358979323846f * s.radius * s.radius;
        scene.lights.push_back(Light{i, area, {0.0f, 0.0f}});
    }
    for (int i = 0; i < (int)scene.triangles.size(); ++i) {
        const Triangle& t = scene.triangles[i];
        if (!emits(scene.materials[t.material])) continue;
        const Vec3 e1 = scene.vertices[t.i1] - scene.vertices[t.i0];
        const Vec3 e2 = scene.vertices[t.i2] - scene.vertices[t.i0];
        scene.lights.push_back(Light{ns + i, 0.5f * length(cross(e1, e2)), {0.0f, 0.0f}});
    }
}

void finalize_scene_bins(Scene& scene, int sah_bins) {
    const std::string err = validate_scene(scene);
    if (!err.empty()) {
        scene.nodes.clear();
        scene.lights.clear();
        throw std::runtime_error(err);
    }
    collect_lights(scene);
    try {
        build_bvh_bins(scene, sah_bins);
    } catch (...) {
        scene.nodes.clear();
        scene.lights.clear();
        throw;
    }
}

void finalize_scene(Scene& scene) { finalize_scene_bins(scene, 8); }

// 64-bit FNV-1a over the data bytes (no padding) in a fixed order (WVM/src/scene.cpp:107-160).
uint64_t scene_hash(const Scene& scene) {
    uint64_t h = 14695981039346656037ULL;
    auto feed = [&h](const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ULL;
        }
    };
    for (const Sphere& s : scene.spheres) {
        feed(&s.center, sizeof(Vec3));
        feed(&s.radius, 4);
        feed(&s.material, 4);
    }
    for (const Vec3& v : scene.vertices) feed(&v, sizeof(Vec3));
    for (const Triangle& t : scene.triangles) {
        feed(&t.i0, 4);
        feed(&t.i1, 4);
        feed(&t.i2, 4);
        feed(&t.material, 4);
    }
    for (const Material& m : scene.materials) {
        feed(&m.type, 4);
        feed(&m.ior, 4);
        feed(&m.albedo, sizeof(Vec3));
        feed(&m.emission, sizeof(Vec3));
    }
    feed(&scene.env, sizeof(Vec3));
    feed(&scene.camera.position, sizeof(Vec3));
    feed(&scene.camera.look_at, sizeof(Vec3));
    feed(&scene.camera.up, sizeof(Vec3));
    feed(&scene.camera.vfov_deg, 4);
    feed(&scene.width, 4);
    feed(&scene.height, 4);
    return h;
}

}  // namespace wf
