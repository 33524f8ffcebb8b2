// The reference's procedural scenes by name (WVM/src/scenes.cpp:29-347): "cornell", "divergence",
// "trianglehv" and "furnace". Their geometry, materials, cameras and environment are data the
// reference's published scene hashes and test expectations pin, so the values (and the float
// expressions that produce the generated ones) are kept exactly; the construction is this file's.
#include <cmath>
#include <stdexcept>
#include <string>
#include "wf/scene.hpp"

namespace wf {
namespace {

Material mat(MaterialType type, Vec3 albedo, Vec3 emission = Vec3{0.0f, 0.0f, 0.0f}, float ior = 0.0f) {
    Material m{};
    m.type = type;
    m.albedo = albedo;
    m.emission = emission;
    m.ior = ior;
    return m;
}

Sphere ball(Vec3 c, float r, int material) {
    Sphere s{};
    s.center = c;
    s.radius = r;
    s.material = material;
    return s;
}

Scene empty_scene(const char* name, int width, int height, Camera cam, Vec3 env) {
    Scene s;
    s.name = name;
    s.width = width;
    s.height = height;
    s.camera = cam;
    s.env = env;
    return s;
}

// Two spheres as the side walls, a back wall, floor and ceiling of triangles, a ceiling light.
Scene cornell(int w, int h) {
    Scene s = empty_scene("cornell", w, h, Camera{{0.0f, 0.0f, 2.5f}, {0.0f, 0.0f, -2.0f}, {0.0f, 1.0f, 0.0f}, 40.0f},
                          Vec3{0.0f, 0.0f, 0.0f});
    s.materials = {mat(kLambert, {0.7f, 0.7f, 0.7f}), mat(kLambert, {0.7f, 0.2f, 0.2f}),
                   mat(kLambert, {0.2f, 0.7f, 0.2f}), mat(kLambert, {0.7f, 0.7f, 0.7f}, {5.0f, 5.0f, 5.0f})};
    s.spheres = {ball({-1.5f, 0.0f, -2.0f}, 0.3f, 1), ball({1.5f, 0.0f, -2.0f}, 0.3f, 2)};
    s.vertices = {{-3.0f, -2.0f, -4.0f}, {3.0f, -2.0f, -4.0f}, {3.0f, 2.0f, -4.0f},  {-3.0f, 2.0f, -4.0f},
                  {-3.0f, -2.0f, 0.0f},  {3.0f, -2.0f, 0.0f},  {-3.0f, 2.0f, 0.0f},  {3.0f, 2.0f, 0.0f},
                  {-1.0f, 1.99f, -2.5f}, {1.0f, 1.99f, -2.5f}, {1.0f, 1.99f, -1.5f}, {-1.0f, 1.99f, -1.5f}};
    s.triangles = {{0, 1, 2, 0}, {0, 2, 3, 0},    // back wall z = -4
                   {0, 4, 5, 0}, {0, 5, 1, 0},    // floor y = -2
                   {3, 2, 7, 0}, {3, 7, 6, 0},    // ceiling y = 2
                   {8, 9, 10, 3}, {8, 10, 11, 3}};  // light quad
    return s;
}

// A 30 x 30 grid of small spheres alternating Lambertian / metal / dielectric on a ground quad,
// lit by one small emissive sphere: material divergence inside every warp.
Scene divergence(int w, int h) {
    Scene s = empty_scene("divergence", w, h, Camera{{0.0f, 2.0f, 6.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, 45.0f},
                          Vec3{0.05f, 0.05f, 0.05f});
    s.materials = {mat(kLambert, {0.5f, 0.5f, 0.5f}),           mat(kLambert, {0.7f, 0.7f, 0.7f}),
                   mat(kLambert, {0.7f, 0.3f, 0.3f}),           mat(kLambert, {0.3f, 0.3f, 0.7f}),
                   mat(kMetal, {0.9f, 0.9f, 0.9f}),             mat(kDielectric, {1.0f, 1.0f, 1.0f}, {0, 0, 0}, 1.5f),
                   mat(kEmissive, {0.0f, 0.0f, 0.0f}, {1.0f, 1.0f, 1.0f})};
    s.vertices = {{-15.0f, -1.0f, -15.0f}, {15.0f, -1.0f, -15.0f}, {15.0f, -1.0f, 15.0f}, {-15.0f, -1.0f, 15.0f}};
    s.triangles = {{0, 1, 2, 0}, {0, 2, 3, 0}};
    const float spacing = 0.33f, radius = 0.16f;
    for (int i = 0; i < 30; ++i)
        for (int j = 0; j < 30; ++j) {
            const int material = ((i + j) & 1) == 0 ? (i + j) % 4 : ((i & 1) ? 5 : 4);
            s.spheres.push_back(ball({-4.95f + i * spacing, 0.2f, -4.95f + j * spacing}, radius, material));
        }
    s.spheres.push_back(ball({0.0f, 5.0f, 0.0f}, 0.2f, 6));
    return s;
}

// A 240 x 240-cell height field (115,200 triangles) with two mirror spheres and a spherical light.
Scene trianglehv(int w, int h) {
    Scene s = empty_scene("trianglehv", w, h, Camera{{5.0f, 3.0f, 5.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, 50.0f},
                          Vec3{0.05f, 0.05f, 0.1f});
    s.materials = {mat(kLambert, {0.7f, 0.7f, 0.7f}), mat(kMetal, {0.9f, 0.9f, 0.9f}),
                   mat(kEmissive, {0.0f, 0.0f, 0.0f}, {3.0f, 3.0f, 3.0f})};
    const int n = 240, half = n / 2;
    const float extent = 10.0f, amplitude = 1.0f;
    s.vertices.reserve((size_t)(n + 1) * (n + 1));
    for (int i = 0; i <= n; ++i)
        for (int j = 0; j <= n; ++j) {
            const float x = (i - half) * extent / half;
            const float z = (j - half) * extent / half;
            const float y = amplitude * (sinf(x) * cosf(z) + 0.5f * (x * x + z * z) / 100.0f);
            s.vertices.push_back(Vec3{x, y, z});
        }
    s.triangles.reserve((size_t)2 * n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const int v0 = i * (n + 1) + j, v1 = v0 + 1, v2 = v0 + (n + 1), v3 = v2 + 1;
            s.triangles.push_back(Triangle{v0, v1, v2, 0});
            s.triangles.push_back(Triangle{v1, v3, v2, 0});
        }
    s.spheres = {ball({0.0f, 2.0f, 0.0f}, 0.5f, 1), ball({3.0f, 1.5f, -2.0f}, 0.4f, 1), ball({0.0f, 5.0f, 0.0f}, 0.3f, 2)};
    return s;
}

// The camera inside an emissive grey sphere: image mean Le / (1 - albedo) (white furnace).
Scene furnace(int w, int h) {
    Scene s = empty_scene("furnace", w, h, Camera{{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, -1.0f}, {0.0f, 1.0f, 0.0f}, 90.0f},
                          Vec3{0.0f, 0.0f, 0.0f});
    s.materials = {mat(kLambert, {0.5f, 0.5f, 0.5f}, {1.0f, 1.0f, 1.0f})};
    s.spheres = {ball({0.0f, 0.0f, 0.0f}, 5.0f, 0)};
    return s;
}

}  // namespace

Scene make_scene(const std::string& name, int width, int height) {
    Scene s;
    if (name == "cornell") s = cornell(width, height);
    else if (name == "divergence") s = divergence(width, height);
    else if (name == "trianglehv") s = trianglehv(width, height);
    else if (name == "furnace") s = furnace(width, height);
    else throw std::invalid_argument("unknown scene name: " + name);
    finalize_scene(s);
    return s;
}

}  // namespace wf
