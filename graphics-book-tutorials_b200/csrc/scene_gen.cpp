// Procedural benchmark scenes and orbit cameras.
//
//   "cornell36"   Cornell box: five walls of the unit box as 10 triangles (grey 0.73, left wall
//                 red (0.65,0.05,0.05), right wall green (0.12,0.45,0.15)), a tall and a short box
//                 (24 triangles, grey 0.73) rotated about y by +18 and -18 degrees, and a ceiling
//                 quad light (2 triangles, emission 15). 36 triangles.
//   "icospheres"  ground quad + 512 level-2 icospheres (320 triangles each), radius U(0.2, 0.6),
//                 centres uniform over a 20 x 20 area on the ground; each sphere's material is
//                 drawn uniformly from {Lambertian albedo U(0,1)^3, metal with roughness U(0, 0.5)
//                 (stored in Material::pad0; shading is the reference's perfect mirror),
//                 dielectric ior 1.5}; an overhead emissive quad (emission 8). 163,844 triangles.
//   "heightfield" 1024 x 1024-vertex grid over a 20 x 20 extent, heights from 6-octave fBm value
//                 noise (lacunarity 2, gain 0.5) scaled to 0.15 of the extent; Lambertian albedo
//                 banded by height (green -> brown -> white, 8 bands); sky emission 1.0 plus a
//                 distant emissive quad. 2,093,058 + 2 triangles.
//
// Random numbers come from SplitMix64 (Steele, Lea, Flood 2014) seeded with the scene seed; a
// float draw is the top 24 bits times 2^-24. The value-noise lattice uses the lowbias32 hash of
// (x, z, octave, seed). Generation uses only IEEE arithmetic, sqrtf and the host libm, so a scene
// is byte-identical on every run of the same build (pinned by scene_hash tests).
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>
#include "scene_gen.hpp"
#include "wf/rng.hpp"
#include "wf/scene.hpp"

namespace wfb {
namespace {

using wf::Vec3;

struct SplitMix64 {
    uint64_t state;
    uint64_t next() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    float uniform() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
    float uniform(float lo, float hi) { return lo + (hi - lo) * uniform(); }
};

wf::Material lambert(Vec3 albedo) {
    wf::Material m{};
    m.type = wf::kLambert;
    m.ior = 1.0f;
    m.albedo = albedo;
    return m;
}

wf::Material emitter(float e) {
    wf::Material m{};
    m.type = wf::kEmissive;
    m.ior = 1.0f;
    m.emission = Vec3{e, e, e};
    return m;
}

int add_vertex(wf::Scene& s, Vec3 v) {
    s.vertices.push_back(v);
    return (int)s.vertices.size() - 1;
}

// Quad a-b-c-d (counter-clockwise seen from the front) as two triangles.
void add_quad(wf::Scene& s, Vec3 a, Vec3 b, Vec3 c, Vec3 d, int material) {
    const int ia = add_vertex(s, a), ib = add_vertex(s, b), ic = add_vertex(s, c), id = add_vertex(s, d);
    s.triangles.push_back(wf::Triangle{ia, ib, ic, material});
    s.triangles.push_back(wf::Triangle{ia, ic, id, material});
}

// Axis-aligned box of half extents (hx, hy, hz) rotated by `deg` about +y, base on y = base_y.
void add_box(wf::Scene& s, Vec3 centre, float hx, float hy, float hz, float deg, int material) {
    const float rad = deg * (wf::kPi / 180.0f);
    const float c = cosf(rad), sn = sinf(rad);
    auto P = [&](float x, float y, float z) {
        return Vec3{centre.x + c * x + sn * z, centre.y + y, centre.z - sn * x + c * z};
    };
    const Vec3 p000 = P(-hx, -hy, -hz), p100 = P(hx, -hy, -hz), p110 = P(hx, hy, -hz),
               p010 = P(-hx, hy, -hz), p001 = P(-hx, -hy, hz), p101 = P(hx, -hy, hz),
               p111 = P(hx, hy, hz), p011 = P(-hx, hy, hz);
    add_quad(s, p001, p101, p111, p011, material);  // +z
    add_quad(s, p100, p000, p010, p110, material);  // -z
    add_quad(s, p101, p100, p110, p111, material);  // +x
    add_quad(s, p000, p001, p011, p010, material);  // -x
    add_quad(s, p011, p111, p110, p010, material);  // +y
    add_quad(s, p000, p100, p101, p001, material);  // -y
}

wf::Scene cornell36() {
    wf::Scene s;
    s.name = "cornell36";
    s.materials = {lambert({0.73f, 0.73f, 0.73f}), lambert({0.65f, 0.05f, 0.05f}),
                   lambert({0.12f, 0.45f, 0.15f}), emitter(15.0f)};
    const int grey = 0, red = 1, green = 2, light = 3;
    // Unit box [0,1]^3 open towards +z.
    add_quad(s, {0, 0, 1}, {1, 0, 1}, {1, 0, 0}, {0, 0, 0}, grey);  // floor (normal +y)
    add_quad(s, {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}, grey);  // ceiling (normal -y)
    add_quad(s, {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, grey);  // back wall (normal +z)
    add_quad(s, {0, 0, 1}, {0, 0, 0}, {0, 1, 0}, {0, 1, 1}, red);   // left wall (normal +x)
    add_quad(s, {1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0}, green); // right wall (normal -x)
    add_box(s, {0.33f, 0.30f, 0.35f}, 0.15f, 0.30f, 0.15f, 18.0f, grey);   // tall box
    add_box(s, {0.66f, 0.15f, 0.63f}, 0.15f, 0.15f, 0.15f, -18.0f, grey);  // short box
    const float y = 0.999f;
    add_quad(s, {0.38f, y, 0.38f}, {0.62f, y, 0.38f}, {0.62f, y, 0.62f}, {0.38f, y, 0.62f}, light);
    s.env = Vec3{0, 0, 0};
    s.camera = wf::Camera{{0.5f, 0.5f, 2.2f}, {0.5f, 0.5f, 0.0f}, {0, 1, 0}, 40.0f};
    return s;
}

// Level-n icosphere on the unit sphere: 20 * 4^n triangles, 10 * 4^n + 2 vertices.
void unit_icosphere(int levels, std::vector<Vec3>* verts, std::vector<int>* tris) {
    const float t = (1.0f + sqrtf(5.0f)) * 0.5f;
    std::vector<Vec3> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                           {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (Vec3& p : v) p = wf::normalize(p);
    std::vector<int> f = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                          11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                          3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (int l = 0; l < levels; ++l) {
        std::vector<int> nf;
        std::vector<std::pair<uint64_t, int>> cache;  // (edge key, midpoint index), small scenes
        auto midpoint = [&](int a, int b) {
            const uint64_t key = a < b ? ((uint64_t)a << 32 | (uint32_t)b) : ((uint64_t)b << 32 | (uint32_t)a);
            for (const auto& e : cache)
                if (e.first == key) return e.second;
            v.push_back(wf::normalize((v[a] + v[b]) * 0.5f));
            cache.emplace_back(key, (int)v.size() - 1);
            return (int)v.size() - 1;
        };
        for (size_t i = 0; i < f.size(); i += 3) {
            const int a = f[i], b = f[i + 1], c = f[i + 2];
            const int ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            nf.insert(nf.end(), {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca});
        }
        f.swap(nf);
    }
    *verts = v;
    *tris = f;
}

wf::Scene icospheres(uint32_t seed) {
    wf::Scene s;
    s.name = "icospheres";
    SplitMix64 rng{seed};
    std::vector<Vec3> uv;
    std::vector<int> ut;
    unit_icosphere(2, &uv, &ut);
    s.materials.push_back(lambert({0.5f, 0.5f, 0.5f}));  // ground
    s.materials.push_back(emitter(8.0f));                // overhead light
    add_quad(s, {-12, 0, 12}, {12, 0, 12}, {12, 0, -12}, {-12, 0, -12}, 0);
    add_quad(s, {-5, 9, -5}, {5, 9, -5}, {5, 9, 5}, {-5, 9, 5}, 1);
    for (int k = 0; k < 512; ++k) {
        const float r = rng.uniform(0.2f, 0.6f);
        const float cx = rng.uniform(-10.0f, 10.0f);
        const float cz = rng.uniform(-10.0f, 10.0f);
        const float pick = rng.uniform();
        wf::Material m{};
        m.ior = 1.0f;
        if (pick < 1.0f / 3.0f) {
            m.type = wf::kLambert;
            const float a = rng.uniform(), b = rng.uniform(), c = rng.uniform();
            m.albedo = Vec3{a, b, c};
        } else if (pick < 2.0f / 3.0f) {
            m.type = wf::kMetal;
            const float a = rng.uniform(0.5f, 1.0f), b = rng.uniform(0.5f, 1.0f), c = rng.uniform(0.5f, 1.0f);
            m.albedo = Vec3{a, b, c};
            m.pad0 = rng.uniform(0.0f, 0.5f);  // roughness (stored, not shaded)
        } else {
            m.type = wf::kDielectric;
            m.ior = 1.5f;
            m.albedo = Vec3{1.0f, 1.0f, 1.0f};
        }
        s.materials.push_back(m);
        const int mat = (int)s.materials.size() - 1;
        const int base = (int)s.vertices.size();
        const Vec3 c{cx, r, cz};
        for (const Vec3& p : uv) s.vertices.push_back(c + p * r);
        for (size_t i = 0; i < ut.size(); i += 3)
            s.triangles.push_back(wf::Triangle{base + ut[i], base + ut[i + 1], base + ut[i + 2], mat});
    }
    s.env = Vec3{0, 0, 0};
    s.camera = wf::Camera{{0.0f, 6.0f, 17.0f}, {0.0f, 0.5f, 0.0f}, {0, 1, 0}, 50.0f};
    return s;
}

float lattice(int x, int z, int octave, uint32_t seed) {
    const uint32_t h = wf::hash_u32((uint32_t)x * 0x8da6b343U ^ (uint32_t)z * 0xd8163841U ^
                                    (uint32_t)octave * 0xcb1ab31fU ^ wf::hash_u32(seed));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// Smoothstep-interpolated value noise in [0, 1).
float value_noise(float x, float z, int octave, uint32_t seed) {
    const float fx = floorf(x), fz = floorf(z);
    const int ix = (int)fx, iz = (int)fz;
    float tx = x - fx, tz = z - fz;
    tx = tx * tx * (3.0f - 2.0f * tx);
    tz = tz * tz * (3.0f - 2.0f * tz);
    const float a = lattice(ix, iz, octave, seed), b = lattice(ix + 1, iz, octave, seed);
    const float c = lattice(ix, iz + 1, octave, seed), d = lattice(ix + 1, iz + 1, octave, seed);
    const float ab = a + (b - a) * tx, cd = c + (d - c) * tx;
    return ab + (cd - ab) * tz;
}

wf::Scene heightfield(uint32_t seed) {
    wf::Scene s;
    s.name = "heightfield";
    const int n = 1024;
    const float extent = 20.0f, half = extent * 0.5f;
    const float amp = 0.15f * extent;
    const int bands = 8;
    const Vec3 green{0.15f, 0.45f, 0.10f}, brown{0.45f, 0.30f, 0.15f}, white{0.90f, 0.90f, 0.90f};
    for (int b = 0; b < bands; ++b) {
        const float t = (b + 0.5f) / bands;
        const Vec3 col = t < 0.5f ? green + (brown - green) * (t * 2.0f) : brown + (white - brown) * ((t - 0.5f) * 2.0f);
        s.materials.push_back(lambert(col));
    }
    s.materials.push_back(emitter(20.0f));
    const int sun = bands;
    std::vector<float> h((size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const float u = (float)i / (float)(n - 1), v = (float)j / (float)(n - 1);
            float sum = 0.0f, norm = 0.0f, a = 1.0f, f = 4.0f;
            for (int o = 0; o < 6; ++o) {
                sum += a * value_noise(u * f, v * f, o, seed);
                norm += a;
                a *= 0.5f;
                f *= 2.0f;
            }
            h[(size_t)j * n + i] = sum / norm;
        }
    s.vertices.reserve((size_t)n * n + 4);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const float x = -half + extent * ((float)i / (float)(n - 1));
            const float z = -half + extent * ((float)j / (float)(n - 1));
            s.vertices.push_back(Vec3{x, amp * h[(size_t)j * n + i], z});
        }
    s.triangles.reserve((size_t)2 * (n - 1) * (n - 1) + 2);
    for (int j = 0; j + 1 < n; ++j)
        for (int i = 0; i + 1 < n; ++i) {
            const int a = j * n + i, b = a + 1, c = a + n, d = c + 1;
            const float hc = (h[a] + h[b] + h[c] + h[d]) * 0.25f;
            int band = (int)(hc * bands);
            band = band < 0 ? 0 : (band >= bands ? bands - 1 : band);
            s.triangles.push_back(wf::Triangle{a, c, b, band});  // normal +y
            s.triangles.push_back(wf::Triangle{b, c, d, band});
        }
    // Distant sun quad facing the terrain.
    add_quad(s, {-40, 60, -80}, {-20, 60, -80}, {-20, 40, -80}, {-40, 40, -80}, sun);
    s.env = Vec3{1.0f, 1.0f, 1.0f};
    s.camera = wf::Camera{{0.0f, 9.0f, 15.0f}, {0.0f, 1.0f, 0.0f}, {0, 1, 0}, 50.0f};
    return s;
}

}  // namespace

wf::Scene make_config_scene(const std::string& name, int width, int height, uint32_t seed,
                            int sah_bins) {
    if (width <= 0 || height <= 0) throw std::invalid_argument("scene resolution must be positive");
    wf::Scene s;
    if (name == "cornell36") s = cornell36();
    else if (name == "icospheres") s = icospheres(seed);
    else if (name == "heightfield") s = heightfield(seed);
    else throw std::invalid_argument("unknown scene: " + name);
    s.width = width;
    s.height = height;
    wf::finalize_scene_bins(s, sah_bins);
    return s;
}

wf::Camera orbit_camera(const wf::Scene& scene, float azimuth_deg, float elevation_deg) {
    const Vec3 target = scene.camera.look_at;
    const float dist = wf::length(scene.camera.position - target);
    const float az = azimuth_deg * (wf::kPi / 180.0f), el = elevation_deg * (wf::kPi / 180.0f);
    const Vec3 dir{cosf(el) * sinf(az), sinf(el), cosf(el) * cosf(az)};
    wf::Camera c = scene.camera;
    c.position = target + dir * dist;
    return c;
}

}  // namespace wfb
