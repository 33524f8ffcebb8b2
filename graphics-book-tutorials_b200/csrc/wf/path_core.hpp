// The path-space estimator: camera rays, surface interaction, next-event estimation with MIS,
// Lambertian / mirror / dielectric scattering and Russian roulette.
//
// API surface and arithmetic of WVM/include/wf/path_core.hpp:11-304. Each step is a template
// over the scene representation S so that the same source -- hence the same sequence of IEEE
// operations -- runs on the reference SceneView (host or device) and on this engine's packed
// device scene (csrc/dev_scene.cuh). A representation provides the members n_spheres,
// n_triangles, n_lights, env, camera, width, height and the accessor overloads
//   load_sphere(s, i) -> Sphere          load_material(s, m) -> Material
//   tri_material(s, t) -> int            tri_normal(s, t) -> normalize(cross(p1-p0, p2-p0))
//   prim_area(s, prim) -> float          load_light(s, idx) -> LightGeom
// Values such as triangle normals and areas may be precomputed by a representation as long as
// they are computed with the same operations (see math.hpp for why that is bit-exact).
#pragma once
#include "wf/bvh.hpp"
#include "wf/math.hpp"
#include "wf/rng.hpp"
#include "wf/scene.hpp"

namespace wf {

constexpr float kRayEps = 1e-4f;

// 76 bytes, reference layout (WVM/include/wf/path_core.hpp:13-21).
struct PathState {
    Ray ray;
    Vec3 throughput;
    Vec3 L;
    int depth;
    int specular;    // 1 after a delta event and at the camera
    float prev_pdf;  // solid-angle pdf of the last BSDF sample, 0 after a delta event
    PathKey key;
};

struct Surface {
    Vec3 p;
    Vec3 n;      // geometric normal facing the incoming ray
    Vec3 n_out;  // outward geometric normal (sphere: radial, triangle: winding)
    int inside;  // ray arrived from behind n_out
    int material;
};

struct LightSample {
    Vec3 p;
    Vec3 n;
    float pdf_solid;  // includes the 1/n_lights pick probability; 0 marks an invalid sample
    Vec3 Le;
};

// Geometry of one light, as needed by sample_light.
struct LightGeom {
    int prim;
    int is_sphere;
    int material;
    float area;
    Vec3 a;  // sphere centre, or triangle p0
    Vec3 b;  // triangle p1
    Vec3 c;  // triangle p2
    Vec3 n;  // triangle normal normalize(cross(p1-p0, p2-p0))
    float radius;
};

// ---- SceneView accessors (reference representation) ----
WF_HD Sphere load_sphere(const SceneView& s, int i) { return s.spheres[i]; }
WF_HD Material load_material(const SceneView& s, int m) { return s.materials[m]; }
WF_HD int tri_material(const SceneView& s, int t) { return s.triangles[t].material; }
WF_HD Vec3 tri_normal(const SceneView& s, int t) {
    const Triangle& tr = s.triangles[t];
    const Vec3 e1 = s.vertices[tr.i1] - s.vertices[tr.i0];
    const Vec3 e2 = s.vertices[tr.i2] - s.vertices[tr.i0];
    return normalize(cross(e1, e2));
}
WF_HD float prim_area(const SceneView& s, int prim) {
    if (prim < s.n_spheres) {
        const float r = s.spheres[prim].radius;
        return 4.0f * kPi * r * r;
    }
    const Triangle& tr = s.triangles[prim - s.n_spheres];
    const Vec3 e1 = s.vertices[tr.i1] - s.vertices[tr.i0];
    const Vec3 e2 = s.vertices[tr.i2] - s.vertices[tr.i0];
    return 0.5f * length(cross(e1, e2));
}
WF_HD LightGeom load_light(const SceneView& s, int idx) {
    LightGeom g;
    g.prim = s.lights[idx].prim;
    g.area = prim_area(s, g.prim);
    g.is_sphere = g.prim < s.n_spheres ? 1 : 0;
    if (g.is_sphere) {
        const Sphere& sp = s.spheres[g.prim];
        g.a = sp.center;
        g.radius = sp.radius;
        g.material = sp.material;
        g.b = g.c = g.n = Vec3{0.0f, 0.0f, 0.0f};
    } else {
        const Triangle& tr = s.triangles[g.prim - s.n_spheres];
        g.a = s.vertices[tr.i0];
        g.b = s.vertices[tr.i1];
        g.c = s.vertices[tr.i2];
        g.n = normalize(cross(g.b - g.a, g.c - g.a));
        g.material = tr.material;
        g.radius = 0.0f;
    }
    return g;
}
WF_HD int prim_material(const SceneView& s, int prim) {
    return prim < s.n_spheres ? s.spheres[prim].material : s.triangles[prim - s.n_spheres].material;
}

// ---- estimator steps ----

// Veach's power heuristic with beta = 2.
WF_HD float power_heuristic(float a, float b) {
    const float a2 = a * a, b2 = b * b;
    const float sum = a2 + b2;
    return sum > 0.0f ? a2 / sum : 0.0f;
}

// Jittered pinhole ray through pixel (px, py); image row 0 is the top row.
template <class S>
WF_HD Ray camera_ray(const S& s, int px, int py, PathKey key) {
    const float jx = rng(key, 0, kDimPixelX);
    const float jy = rng(key, 0, kDimPixelY);
    const float u = ((float)px + jx) / (float)s.width;
    const float v = ((float)(s.height - 1 - py) + jy) / (float)s.height;
    const Vec3 target = s.camera.lower_left + s.camera.horizontal * u + s.camera.vertical * v;
    Ray r;
    r.o = s.camera.origin;
    r.d = normalize(target - s.camera.origin);
    r.tmin = kRayEps;
    r.tmax = kInf;
    return r;
}

template <class S>
WF_HD PathState init_path(const S& s, int px, int py, uint32_t sample, uint32_t seed) {
    PathState ps;
    ps.key = make_path_key(seed, (uint32_t)(py * s.width + px), sample);
    ps.ray = camera_ray(s, px, py, ps.key);
    ps.throughput = Vec3{1.0f, 1.0f, 1.0f};
    ps.L = Vec3{0.0f, 0.0f, 0.0f};
    ps.depth = 0;
    ps.specular = 1;
    ps.prev_pdf = 0.0f;
    return ps;
}

template <class S>
WF_HD Surface make_surface(const S& s, const Ray& ray, const HitRecord& h) {
    Surface f;
    f.p = ray.o + ray.d * h.t;
    if (h.prim < s.n_spheres) {
        const Sphere sp = load_sphere(s, h.prim);
        f.n_out = (f.p - sp.center) / sp.radius;
        f.material = sp.material;
    } else {
        const int t = h.prim - s.n_spheres;
        f.n_out = tri_normal(s, t);
        f.material = tri_material(s, t);
    }
    f.inside = dot(f.n_out, ray.d) > 0.0f ? 1 : 0;
    f.n = f.inside ? -f.n_out : f.n_out;
    return f;
}

// Uniform area sample on one uniformly picked light, converted to a solid-angle pdf at `from`.
template <class S>
WF_HD LightSample sample_light(const S& s, Vec3 from, PathKey key, uint32_t depth) {
    LightSample ls;
    ls.pdf_solid = 0.0f;
    ls.p = from;
    ls.n = Vec3{0.0f, 0.0f, 1.0f};
    ls.Le = Vec3{0.0f, 0.0f, 0.0f};
    if (s.n_lights <= 0) return ls;
    int idx = (int)(rng(key, depth, kDimLightPick) * (float)s.n_lights);
    if (idx >= s.n_lights) idx = s.n_lights - 1;
    const LightGeom g = load_light(s, idx);
    const float u1 = rng(key, depth, kDimLightU), u2 = rng(key, depth, kDimLightV);
    if (g.is_sphere) {
        // Uniform direction on the unit sphere (z = 1 - 2 u1, phi = 2 pi u2).
        const float z = 1.0f - 2.0f * u1;
        const float rxy = sqrtf(fmaxf3(0.0f, 1.0f - z * z));
        const float phi = 2.0f * kPi * u2;
        const Vec3 dir{rxy * cosf(phi), rxy * sinf(phi), z};
        ls.n = dir;
        ls.p = g.a + dir * g.radius;
    } else {
        // Uniform barycentrics by the square-root warp (Shirley).
        const float su = sqrtf(u1);
        const float b0 = 1.0f - su, b1 = u2 * su;
        ls.p = g.a * (1.0f - b0 - b1) + g.b * b0 + g.c * b1;
        ls.n = g.n;
    }
    ls.Le = load_material(s, g.material).emission;
    const Vec3 d = ls.p - from;
    const float dist2 = length2(d);
    const float dist = sqrtf(dist2);
    if (dist <= 0.0f) return ls;
    const float cosl = fabsf(dot(ls.n, d)) / dist;
    if (cosl <= 1e-6f) return ls;
    ls.pdf_solid = (dist2 / (cosl * g.area)) / (float)s.n_lights;
    return ls;
}

// Light-sampling pdf (solid angle, with pick probability) of a BSDF-sampled ray that hit light `prim`.
template <class S>
WF_HD float light_pdf_at_hit(const S& s, int prim, float t, Vec3 dir, Vec3 n_out) {
    const float cosl = fabsf(dot(n_out, dir));
    if (cosl <= 1e-6f) return 0.0f;
    return ((t * t) / (cosl * prim_area(s, prim))) / (float)s.n_lights;
}

// Miss / emission (MIS-weighted after a non-delta bounce) / termination. Returns the material type
// to shade (kLambert, kMetal, kDielectric) or -1 when the path ends here.
template <class S>
WF_HD int classify(const S& s, PathState& ps, const HitRecord& h, int max_depth, Surface* surf) {
    if (h.prim < 0) {
        ps.L += ps.throughput * s.env;
        return -1;
    }
    *surf = make_surface(s, ps.ray, h);
    const Material m = load_material(s, surf->material);
    if (m.emission.x > 0.0f || m.emission.y > 0.0f || m.emission.z > 0.0f) {
        float w = 1.0f;
        if (!ps.specular && ps.prev_pdf > 0.0f) {
            const float pl = light_pdf_at_hit(s, h.prim, h.t, ps.ray.d, surf->n_out);
            w = power_heuristic(ps.prev_pdf, pl);
        }
        ps.L += ps.throughput * m.emission * w;
    }
    if (m.type == kEmissive) return -1;
    if (ps.depth >= max_depth) return -1;
    return m.type;
}

// Survival probability clamp(max throughput, 0.05, 0.95) from depth 3 on; survivors are reweighted.
WF_HD bool russian_roulette(PathState& ps) {
    if (ps.depth < 3) return true;
    const float q = clampf(max_component(ps.throughput), 0.05f, 0.95f);
    if (rng(ps.key, (uint32_t)ps.depth, kDimRoulette) >= q) return false;
    ps.throughput = ps.throughput / q;
    return true;
}

WF_HD void set_next_ray(PathState& ps, Vec3 origin, Vec3 dir) {
    ps.ray.o = origin;
    ps.ray.d = dir;
    ps.ray.tmin = kRayEps;
    ps.ray.tmax = kInf;
}

// Lambertian: next-event estimation (the shadow ray is returned, not traced), cosine-weighted
// scattering, roulette. The caller adds *contrib to ps.L if the shadow ray is unoccluded, before
// the next classify.
template <class S>
WF_HD bool shade_lambert(const S& s, PathState& ps, const Surface& f, Ray* shadow, Vec3* contrib,
                         int* has_shadow) {
    const Material m = load_material(s, f.material);
    const uint32_t d = (uint32_t)ps.depth;
    *has_shadow = 0;
    const Vec3 org = f.p + f.n * kRayEps;
    if (s.n_lights > 0) {
        const LightSample ls = sample_light(s, org, ps.key, d);
        if (ls.pdf_solid > 0.0f) {
            const Vec3 to = ls.p - org;
            const float dist = length(to);
            const Vec3 wi = to / dist;
            const float cos_s = dot(f.n, wi);
            if (cos_s > 0.0f) {
                const float pb = cos_s * kInvPi;
                const float w = power_heuristic(ls.pdf_solid, pb);
                *contrib = ps.throughput * m.albedo * ls.Le * (cos_s * kInvPi * w / ls.pdf_solid);
                shadow->o = org;
                shadow->d = wi;
                shadow->tmin = kRayEps;
                shadow->tmax = dist * (1.0f - 1e-3f);
                *has_shadow = 1;
            }
        }
    }
    // Cosine-weighted direction by Malley's method (uniform disk lifted to the hemisphere).
    const float u1 = rng(ps.key, d, kDimBsdfU), u2 = rng(ps.key, d, kDimBsdfV);
    const float r = sqrtf(u1), phi = 2.0f * kPi * u2;
    Vec3 t, b;
    make_basis(f.n, &t, &b);
    const float z = sqrtf(fmaxf3(0.0f, 1.0f - u1));
    const Vec3 dir = normalize(t * (r * cosf(phi)) + b * (r * sinf(phi)) + f.n * z);
    ps.throughput = ps.throughput * m.albedo;
    ps.specular = 0;
    ps.prev_pdf = dot(dir, f.n) * kInvPi;
    ps.depth += 1;
    set_next_ray(ps, org, dir);
    return russian_roulette(ps);
}

// Tinted perfect mirror.
template <class S>
WF_HD bool shade_metal(const S& s, PathState& ps, const Surface& f) {
    const Material m = load_material(s, f.material);
    const Vec3 dir = reflect(ps.ray.d, f.n);
    if (dot(dir, f.n) <= 0.0f) return false;
    ps.throughput = ps.throughput * m.albedo;
    ps.specular = 1;
    ps.prev_pdf = 0.0f;
    ps.depth += 1;
    set_next_ray(ps, f.p + f.n * kRayEps, normalize(dir));
    return russian_roulette(ps);
}

// Unpolarised Fresnel reflectance of a smooth dielectric interface; cos_i >= 0 against the
// facing normal. Returns 1 under total internal reflection.
WF_HD float fresnel_dielectric(float cos_i, float eta_i, float eta_t) {
    const float sin_t = eta_i / eta_t * sqrtf(fmaxf3(0.0f, 1.0f - cos_i * cos_i));
    if (sin_t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(fmaxf3(0.0f, 1.0f - sin_t * sin_t));
    const float r_par = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
    const float r_perp = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
    return 0.5f * (r_par * r_par + r_perp * r_perp);
}

// Smooth dielectric: reflect with probability F, otherwise refract (Snell).
template <class S>
WF_HD bool shade_dielectric(const S& s, PathState& ps, const Surface& f) {
    const Material m = load_material(s, f.material);
    const float eta_i = f.inside ? m.ior : 1.0f;
    const float eta_t = f.inside ? 1.0f : m.ior;
    const float cos_i = clampf(-dot(ps.ray.d, f.n), 0.0f, 1.0f);
    const float F = fresnel_dielectric(cos_i, eta_i, eta_t);
    const float u = rng(ps.key, (uint32_t)ps.depth, kDimDielectric);
    Vec3 org, dir;
    if (u < F) {
        dir = reflect(ps.ray.d, f.n);
        org = f.p + f.n * kRayEps;
    } else {
        const float eta = eta_i / eta_t;
        const float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
        const float cos_t = sqrtf(fmaxf3(0.0f, 1.0f - sin2_t));
        dir = ps.ray.d * eta + f.n * (eta * cos_i - cos_t);
        org = f.p - f.n * kRayEps;
    }
    ps.throughput = ps.throughput * m.albedo;
    ps.specular = 1;
    ps.prev_pdf = 0.0f;
    ps.depth += 1;
    set_next_ray(ps, org, normalize(dir));
    return russian_roulette(ps);
}

// Whole path of one (pixel, sample) over a SceneView: the reference's trace_path
// (WVM/include/wf/path_core.hpp:279-304).
WF_HD Vec3 trace_path(const SceneView& s, int px, int py, uint32_t sample, uint32_t seed,
                      int max_depth) {
    PathState ps = init_path(s, px, py, sample, seed);
    for (;;) {
        HitRecord h;
        intersect(s, ps.ray, &h);
        Surface f;
        const int mat = classify(s, ps, h, max_depth, &f);
        if (mat < 0) break;
        bool alive;
        if (mat == kLambert) {
            Ray sh;
            Vec3 c;
            int has;
            alive = shade_lambert(s, ps, f, &sh, &c, &has);
            if (has) {
                HitRecord sh_hit;
                if (!intersect(s, sh, &sh_hit, true)) ps.L += c;
            }
        } else if (mat == kMetal) {
            alive = shade_metal(s, ps, f);
        } else {
            alive = shade_dielectric(s, ps, f);
        }
        if (!alive) break;
    }
    return ps.L;
}

}  // namespace wf
