// Primitive intersection and the stackless skip-link BVH traversal over a SceneView.
//
// API surface of WVM/include/wf/bvh.hpp:25-129. The per-primitive tests are written once as
// "core" functions on plain values (sphere centre/radius; triangle p0 and the edges e1, e2) so the
// device engine can feed them from its own packed layout: e1 = p1 - p0 and e2 = p2 - p0 are single
// IEEE subtractions, so precomputing them on the host gives the same bits as computing them per ray.
#pragma once
#include "wf/math.hpp"
#include "wf/scene.hpp"

namespace wf {

// Sphere test with the projected-distance discriminant: w = oc - d (oc.d / d.d) is the offset of
// the centre from the ray line, so disc = r^2 - |w|^2 does not cancel catastrophically for small
// or distant spheres (Haines et al., Ray Tracing Gems ch. 7). Nearest root in (tmin, tmax).
WF_HD bool hit_sphere_core(Vec3 center, float radius, const Ray& r, float* t_out) {
    const Vec3 oc = r.o - center;
    const float a = dot(r.d, r.d);
    const float b = dot(oc, r.d);
    const Vec3 w = oc - r.d * (b / a);
    const float disc = radius * radius - dot(w, w);
    if (disc < 0.0f) return false;
    const float mid = -b / a;
    const float sq = sqrtf(disc / a);
    float t = mid - sq;
    if (!(t > r.tmin && t < r.tmax)) {
        t = mid + sq;
        if (!(t > r.tmin && t < r.tmax)) return false;
    }
    *t_out = t;
    return true;
}

// Moller-Trumbore with precomputed edges; (u, v) are the barycentrics of p1 and p2.
WF_HD bool hit_triangle_core(Vec3 p0, Vec3 e1, Vec3 e2, const Ray& r, float* t_out, float* u_out,
                             float* v_out) {
    const Vec3 pv = cross(r.d, e2);
    const float det = dot(e1, pv);
    if (det == 0.0f) return false;
    const float inv = 1.0f / det;
    const Vec3 tv = r.o - p0;
    const float u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const Vec3 qv = cross(tv, e1);
    const float v = dot(r.d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    const float t = dot(e2, qv) * inv;
    if (!(t > r.tmin && t < r.tmax)) return false;
    *t_out = t;
    *u_out = u;
    *v_out = v;
    return true;
}

WF_HD bool hit_sphere(const Sphere& s, const Ray& r, float* t_out) {
    return hit_sphere_core(s.center, s.radius, r, t_out);
}

WF_HD bool hit_triangle(Vec3 p0, Vec3 p1, Vec3 p2, const Ray& r, float* t_out, float* u_out,
                        float* v_out) {
    return hit_triangle_core(p0, p1 - p0, p2 - p0, r, t_out, u_out, v_out);
}

// Slab test on [tmin, tmax]. The compare-and-swap and the two ternary clamps are kept literally:
// a NaN slab distance (origin on a slab plane with a zero direction component) leaves t0/t1
// unchanged, which plain min/max would not reproduce (hit_box_minmax maps NaN first).
WF_HD bool hit_box(Vec3 lo, Vec3 hi, Vec3 o, Vec3 inv_d, float tmin, float tmax) {
    float t0 = tmin, t1 = tmax;
    float tn = (lo.x - o.x) * inv_d.x, tf = (hi.x - o.x) * inv_d.x;
    if (tn > tf) { const float s = tn; tn = tf; tf = s; }
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
    if (t0 > t1) return false;
    tn = (lo.y - o.y) * inv_d.y;
    tf = (hi.y - o.y) * inv_d.y;
    if (tn > tf) { const float s = tn; tn = tf; tf = s; }
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
    if (t0 > t1) return false;
    tn = (lo.z - o.z) * inv_d.z;
    tf = (hi.z - o.z) * inv_d.z;
    if (tn > tf) { const float s = tn; tn = tf; tf = s; }
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
    return t0 <= t1;
}

// hit_box on min/max operations, with the same result for every input, NaN included (the GPU
// traversal's box test: fminf/fmaxf are one instruction each, a compare-and-select two). In
// hit_box the early exits and the final t0 <= t1 agree once t0 > t1, so they can go. Per axis, a
// NaN slab distance (a NaN factor, or 0 * inf when the origin lies on the slab plane of an axis
// the ray is parallel to) is never swapped, so a NaN tn reaches only the t0 clamp and a NaN tf
// only the t1 clamp, and a clamp with a NaN operand leaves t0/t1 unchanged. Here a NaN tn reads as
// -inf and a NaN tf as +inf (fmaxf/fminf return their non-NaN operand), which the clamps ignore in
// the same way; with no NaN left, compare-and-select and fminf/fmaxf pick the same value up to the
// sign of a zero, which no comparison sees. t0 starts at tmin, never NaN; a NaN tmax leaves
// hit_box's t1 NaN and its result false, so tmax joins last, by compare-and-select.
WF_HD bool hit_box_minmax(Vec3 lo, Vec3 hi, Vec3 o, Vec3 inv_d, float tmin, float tmax) {
    const float xn = fmaxf((lo.x - o.x) * inv_d.x, -INFINITY), xf = fminf((hi.x - o.x) * inv_d.x, INFINITY);
    const float yn = fmaxf((lo.y - o.y) * inv_d.y, -INFINITY), yf = fminf((hi.y - o.y) * inv_d.y, INFINITY);
    const float zn = fmaxf((lo.z - o.z) * inv_d.z, -INFINITY), zf = fminf((hi.z - o.z) * inv_d.z, INFINITY);
    const float t0 = fmaxf(fmaxf(fminf(xn, xf), fminf(yn, yf)), fmaxf(fminf(zn, zf), tmin));
    const float b = fminf(fminf(fmaxf(xn, xf), fmaxf(yn, yf)), fmaxf(zn, zf));
    const float t1 = b < tmax ? b : tmax;
    return t0 <= t1;
}

WF_HD bool hit_prim(const SceneView& s, int prim, const Ray& r, float* t, float* u, float* v) {
    if (prim < s.n_spheres) {
        *u = 0.0f;
        *v = 0.0f;
        return hit_sphere(s.spheres[prim], r, t);
    }
    const Triangle& tri = s.triangles[prim - s.n_spheres];
    return hit_triangle(s.vertices[tri.i0], s.vertices[tri.i1], s.vertices[tri.i2], r, t, u, v);
}

// Closest hit (or, with anyhit, the first hit found) by stackless preorder traversal: descend to
// N+1 on a box hit, follow `skip` on a miss or after a leaf. A primitive replaces the current hit
// only when strictly nearer, so among equal t the earliest one in preorder wins.
WF_HD bool intersect(const SceneView& s, Ray r, HitRecord* h, bool anyhit = false) {
    h->t = r.tmax;
    h->prim = -1;
    h->u = 0.0f;
    h->v = 0.0f;
    const Vec3 inv_d{1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z};
    int n = 0;
    while (n >= 0 && n < s.n_nodes) {
        const BvhNode& node = s.nodes[n];
        if (!hit_box(node.lo, node.hi, r.o, inv_d, r.tmin, r.tmax)) {
            n = node.skip;
            continue;
        }
        if (node.prim_count <= 0) {
            n = n + 1;
            continue;
        }
        for (int i = 0; i < node.prim_count; ++i) {
            const int p = s.prim_order[node.prim_start + i];
            float t, u, v;
            if (hit_prim(s, p, r, &t, &u, &v)) {
                r.tmax = t;
                h->t = t;
                h->prim = p;
                h->u = u;
                h->v = v;
                if (anyhit) return true;
            }
        }
        n = node.skip;
    }
    return h->prim >= 0;
}

// Test oracle: every primitive in id order with the same strictly-nearer rule.
WF_HD bool intersect_bruteforce(const SceneView& s, Ray r, HitRecord* h) {
    h->t = r.tmax;
    h->prim = -1;
    h->u = 0.0f;
    h->v = 0.0f;
    const int total = s.n_spheres + s.n_triangles;
    for (int p = 0; p < total; ++p) {
        float t, u, v;
        if (hit_prim(s, p, r, &t, &u, &v)) {
            r.tmax = t;
            h->t = t;
            h->prim = p;
            h->u = u;
            h->v = v;
        }
    }
    return h->prim >= 0;
}

}  // namespace wf
