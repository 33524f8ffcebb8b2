/*
 * ORACLE -- test infrastructure only. Never linked into or called by the engine.
 *
 * A plain-C restatement of the reference path tracer's CPU arm (us-llm-engineer/
 * graphics-book-tutorials, WVM = wavefront-vs-megakernel-path-tracing): counter-based RNG,
 * camera rays, stackless skip-link BVH traversal, the estimator steps with next-event estimation
 * and MIS, and the per-pixel film sums in sample order. Used by tests/ (parity checker),
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg only.
 *
 * Pinned against the reference itself: tests compare this oracle bit-for-bit with the reference's
 * own render_cpu built from its sources (oracle/Makefile -> oracle/_ref/libwfref.so) and with
 * committed golden films produced by that build (tests/golden/make_golden.py).
 *
 * Compiled with -ffp-contract=off (no fused multiply-add) so every float operation rounds as in
 * the reference's CPU arm (WVM/CMakeLists.txt:16-17). Each function cites the reference lines
 * whose arithmetic it restates.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } v3;
typedef struct { v3 o; float tmin; v3 d; float tmax; } ray_t;
typedef struct { uint32_t k0, k1; } pkey;

/* Reference byte layouts (WVM/include/wf/scene.hpp:12-100). */
typedef struct { v3 center; float radius; int material; int pad[3]; } o_sphere;
typedef struct { int i0, i1, i2, material; } o_tri;
typedef struct { int type; float ior, pad0, pad1; v3 albedo; float pad2; v3 emission; float pad3; } o_mat;
typedef struct { v3 lo; int skip; v3 hi; int prim_start, prim_count; int pad[3]; } o_node;
typedef struct { int prim; float area; float pad[2]; } o_light;
typedef struct { float t; int prim; float u, v; } o_hit;

/* Scene handed in by the tests (same field order as the engine's wfb_scene_desc). */
typedef struct {
    const o_sphere* spheres; int n_spheres;
    const v3* vertices;      int n_vertices;
    const o_tri* triangles;  int n_triangles;
    const o_mat* materials;  int n_materials;
    const o_node* nodes;     int n_nodes;
    const int* prim_order;   int n_prim_order;
    const o_light* lights;   int n_lights;
    float env[3];
    float cam_position[3], cam_look_at[3], cam_up[3], cam_vfov_deg;
    int width, height;
} oracle_scene;

typedef struct { v3 origin, lower_left, horizontal, vertical; } rig_t;

static const float PI_F = 3.14159265358979323846f;
static const float INV_PI_F = 0.31830988618379067154f;
static const float INF_F = 3.402823466e+38f;
static const float RAY_EPS = 1e-4f;

/* ---- vector algebra, WVM/include/wf/math.hpp:22-60 ---- */
static v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static v3 mulv(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static v3 muls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 divs(v3 a, float s) { float r = 1.0f / s; return V(a.x * r, a.y * r, a.z * r); }
static float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 cross3(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float len3(v3 a) { return sqrtf(dot3(a, a)); }
static v3 norm3(v3 a) { float l = len3(a); return l > 0.0f ? divs(a, l) : a; }
static float mx(float a, float b) { return a > b ? a : b; }
static float clampf_(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static v3 reflect3(v3 d, v3 n) { return sub(d, muls(n, 2.0f * dot3(d, n))); }
static float lum(v3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

static void basis(v3 n, v3* t, v3* b) {
    float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sign + n.z);
    float c = n.x * n.y * a;
    *t = V(1.0f + sign * n.x * n.x * a, sign * c, -sign * n.x);
    *b = V(c, sign + n.y * n.y * a, -n.y);
}

/* ---- RNG, WVM/include/wf/rng.hpp:8-42 ---- */
static uint32_t hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
static pkey path_key(uint32_t seed, uint32_t pixel, uint32_t sample) {
    uint32_t a = hash32(seed ^ 0x9e3779b9U);
    uint32_t b = hash32(seed + 0x85ebca6bU);
    pkey k;
    k.k0 = hash32(hash32(a + pixel * 0xc2b2ae35U) ^ (sample * 0x27d4eb2fU + 0x165667b1U));
    k.k1 = hash32(hash32(b ^ (pixel * 0x9e3779b1U)) + (sample * 0x85ebca77U + 0xc2b2ae3dU));
    return k;
}
enum { D_PX = 0, D_PY = 1, D_LPICK = 2, D_LU = 3, D_LV = 4, D_BU = 5, D_BV = 6, D_RR = 7, D_DIEL = 8, D_COUNT = 16 };
static float rnd(pkey k, uint32_t depth, uint32_t dim) {
    uint32_t ctr = depth * D_COUNT + dim;
    uint32_t h = hash32(k.k0 ^ hash32(ctr * 0x9e3779b9U + k.k1));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

/* ---- camera rig, WVM/include/wf/scene.hpp:129-141 (host tanf) ---- */
static rig_t make_rig(const oracle_scene* s) {
    v3 pos = V(s->cam_position[0], s->cam_position[1], s->cam_position[2]);
    v3 at = V(s->cam_look_at[0], s->cam_look_at[1], s->cam_look_at[2]);
    v3 up = V(s->cam_up[0], s->cam_up[1], s->cam_up[2]);
    float aspect = (float)s->width / (float)s->height;
    float h = tanf(s->cam_vfov_deg * 0.5f * PI_F / 180.0f);
    v3 w = norm3(sub(pos, at));
    v3 u = norm3(cross3(up, w));
    v3 v = cross3(w, u);
    rig_t r;
    r.origin = pos;
    r.horizontal = muls(u, 2.0f * h * aspect);
    r.vertical = muls(v, 2.0f * h);
    r.lower_left = sub(sub(sub(r.origin, muls(r.horizontal, 0.5f)), muls(r.vertical, 0.5f)), w);
    return r;
}

/* ---- primitives and traversal, WVM/include/wf/bvh.hpp:25-116 ---- */
static int hit_sphere(const o_sphere* s, const ray_t* r, float* t_out) {
    v3 oc = sub(r->o, s->center);
    float a = dot3(r->d, r->d);
    float b = dot3(oc, r->d);
    v3 w = sub(oc, muls(r->d, b / a));
    float disc = s->radius * s->radius - dot3(w, w);
    if (disc < 0.0f) return 0;
    float mid = -b / a;
    float sq = sqrtf(disc / a);
    float t = mid - sq;
    if (!(t > r->tmin && t < r->tmax)) {
        t = mid + sq;
        if (!(t > r->tmin && t < r->tmax)) return 0;
    }
    *t_out = t;
    return 1;
}

static int hit_tri(v3 p0, v3 p1, v3 p2, const ray_t* r, float* t_out, float* u_out, float* v_out) {
    v3 e1 = sub(p1, p0), e2 = sub(p2, p0);
    v3 pv = cross3(r->d, e2);
    float det = dot3(e1, pv);
    if (det == 0.0f) return 0;
    float inv = 1.0f / det;
    v3 tv = sub(r->o, p0);
    float u = dot3(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return 0;
    v3 qv = cross3(tv, e1);
    float v = dot3(r->d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return 0;
    float t = dot3(e2, qv) * inv;
    if (!(t > r->tmin && t < r->tmax)) return 0;
    *t_out = t; *u_out = u; *v_out = v;
    return 1;
}

static int hit_box(v3 lo, v3 hi, v3 o, v3 inv_d, float tmin, float tmax) {
    float t0 = tmin, t1 = tmax, tn, tf, s;
    tn = (lo.x - o.x) * inv_d.x; tf = (hi.x - o.x) * inv_d.x;
    if (tn > tf) { s = tn; tn = tf; tf = s; }
    t0 = tn > t0 ? tn : t0; t1 = tf < t1 ? tf : t1;
    if (t0 > t1) return 0;
    tn = (lo.y - o.y) * inv_d.y; tf = (hi.y - o.y) * inv_d.y;
    if (tn > tf) { s = tn; tn = tf; tf = s; }
    t0 = tn > t0 ? tn : t0; t1 = tf < t1 ? tf : t1;
    if (t0 > t1) return 0;
    tn = (lo.z - o.z) * inv_d.z; tf = (hi.z - o.z) * inv_d.z;
    if (tn > tf) { s = tn; tn = tf; tf = s; }
    t0 = tn > t0 ? tn : t0; t1 = tf < t1 ? tf : t1;
    return t0 <= t1;
}

static int hit_prim(const oracle_scene* s, int p, const ray_t* r, float* t, float* u, float* v) {
    if (p < s->n_spheres) { *u = 0.0f; *v = 0.0f; return hit_sphere(&s->spheres[p], r, t); }
    const o_tri* tr = &s->triangles[p - s->n_spheres];
    return hit_tri(s->vertices[tr->i0], s->vertices[tr->i1], s->vertices[tr->i2], r, t, u, v);
}

static int intersect(const oracle_scene* s, ray_t r, o_hit* h, int anyhit) {
    h->t = r.tmax; h->prim = -1; h->u = 0.0f; h->v = 0.0f;
    v3 inv_d = V(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    int n = 0;
    while (n >= 0 && n < s->n_nodes) {
        const o_node* node = &s->nodes[n];
        if (hit_box(node->lo, node->hi, r.o, inv_d, r.tmin, r.tmax)) {
            if (node->prim_count > 0) {
                for (int i = 0; i < node->prim_count; ++i) {
                    int p = s->prim_order[node->prim_start + i];
                    float t, u, v;
                    if (hit_prim(s, p, &r, &t, &u, &v)) {
                        r.tmax = t; h->t = t; h->prim = p; h->u = u; h->v = v;
                        if (anyhit) return 1;
                    }
                }
                n = node->skip;
            } else {
                n = n + 1;
            }
        } else {
            n = node->skip;
        }
    }
    return h->prim >= 0;
}

/* ---- estimator, WVM/include/wf/path_core.hpp:13-304 ---- */
typedef struct { ray_t ray; v3 thr; v3 L; int depth; int specular; float prev_pdf; pkey key; } pstate;
typedef struct { v3 p, n, n_out; int inside, material; } surf_t;
typedef struct { v3 p, n; float pdf; v3 Le; } lsample;

static float power_h(float a, float b) {
    float a2 = a * a, b2 = b * b, s = a2 + b2;
    return s > 0.0f ? a2 / s : 0.0f;
}

static float prim_area(const oracle_scene* s, int prim) {
    if (prim < s->n_spheres) { float r = s->spheres[prim].radius; return 4.0f * PI_F * r * r; }
    const o_tri* t = &s->triangles[prim - s->n_spheres];
    v3 e1 = sub(s->vertices[t->i1], s->vertices[t->i0]);
    v3 e2 = sub(s->vertices[t->i2], s->vertices[t->i0]);
    return 0.5f * len3(cross3(e1, e2));
}

static ray_t cam_ray(const oracle_scene* s, const rig_t* rig, int px, int py, pkey key) {
    float jx = rnd(key, 0, D_PX), jy = rnd(key, 0, D_PY);
    float u = ((float)px + jx) / (float)s->width;
    float v = ((float)(s->height - 1 - py) + jy) / (float)s->height;
    v3 target = add(add(rig->lower_left, muls(rig->horizontal, u)), muls(rig->vertical, v));
    ray_t r;
    r.o = rig->origin;
    r.d = norm3(sub(target, rig->origin));
    r.tmin = RAY_EPS;
    r.tmax = INF_F;
    return r;
}

static pstate init_path(const oracle_scene* s, const rig_t* rig, int px, int py, uint32_t sample, uint32_t seed) {
    pstate ps;
    ps.key = path_key(seed, (uint32_t)(py * s->width + px), sample);
    ps.ray = cam_ray(s, rig, px, py, ps.key);
    ps.thr = V(1.0f, 1.0f, 1.0f);
    ps.L = V(0.0f, 0.0f, 0.0f);
    ps.depth = 0;
    ps.specular = 1;
    ps.prev_pdf = 0.0f;
    return ps;
}

static surf_t make_surface(const oracle_scene* s, const ray_t* ray, const o_hit* h) {
    surf_t f;
    f.p = add(ray->o, muls(ray->d, h->t));
    if (h->prim < s->n_spheres) {
        const o_sphere* sp = &s->spheres[h->prim];
        f.n_out = divs(sub(f.p, sp->center), sp->radius);
        f.material = sp->material;
    } else {
        const o_tri* t = &s->triangles[h->prim - s->n_spheres];
        v3 e1 = sub(s->vertices[t->i1], s->vertices[t->i0]);
        v3 e2 = sub(s->vertices[t->i2], s->vertices[t->i0]);
        f.n_out = norm3(cross3(e1, e2));
        f.material = t->material;
    }
    f.inside = dot3(f.n_out, ray->d) > 0.0f ? 1 : 0;
    f.n = f.inside ? neg(f.n_out) : f.n_out;
    return f;
}

static lsample sample_light(const oracle_scene* s, v3 from, pkey key, uint32_t depth) {
    lsample ls;
    ls.pdf = 0.0f; ls.p = from; ls.n = V(0, 0, 1); ls.Le = V(0, 0, 0);
    if (s->n_lights <= 0) return ls;
    int idx = (int)(rnd(key, depth, D_LPICK) * (float)s->n_lights);
    if (idx >= s->n_lights) idx = s->n_lights - 1;
    int prim = s->lights[idx].prim;
    float u1 = rnd(key, depth, D_LU), u2 = rnd(key, depth, D_LV);
    float area = prim_area(s, prim);
    if (prim < s->n_spheres) {
        const o_sphere* sp = &s->spheres[prim];
        float z = 1.0f - 2.0f * u1;
        float r = sqrtf(mx(0.0f, 1.0f - z * z));
        float phi = 2.0f * PI_F * u2;
        v3 dir = V(r * cosf(phi), r * sinf(phi), z);
        ls.n = dir;
        ls.p = add(sp->center, muls(dir, sp->radius));
        ls.Le = s->materials[sp->material].emission;
    } else {
        const o_tri* t = &s->triangles[prim - s->n_spheres];
        float su = sqrtf(u1);
        float b0 = 1.0f - su, b1 = u2 * su;
        v3 p0 = s->vertices[t->i0], p1 = s->vertices[t->i1], p2 = s->vertices[t->i2];
        ls.p = add(add(muls(p0, 1.0f - b0 - b1), muls(p1, b0)), muls(p2, b1));
        ls.n = norm3(cross3(sub(p1, p0), sub(p2, p0)));
        ls.Le = s->materials[t->material].emission;
    }
    v3 d = sub(ls.p, from);
    float dist2 = dot3(d, d);
    float dist = sqrtf(dist2);
    if (dist <= 0.0f) return ls;
    float cosl = fabsf(dot3(ls.n, d)) / dist;
    if (cosl <= 1e-6f) return ls;
    ls.pdf = (dist2 / (cosl * area)) / (float)s->n_lights;
    return ls;
}

static float light_pdf_at_hit(const oracle_scene* s, int prim, float t, v3 dir, v3 n_out) {
    float cosl = fabsf(dot3(n_out, dir));
    if (cosl <= 1e-6f) return 0.0f;
    return ((t * t) / (cosl * prim_area(s, prim))) / (float)s->n_lights;
}

static int classify(const oracle_scene* s, pstate* ps, const o_hit* h, int max_depth, surf_t* f) {
    if (h->prim < 0) {
        ps->L = add(ps->L, mulv(ps->thr, V(s->env[0], s->env[1], s->env[2])));
        return -1;
    }
    *f = make_surface(s, &ps->ray, h);
    const o_mat* m = &s->materials[f->material];
    if (m->emission.x > 0.0f || m->emission.y > 0.0f || m->emission.z > 0.0f) {
        float w = 1.0f;
        if (!ps->specular && ps->prev_pdf > 0.0f) {
            float pl = light_pdf_at_hit(s, h->prim, h->t, ps->ray.d, f->n_out);
            w = power_h(ps->prev_pdf, pl);
        }
        ps->L = add(ps->L, muls(mulv(ps->thr, m->emission), w));
    }
    if (m->type == 3) return -1;
    if (ps->depth >= max_depth) return -1;
    return m->type;
}

static int roulette(pstate* ps) {
    if (ps->depth < 3) return 1;
    float q = clampf_(mx(ps->thr.x, mx(ps->thr.y, ps->thr.z)), 0.05f, 0.95f);
    if (rnd(ps->key, (uint32_t)ps->depth, D_RR) >= q) return 0;
    ps->thr = divs(ps->thr, q);
    return 1;
}

static void next_ray(pstate* ps, v3 o, v3 d) {
    ps->ray.o = o; ps->ray.d = d; ps->ray.tmin = RAY_EPS; ps->ray.tmax = INF_F;
}

static int shade_lambert(const oracle_scene* s, pstate* ps, const surf_t* f, ray_t* sh, v3* contrib, int* has) {
    const o_mat* m = &s->materials[f->material];
    uint32_t d = (uint32_t)ps->depth;
    *has = 0;
    v3 org = add(f->p, muls(f->n, RAY_EPS));
    if (s->n_lights > 0) {
        lsample ls = sample_light(s, org, ps->key, d);
        if (ls.pdf > 0.0f) {
            v3 to = sub(ls.p, org);
            float dist = len3(to);
            v3 wi = divs(to, dist);
            float cos_s = dot3(f->n, wi);
            if (cos_s > 0.0f) {
                float pb = cos_s * INV_PI_F;
                float w = power_h(ls.pdf, pb);
                *contrib = muls(mulv(mulv(ps->thr, m->albedo), ls.Le), cos_s * INV_PI_F * w / ls.pdf);
                sh->o = org; sh->d = wi; sh->tmin = RAY_EPS; sh->tmax = dist * (1.0f - 1e-3f);
                *has = 1;
            }
        }
    }
    float u1 = rnd(ps->key, d, D_BU), u2 = rnd(ps->key, d, D_BV);
    float r = sqrtf(u1), phi = 2.0f * PI_F * u2;
    v3 t, b;
    basis(f->n, &t, &b);
    float z = sqrtf(mx(0.0f, 1.0f - u1));
    v3 dir = norm3(add(add(muls(t, r * cosf(phi)), muls(b, r * sinf(phi))), muls(f->n, z)));
    ps->thr = mulv(ps->thr, m->albedo);
    ps->specular = 0;
    ps->prev_pdf = dot3(dir, f->n) * INV_PI_F;
    ps->depth += 1;
    next_ray(ps, org, dir);
    return roulette(ps);
}

static int shade_metal(const oracle_scene* s, pstate* ps, const surf_t* f) {
    const o_mat* m = &s->materials[f->material];
    v3 dir = reflect3(ps->ray.d, f->n);
    if (dot3(dir, f->n) <= 0.0f) return 0;
    ps->thr = mulv(ps->thr, m->albedo);
    ps->specular = 1;
    ps->prev_pdf = 0.0f;
    ps->depth += 1;
    next_ray(ps, add(f->p, muls(f->n, RAY_EPS)), norm3(dir));
    return roulette(ps);
}

static float fresnel(float cos_i, float eta_i, float eta_t) {
    float sin_t = eta_i / eta_t * sqrtf(mx(0.0f, 1.0f - cos_i * cos_i));
    if (sin_t >= 1.0f) return 1.0f;
    float cos_t = sqrtf(mx(0.0f, 1.0f - sin_t * sin_t));
    float rpar = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
    float rperp = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
    return 0.5f * (rpar * rpar + rperp * rperp);
}

static int shade_dielectric(const oracle_scene* s, pstate* ps, const surf_t* f) {
    const o_mat* m = &s->materials[f->material];
    float eta_i = f->inside ? m->ior : 1.0f;
    float eta_t = f->inside ? 1.0f : m->ior;
    float cos_i = clampf_(-dot3(ps->ray.d, f->n), 0.0f, 1.0f);
    float F = fresnel(cos_i, eta_i, eta_t);
    float u = rnd(ps->key, (uint32_t)ps->depth, D_DIEL);
    v3 org, dir;
    if (u < F) {
        dir = reflect3(ps->ray.d, f->n);
        org = add(f->p, muls(f->n, RAY_EPS));
    } else {
        float eta = eta_i / eta_t;
        float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
        float cos_t = sqrtf(mx(0.0f, 1.0f - sin2_t));
        dir = add(muls(ps->ray.d, eta), muls(f->n, eta * cos_i - cos_t));
        org = sub(f->p, muls(f->n, RAY_EPS));
    }
    ps->thr = mulv(ps->thr, m->albedo);
    ps->specular = 1;
    ps->prev_pdf = 0.0f;
    ps->depth += 1;
    next_ray(ps, org, norm3(dir));
    return roulette(ps);
}

static v3 trace_path(const oracle_scene* s, const rig_t* rig, int px, int py, uint32_t sample, uint32_t seed,
                     int max_depth, uint64_t* n_ext, uint64_t* n_sh) {
    pstate ps = init_path(s, rig, px, py, sample, seed);
    for (;;) {
        o_hit h;
        intersect(s, ps.ray, &h, 0);
        ++*n_ext;
        surf_t f;
        int mat = classify(s, &ps, &h, max_depth, &f);
        if (mat < 0) break;
        int alive;
        if (mat == 0) {
            ray_t sh; v3 c = V(0.0f, 0.0f, 0.0f); int has = 0;
            alive = shade_lambert(s, &ps, &f, &sh, &c, &has);
            if (has) {
                o_hit sh_hit;
                ++*n_sh;
                if (!intersect(s, sh, &sh_hit, 1)) ps.L = add(ps.L, c);
            }
        } else if (mat == 1) {
            alive = shade_metal(s, &ps, &f);
        } else {
            alive = shade_dielectric(s, &ps, &f);
        }
        if (!alive) break;
    }
    return ps.L;
}

/* ---- film: per-pixel sums in sample order (WVM/src/cpu_renderer.cpp:55-74) ---- */
typedef struct {
    const oracle_scene* s;
    rig_t rig;
    int first_sample, count, max_depth;
    uint32_t seed;
    int row_begin, row_end;
    float *rgb, *lsum, *l2sum;
    uint64_t n_ext, n_sh;
} band_t;

static void* render_band(void* arg) {
    band_t* b = (band_t*)arg;
    const oracle_scene* s = b->s;
    for (int py = b->row_begin; py < b->row_end; ++py)
        for (int px = 0; px < s->width; ++px) {
            int p = py * s->width + px;
            for (int k = 0; k < b->count; ++k) {
                v3 L = trace_path(s, &b->rig, px, py, (uint32_t)(b->first_sample + k), b->seed, b->max_depth,
                                  &b->n_ext, &b->n_sh);
                b->rgb[3 * p] += L.x;
                b->rgb[3 * p + 1] += L.y;
                b->rgb[3 * p + 2] += L.z;
                float l = lum(L);
                b->lsum[p] += l;
                b->l2sum[p] += l * l;
            }
        }
    return NULL;
}

/*
 * Adds samples [first_sample, first_sample + count) of every pixel to the film sums (rgb 3*w*h,
 * lum w*h, lum2 w*h), row bands on `threads` threads (the result does not depend on the thread
 * count). Optional ray counts (extension, shadow) in rays[2]. Returns 0, or -1 on bad input.
 */
int oracle_render_sums(const oracle_scene* s, int first_sample, int count, uint32_t seed, int max_depth,
                       int threads, float* rgb, float* lsum, float* l2sum, uint64_t* rays) {
    if (!s || !rgb || !lsum || !l2sum || s->width <= 0 || s->height <= 0 || count < 0) return -1;
    if (threads <= 0) threads = 1;
    if (threads > s->height) threads = s->height;
    band_t* bands = (band_t*)calloc((size_t)threads, sizeof(band_t));
    pthread_t* tid = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    if (!bands || !tid) { free(bands); free(tid); return -1; }
    int per = (s->height + threads - 1) / threads;
    rig_t rig = make_rig(s);
    for (int t = 0; t < threads; ++t) {
        band_t* b = &bands[t];
        b->s = s; b->rig = rig; b->first_sample = first_sample; b->count = count;
        b->max_depth = max_depth; b->seed = seed;
        b->row_begin = t * per;
        b->row_end = (t + 1) * per < s->height ? (t + 1) * per : s->height;
        b->rgb = rgb; b->lsum = lsum; b->l2sum = l2sum;
    }
    int started = 0;
    for (int t = 0; t < threads; ++t) {
        if (bands[t].row_begin >= bands[t].row_end) continue;
        if (threads == 1 || pthread_create(&tid[t], NULL, render_band, &bands[t]) != 0) {
            render_band(&bands[t]);
            tid[t] = 0;
        } else {
            started = 1;
        }
    }
    (void)started;
    uint64_t ne = 0, nsh = 0;
    for (int t = 0; t < threads; ++t) {
        if (tid[t]) pthread_join(tid[t], NULL);
        ne += bands[t].n_ext;
        nsh += bands[t].n_sh;
    }
    if (rays) { rays[0] = ne; rays[1] = nsh; }
    free(bands);
    free(tid);
    return 0;
}

/*
 * The reference CPU arm's download convention (WVM/src/cpu_renderer.cpp:106-120): mean = sum / spp
 * in float, lum_var = max(0, (lum2 - spp * mean * mean) / (spp - 1)) in float, 0 when spp == 1.
 */
void oracle_cpu_convention(int pixels, int spp, const float* rgb_sum, const float* lsum, const float* l2sum,
                           float* rgb, float* lum_var) {
    for (int i = 0; i < pixels; ++i) {
        rgb[3 * i] = rgb_sum[3 * i] / spp;
        rgb[3 * i + 1] = rgb_sum[3 * i + 1] / spp;
        rgb[3 * i + 2] = rgb_sum[3 * i + 2] / spp;
        float mean = lsum[i] / spp;
        if (spp > 1) {
            float ssd = l2sum[i] - spp * mean * mean;
            float v = ssd / (spp - 1);
            lum_var[i] = v > 0.0f ? v : 0.0f;
        } else {
            lum_var[i] = 0.0f;
        }
    }
}

/* Closest-hit (anyhit = 0) or any-hit queries of a ray batch (32-byte rays, 16-byte hits). */
void oracle_intersect_batch(const oracle_scene* s, const ray_t* rays, int n, int anyhit, o_hit* hits) {
    for (int i = 0; i < n; ++i) intersect(s, rays[i], &hits[i], anyhit);
}

/* Brute-force closest hit over every primitive (WVM/include/wf/bvh.hpp:119-129). */
void oracle_intersect_bruteforce(const oracle_scene* s, const ray_t* rays, int n, o_hit* hits) {
    int total = s->n_spheres + s->n_triangles;
    for (int i = 0; i < n; ++i) {
        ray_t r = rays[i];
        o_hit* h = &hits[i];
        h->t = r.tmax; h->prim = -1; h->u = 0.0f; h->v = 0.0f;
        for (int p = 0; p < total; ++p) {
            float t, u, v;
            if (hit_prim(s, p, &r, &t, &u, &v)) { r.tmax = t; h->t = t; h->prim = p; h->u = u; h->v = v; }
        }
    }
}

/* 64-bit FNV-1a of a byte buffer (the hash used by the reference's image and scene pins). */
uint64_t oracle_fnv1a64(const void* data, size_t n) {
    const unsigned char* b = (const unsigned char*)data;
    uint64_t h = 14695981039346656037ULL;
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ULL; }
    return h;
}
