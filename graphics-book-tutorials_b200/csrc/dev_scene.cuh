// Device-resident scene in this engine's packed layout, and the traversal over it.
//
// Layout (arrays 256-byte aligned, read through the read-only path; nodes with 32-byte loads, the
// rest with 16-byte loads):
//   nodes     2 x float4 per BVH node, preorder (same order and skip links as wf::BvhNode):
//               {lo.x, lo.y, lo.z, skip}  {hi.x, hi.y, hi.z, leaf}
//             leaf = -1 for an internal node, else prim_start * 16 + prim_count (count 1..15).
//             32 B per node instead of 48 B: a box test is one 32-byte load.
//   prims     3 x float4 per prim_order entry (leaf primitives are contiguous):
//               triangle {p0, id} {e1, 0} {e2, 0} with e1 = p1 - p0, e2 = p2 - p0
//               sphere   {centre, id} {radius, 0, 0, 0} {0}
//             one dependent load level (node -> record) instead of three
//             (node -> prim_order -> triangle -> 3 vertices).
//   spheres   2 x float4 per sphere (wf::Sphere bytes)
//   tri_shade 1 x float4 per triangle {normalize(cross(e1, e2)), material}
//   tri_area  1 float per triangle: 0.5 * length(cross(e1, e2))
//   materials 3 x float4 per material (wf::Material bytes)
//   lights    4 x float4 per light {a, prim} {b, area} {c, material} {n, radius}
// Every precomputed float is produced on the host by the same IEEE operations the reference
// evaluates per ray (WVM/include/wf/bvh.hpp:44-61, WVM/include/wf/path_core.hpp:44-53,84-101,
// 124-131), so the device results are bit-identical to the reference's.
#pragma once
#include <cuda_runtime.h>
#include "wf/path_core.hpp"

namespace wfb {

struct DevScene {
    const float4* nodes;
    const float4* prims;
    const float4* spheres;
    const float4* tri_shade;
    const float* tri_area;
    const float4* materials;
    const float4* lights;
    int n_spheres, n_triangles, n_materials, n_nodes, n_lights;
    wf::Vec3 env;
    wf::CameraRig camera;
    int width, height;
    // 1 when every node's box lies inside the box of each node whose subtree holds it (checked at
    // upload): the condition under which speculative closest-hit traversal is exact (box_step).
    int boxes_nested;
};

constexpr int kLeafCountBits = 4;
constexpr int kLeafCountMask = (1 << kLeafCountBits) - 1;
constexpr int kMaxLeafPrims = kLeafCountMask;
constexpr long long kMaxLeafStart = (1LL << (31 - kLeafCountBits)) - 1;

template <class T>
WF_HD T ro_load(const T* p) {
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

WF_HD int f2i(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_int(f);
#else
    int i;
    __builtin_memcpy(&i, &f, 4);
    return i;
#endif
}

// Split-mode radiance slots (3 floats per (pixel, sample) of a call), sample-major: the slots of
// one sample of neighbouring pixels are adjacent, so a warp of neighbouring pixels writes (and the
// ordered commit reads) one contiguous run instead of scattered 12-byte pieces.
WF_HD size_t sample_slot(int pixel, int sample_index, int pixels) {
    return 3 * ((size_t)sample_index * (size_t)pixels + (size_t)pixel);
}

// ---- accessors used by the estimator templates (wf/path_core.hpp) ----
WF_HD wf::Sphere load_sphere(const DevScene& s, int i) {
    const float4 a = ro_load(&s.spheres[2 * i]);
    const float4 b = ro_load(&s.spheres[2 * i + 1]);
    wf::Sphere sp;
    sp.center = wf::Vec3{a.x, a.y, a.z};
    sp.radius = a.w;
    sp.material = f2i(b.x);
    sp.pad[0] = sp.pad[1] = sp.pad[2] = 0;
    return sp;
}
WF_HD wf::Material load_material(const DevScene& s, int m) {
    const float4 a = ro_load(&s.materials[3 * m]);
    const float4 b = ro_load(&s.materials[3 * m + 1]);
    const float4 c = ro_load(&s.materials[3 * m + 2]);
    wf::Material mat;
    mat.type = f2i(a.x);
    mat.ior = a.y;
    mat.pad0 = a.z;
    mat.pad1 = a.w;
    mat.albedo = wf::Vec3{b.x, b.y, b.z};
    mat.pad2 = b.w;
    mat.emission = wf::Vec3{c.x, c.y, c.z};
    mat.pad3 = c.w;
    return mat;
}
WF_HD int tri_material(const DevScene& s, int t) { return f2i(ro_load(&s.tri_shade[t]).w); }
WF_HD wf::Vec3 tri_normal(const DevScene& s, int t) {
    const float4 a = ro_load(&s.tri_shade[t]);
    return wf::Vec3{a.x, a.y, a.z};
}
WF_HD float prim_area(const DevScene& s, int prim) {
    if (prim < s.n_spheres) {
        const float r = ro_load(&s.spheres[2 * prim]).w;
        return 4.0f * wf::kPi * r * r;
    }
    return ro_load(&s.tri_area[prim - s.n_spheres]);
}
WF_HD wf::LightGeom load_light(const DevScene& s, int idx) {
    const float4 a = ro_load(&s.lights[4 * idx]);
    const float4 b = ro_load(&s.lights[4 * idx + 1]);
    const float4 c = ro_load(&s.lights[4 * idx + 2]);
    const float4 d = ro_load(&s.lights[4 * idx + 3]);
    wf::LightGeom g;
    g.prim = f2i(a.w);
    g.is_sphere = g.prim < s.n_spheres ? 1 : 0;
    g.a = wf::Vec3{a.x, a.y, a.z};
    g.b = wf::Vec3{b.x, b.y, b.z};
    g.area = b.w;
    g.c = wf::Vec3{c.x, c.y, c.z};
    g.material = f2i(c.w);
    g.n = wf::Vec3{d.x, d.y, d.z};
    g.radius = d.w;
    return g;
}

#if defined(__CUDACC__)
// Direction of a ray being traversed by the resumable traversal below. Its origin is passed to
// each step (the path's current ray origin) and its tmin is kRayEps: every ray the estimator
// creates has tmin = kRayEps (camera_ray, set_next_ray, the shadow ray of shade_lambert,
// WVM/include/wf/path_core.hpp:67,184,211), so neither is stored per ray.
struct TravRay {
    wf::Vec3 d, inv_d;
};

// Resumable stackless skip-link traversal over the packed nodes (the steps compile for the host
// too: wfb_test_traverse runs them in simulated warps against the oracle), split into box steps and
// primitive steps. A ray's whole traversal state is its next node (`node`, -1 when none is left),
// its pending leaf (`pend`) and its best hit (`h`; h.t is the current tmax).
//
// A box step tests the lane's next node; at a leaf whose box the ray enters it records the leaf as
// pending (`pend` = first record * 16 + count, the node's own leaf encoding; 0 = none) and moves
// `node` past the leaf (to its skip link). A primitive step tests the next primitive of the pending
// leaf (pend += 15: next record, one fewer left). Taken one after another until node < 0 and
// pend == 0, the steps visit nodes and primitives in wf::intersect's order (preorder, skip link on
// a miss and after a leaf, every primitive of a leaf in leaf order against tmax = the nearest hit
// so far, a hit replacing the best only when strictly nearer; WVM/include/wf/bvh.hpp:91-116) with
// its box and primitive arithmetic, so hit ids, t, u and v are bit-identical; `anyhit` ends the
// query at the first hit. Splitting the steps lets a warp group them: rounds of box steps, and
// rounds of primitive steps once enough lanes hold a pending leaf, instead of every box round
// waiting while the one or two lanes that reached a leaf test its primitives one after another.
//
// Speculation (after Aila and Laine's speculative traversal, HPG 2009, made exact): a lane that
// holds a pending leaf may go on taking box steps, against the current tmax, which does not yet
// include that leaf's hits. The first leaf it reaches that way is not recorded: the step marks
// `node` with kNodeHeld and the lane stops there; once the pending leaf is done, the mark is
// cleared and the same node takes an ordinary box step, against the tmax preorder traversal has at
// that point, which decides the leaf. So leaves are entered in preorder with preorder's tmax, one at
// a time, and the hit is the same. What speculation adds is box steps on nodes that preorder
// traversal would have culled with its smaller tmax; their leaves then fail that final step, for
// the box test is monotone in tmax and in the box (a box inside another, tested with the same tmax,
// passes only if the outer one does: per axis its slab distances lie inside the outer box's, IEEE
// rounding being monotone) -- so a leaf that preorder traversal never reaches, because an
// enclosing node failed, fails too. Two conditions make that hold: nested boxes (the scene's
// `boxes_nested`), and finite 1/d (a zero direction component makes slab distances 0 * inf, whose
// NaN mapping is not monotone in the box). Any-hit queries never lower tmax, so for them
// speculation needs neither.
constexpr int kNodeHeld = 1 << 30;

WF_HD bool finite_inv(const TravRay& ray) {
    return fmaxf(fmaxf(fabsf(ray.inv_d.x), fabsf(ray.inv_d.y)), fabsf(ray.inv_d.z)) < INFINITY;
}

// A lane may take a box step: it has a node to test and no pending leaf, or it speculates and its
// node is not a held leaf.
WF_HD bool can_box_step(int node, int pend, bool spec) {
    return node >= 0 && (pend == 0 || (spec && node < kNodeHeld));
}

WF_HD void box_step(const float4* __restrict__ nodes, int n_nodes, const wf::Vec3& o,
                                         const TravRay& ray, float tmax, int& node, int& pend) {
    // the whole 32-byte node in one 256-bit load (nodes are 32-byte aligned: a 256-byte aligned array
    // of 32-byte records); +0.9% on icospheres over two 128-bit loads, the same bits
    float4 na, nb;
#if defined(__CUDA_ARCH__)
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(na.x), "=f"(na.y), "=f"(na.z), "=f"(na.w), "=f"(nb.x), "=f"(nb.y), "=f"(nb.z), "=f"(nb.w)
        : "l"(nodes + 2 * node));
#else
    na = nodes[2 * node];
    nb = nodes[2 * node + 1];
#endif
    const int skip = f2i(na.w);
    if (!wf::hit_box_minmax(wf::Vec3{na.x, na.y, na.z}, wf::Vec3{nb.x, nb.y, nb.z}, o, ray.inv_d, wf::kRayEps, tmax)) {
        node = skip;
    } else {
        const int leaf = f2i(nb.w);
        if (leaf < 0) {
            node = node + 1;
        } else if (pend == 0) {
            node = skip;
            pend = leaf;
        } else {
            node |= kNodeHeld;  // speculative: decided again once the pending leaf is done
            return;
        }
    }
    if (node >= n_nodes) node = -1;
}

WF_HD void prim_step(const float4* __restrict__ prims, int n_spheres, const wf::Vec3& o,
                                          const TravRay& ray, bool anyhit, int& node, int& pend, wf::HitRecord& h) {
    const float4* rec = prims + 3 * (pend >> kLeafCountBits);
    const float4 q0 = ro_load(rec);
    const float4 q1 = ro_load(rec + 1);
    const int p = f2i(q0.w);
    wf::Ray r;
    r.o = o;
    r.d = ray.d;
    r.tmin = wf::kRayEps;
    r.tmax = h.t;
    float t, u = 0.0f, v = 0.0f;
    bool hit;
    if (p < n_spheres) {
        hit = wf::hit_sphere_core(wf::Vec3{q0.x, q0.y, q0.z}, q1.x, r, &t);
    } else {
        const float4 q2 = ro_load(rec + 2);
        hit = wf::hit_triangle_core(wf::Vec3{q0.x, q0.y, q0.z}, wf::Vec3{q1.x, q1.y, q1.z},
                                    wf::Vec3{q2.x, q2.y, q2.z}, r, &t, &u, &v);
    }
    pend += (1 << kLeafCountBits) - 1;
    if ((pend & kLeafCountMask) == 0) {
        pend = 0;
        if (node >= kNodeHeld) node -= kNodeHeld;  // a leaf held back by speculation takes its box step next
    }
    if (hit) {
        h.t = t;
        h.prim = p;
        h.u = u;
        h.v = v;
        if (anyhit) {
            node = -1;
            pend = 0;
        }
    }
}

// intersect() prologue (WVM/include/wf/bvh.hpp:92-94): the ray's traversal state before step 0.
WF_HD void traversal_begin(int n_nodes, wf::Vec3 d, float tmax, TravRay* ray, int* node,
                                                wf::HitRecord* h) {
    ray->d = d;
    ray->inv_d = wf::Vec3{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    h->t = tmax;
    h->prim = -1;
    h->u = 0.0f;
    h->v = 0.0f;
    *node = n_nodes > 0 ? 0 : -1;
}

// Validity check applied after every closest-hit query (WVM/src/gpu/engine.cuh:44-48).
__device__ __forceinline__ bool hit_is_valid(const DevScene& s, const wf::HitRecord& h) {
    if (h.prim < 0) return true;
    const int total = s.n_spheres + s.n_triangles;
    return h.prim < total && wf::is_finite1(h.t) && h.t > 0.0f;
}

#endif  // __CUDACC__

// Per-pixel running sums (WVM/src/gpu/engine.cuh:18-32): rgb[3P], lum[P], lum2[P]. A pixel has one
// writer at a time and samples are added in ascending sample order, never with atomics.
struct DevFilm {
    float* rgb;
    float* lum;
    float* lum2;
    int pixels;
};

// Counters shared by every engine (layout is internal to this library).
struct DevCounters {
    unsigned long long extension_rays;
    unsigned long long shadow_rays;
    unsigned int invalid_hits;
    unsigned int overflows;
    unsigned int high_water[5];
    unsigned int error;  // nonzero: a bounded wait gave up (see kErr* codes)
    unsigned int pad;
    unsigned long long node_visits;  // traversal steps (box tests), when counting rays
    unsigned long long prim_tests;   // primitive intersection tests, when counting rays
};

enum : unsigned int {
    kErrNone = 0,
    kErrSpinTimeout = 1,  // a grid-wide wait or a scan lookback exceeded its poll limit
};

}  // namespace wfb
