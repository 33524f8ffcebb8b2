// Host run of the device traversal steps (box_step, prim_step, can_box_step; dev_scene.cuh) in
// simulated warps, for tests: 32 lanes take rays from a list, and each round the warp runs either a
// primitive step on every lane holding a pending leaf or up to `box_steps` box steps on every lane
// that can take one -- the megakernel's choice (a primitive round once `leaf_batch` lanes hold a
// leaf or they outnumber the box lanes) -- with speculation on or off. The interleavings it makes
// are those the kernels make, so comparing its hits with the oracle's preorder traversal
// (WVM/include/wf/bvh.hpp:91-116) on adversarial rays checks that speculation enters the reference's
// leaves in the reference's order. No GPU is involved.
#include <cstring>
#include <vector>
#include "engine.hpp"
#include "../../include/wfb200.h"

namespace wfb {

void traverse_check(const wf::Scene& host, const float* rays, int n, bool anyhit, bool speculate, int box_steps,
                    int leaf_batch, float* hits) {
    if (n < 0 || box_steps < 1 || leaf_batch < 1) throw Error(WFB_ERR_INVALID_ARGUMENT, "bad traversal check arguments");
    if (host.nodes.empty()) throw Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
    const int nn = (int)host.nodes.size(), np = (int)host.prim_order.size();
    if (nn >= kNodeHeld) throw Error(WFB_ERR_UNSUPPORTED, "BVH has 2^30 nodes or more");
    std::vector<float4> nodes(2 * (size_t)nn), prims(3 * (size_t)(np > 0 ? np : 1));
    for (int i = 0; i < nn; ++i) pack_node(host, i, &nodes[2 * (size_t)i]);
    for (int j = 0; j < np; ++j) pack_prim(host, j, &prims[3 * (size_t)j]);
    const bool nested = check_boxes_nested(host.nodes) != 0;
    const int ns = (int)host.spheres.size();

    struct Lane {
        int ray = -1;
        wf::Vec3 o{0.f, 0.f, 0.f};
        TravRay tr;
        wf::HitRecord h;
        int node = -1, pend = 0;
        bool spec = false;
    };
    Lane lanes[32];
    int cursor = 0;
    auto fetch = [&](Lane& l) {
        if (cursor >= n) {
            l.ray = -1;
            return;
        }
        l.ray = cursor++;
        const float* r = rays + 8 * (size_t)l.ray;
        l.o = wf::Vec3{r[0], r[1], r[2]};
        traversal_begin(nn, wf::Vec3{r[4], r[5], r[6]}, r[7], &l.tr, &l.node, &l.h);
        l.pend = 0;
        l.spec = speculate && (anyhit || (nested && finite_inv(l.tr)));
    };
    for (Lane& l : lanes) fetch(l);
    for (;;) {
        bool any = false;
        for (Lane& l : lanes) {
            while (l.ray >= 0 && l.node < 0 && l.pend == 0) {
                float* out = hits + 4 * (size_t)l.ray;
                out[0] = l.h.t;
                std::memcpy(&out[1], &l.h.prim, 4);
                out[2] = l.h.u;
                out[3] = l.h.v;
                fetch(l);
            }
            any = any || l.ray >= 0;
        }
        if (!any) break;
        int n_leaf = 0, n_box = 0;
        bool in_leaf[32], at_box[32];
        for (int k = 0; k < 32; ++k) {
            const Lane& l = lanes[k];
            in_leaf[k] = l.ray >= 0 && l.pend != 0;
            at_box[k] = l.ray >= 0 && can_box_step(l.node, l.pend, l.spec);
            n_leaf += in_leaf[k];
            n_box += at_box[k];
        }
        if (n_leaf != 0 && (n_leaf >= leaf_batch || n_leaf >= n_box)) {
            for (int k = 0; k < 32; ++k)
                if (in_leaf[k]) {
                    Lane& l = lanes[k];
                    prim_step(prims.data(), ns, l.o, l.tr, anyhit, l.node, l.pend, l.h);
                }
        } else {
            for (int k = 0; k < 32; ++k)
                if (at_box[k]) {
                    Lane& l = lanes[k];
                    for (int s = 0; s < box_steps; ++s)
                        if (s == 0 || can_box_step(l.node, l.pend, l.spec))
                            box_step(nodes.data(), nn, l.o, l.tr, l.h.t, l.node, l.pend);
                }
        }
    }
}


// Host model of a 4-wide traversal over the same tree (a kernel to come), on the packed wide records
// (pack_wide): at an internal node one 128-byte record holds the boxes of its grandchildren (a leaf
// child stands for itself); they are tested together against the current tmax, and the passing ones
// go on a stack in reverse preorder as (node id, code, tmax of that test). A node taken off the stack is
// entered at once if tmax has not moved since (same tmax, same box test), else its own node record is
// loaded and tested against the exact tmax. Middle nodes are never tested: a grandchild that passes
// lies in its parent's box, which would have passed. On a nested tree with a finite 1/d (the
// conditions of box_step's speculation) preorder traversal enters the same leaves in the same order
// with the same tmax; other rays take the binary steps. counts: wide-record fetches, pops, re-tests
// after a tmax change (node-record fetches), binary box steps of the same rays (for comparison).
void traverse_wide_check(const wf::Scene& host, const float* rays, int n, bool anyhit, float* hits,
                         long long* counts) {
    if (n < 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "bad traversal check arguments");
    if (host.nodes.empty()) throw Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
    const int nn = (int)host.nodes.size(), np = (int)host.prim_order.size();
    if (nn >= kNodeHeld) throw Error(WFB_ERR_UNSUPPORTED, "BVH has 2^30 nodes or more");
    std::vector<float4> nodes(2 * (size_t)nn), prims(3 * (size_t)(np > 0 ? np : 1));
    for (int i = 0; i < nn; ++i) pack_node(host, i, &nodes[2 * (size_t)i]);
    for (int j = 0; j < np; ++j) pack_prim(host, j, &prims[3 * (size_t)j]);
    std::vector<float4> wide;
    std::vector<int> code_of;
    const bool wide_ok = pack_wide(host, &wide, &code_of);
    const bool nested = check_boxes_nested(host.nodes) != 0;
    const int ns = (int)host.spheres.size();
    long long fetches = 0, pops = 0, retests = 0, binary_steps = 0;
    struct Entry {
        int node, code;
        float t;
        bool tested;
    };
    std::vector<Entry> stack;
    for (int k = 0; k < n; ++k) {
        const float* r = rays + 8 * (size_t)k;
        const wf::Vec3 o{r[0], r[1], r[2]};
        TravRay tr;
        wf::HitRecord h;
        int node = 0, pend = 0;
        // binary preorder steps: the fallback, and the comparison count
        traversal_begin(nn, wf::Vec3{r[4], r[5], r[6]}, r[7], &tr, &node, &h);
        const wf::HitRecord h0 = h;
        while (node >= 0 || pend != 0) {
            if (pend != 0) {
                prim_step(prims.data(), ns, o, tr, anyhit, node, pend, h);
            } else {
                ++binary_steps;
                box_step(nodes.data(), nn, o, tr, h.t, node, pend);
            }
        }
        if (wide_ok && nested && finite_inv(tr)) {
            h = h0;
            stack.clear();
            stack.push_back(Entry{0, code_of[0], 0.0f, false});
            bool done = false;
            while (!stack.empty() && !done) {
                const Entry e = stack.back();
                stack.pop_back();
                ++pops;
                if (!e.tested || e.t != h.t) {
                    if (e.tested) ++retests;
                    const float4 a = nodes[2 * (size_t)e.node], b = nodes[2 * (size_t)e.node + 1];
                    if (!wf::hit_box_minmax(wf::Vec3{a.x, a.y, a.z}, wf::Vec3{b.x, b.y, b.z}, o, tr.inv_d, wf::kRayEps,
                                            h.t))
                        continue;
                }
                if (e.code >= 0) {  // a leaf: its primitives in leaf order
                    int p = e.code, dummy = 0;
                    while (p != 0) prim_step(prims.data(), ns, o, tr, anyhit, dummy, p, h);
                    done = anyhit && h.prim >= 0;
                    continue;
                }
                ++fetches;
                const float4* w = &wide[8 * (size_t)~e.code];
                for (int s = 3; s >= 0; --s) {
                    const float4 lo = w[2 * s], hi = w[2 * s + 1];
                    const int id = f2i(lo.w);
                    if (id < 0) continue;
                    if (wf::hit_box_minmax(wf::Vec3{lo.x, lo.y, lo.z}, wf::Vec3{hi.x, hi.y, hi.z}, o, tr.inv_d,
                                           wf::kRayEps, h.t))
                        stack.push_back(Entry{id, f2i(hi.w), h.t, true});
                }
            }
        }
        float* out = hits + 4 * (size_t)k;
        out[0] = h.t;
        std::memcpy(&out[1], &h.prim, 4);
        out[2] = h.u;
        out[3] = h.v;
    }
    counts[0] = fetches;
    counts[1] = pops;
    counts[2] = retests;
    counts[3] = binary_steps;
}

}  // namespace wfb
