// Binned-SAH BVH builder emitting the preorder skip-link layout, and its validator.
//
// Output format (API surface, WVM/include/wf/bvh.hpp:8-18): nodes in preorder, node 0 the root,
// the left child of an internal node N at N+1, `skip` of a left child = its right sibling, `skip`
// of a right child = its parent's skip, -1 past the last subtree; leaves hold <= 4 primitives as a
// range of prim_order, and prim_order lists leaf primitives in preorder.
//
// The tree is built depth-first over index ranges with an explicit work stack (no recursion, no
// per-node vector copies), writing nodes straight into preorder; a left child's skip is patched
// when its right sibling is emitted.
//
// Two split policies:
//   sah_bins == 8  (reference-compatible, WVM/src/bvh_build.cpp:60-187): the split axis is the
//                  one with the largest centroid extent, 8 bins, a node with <= 4 primitives is
//                  always a leaf. The bin index, cost and fallback arithmetic are the reference's,
//                  so this mode reproduces the reference's tree node for node (pinned by a test).
//   sah_bins != 8  (default 16 for the benchmark scenes): all three axes are binned and the
//                  cheapest split wins; a node with <= 4 primitives becomes a leaf unless a split
//                  is cheaper under the surface-area heuristic (traversal cost 0.5, intersection 1:
//                  measured fastest for the stackless traversal, where primitive tests cost more
//                  than box tests).
#include <algorithm>
#include <stdexcept>
#include <vector>
#include "wf/bvh.hpp"
#include "wf/scene.hpp"

namespace wf {
namespace {

struct Box {
    Vec3 lo{kInf, kInf, kInf};
    Vec3 hi{-kInf, -kInf, -kInf};
    void grow(Vec3 p) {
        lo = Vec3{fminf3(lo.x, p.x), fminf3(lo.y, p.y), fminf3(lo.z, p.z)};
        hi = Vec3{fmaxf3(hi.x, p.x), fmaxf3(hi.y, p.y), fmaxf3(hi.z, p.z)};
    }
    void grow(const Box& b) {
        lo = Vec3{fminf3(lo.x, b.lo.x), fminf3(lo.y, b.lo.y), fminf3(lo.z, b.lo.z)};
        hi = Vec3{fmaxf3(hi.x, b.hi.x), fmaxf3(hi.y, b.hi.y), fmaxf3(hi.z, b.hi.z)};
    }
    // Empty boxes give inf here, and 0 * inf = NaN makes an empty-side split never win.
    float area() const {
        const Vec3 d = hi - lo;
        return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
};

inline float axis_of(Vec3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct PrimInfo {
    Box box;
    Vec3 centroid;
};

std::vector<PrimInfo> prim_infos(const Scene& scene) {
    const int ns = (int)scene.spheres.size();
    std::vector<PrimInfo> info(scene.n_prims());
    for (int p = 0; p < (int)info.size(); ++p) {
        PrimInfo& pi = info[p];
        if (p < ns) {
            const Sphere& s = scene.spheres[p];
            const Vec3 r{s.radius, s.radius, s.radius};
            pi.box.lo = s.center - r;
            pi.box.hi = s.center + r;
            pi.centroid = s.center;
        } else {
            const Triangle& t = scene.triangles[p - ns];
            const Vec3 a = scene.vertices[t.i0], b = scene.vertices[t.i1], c = scene.vertices[t.i2];
            pi.box.lo = a;
            pi.box.hi = a;
            pi.box.grow(b);
            pi.box.grow(c);
            pi.centroid = (a + b + c) * (1.0f / 3.0f);
        }
    }
    return info;
}

struct Work {
    int begin, end;  // range of `ids`
    int parent;      // internal node whose RIGHT child is built from this range (-1: none)
};

class Builder {
public:
    Builder(const Scene& scene, int bins, int max_leaf, float traversal_cost)
        : info_(prim_infos(scene)), bins_(bins), max_leaf_(max_leaf), ct_(traversal_cost) {
        ids_.resize(info_.size());
        for (int i = 0; i < (int)ids_.size(); ++i) ids_[i] = i;
    }

    void run(std::vector<BvhNode>* nodes, std::vector<int>* order) {
        nodes->clear();
        order->clear();
        nodes->reserve(2 * ids_.size());
        order->reserve(ids_.size());
        std::vector<int> right_child;  // per node: index of its right child (-1 for leaves)
        right_child.reserve(2 * ids_.size());
        std::vector<Work> stack{{0, (int)ids_.size(), -1}};
        while (!stack.empty()) {
            const Work w = stack.back();
            stack.pop_back();
            const int idx = (int)nodes->size();
            if (w.parent >= 0) right_child[w.parent] = idx;
            Box bounds, cbounds;
            for (int i = w.begin; i < w.end; ++i) {
                bounds.grow(info_[ids_[i]].box);
                cbounds.grow(info_[ids_[i]].centroid);
            }
            BvhNode node{};
            node.lo = bounds.lo;
            node.hi = bounds.hi;
            node.skip = -1;
            int mid = -1;
            right_child.push_back(-1);
            if (!make_leaf(w.begin, w.end, bounds, cbounds, &mid)) {
                node.prim_start = -1;
                node.prim_count = 0;
                nodes->push_back(node);
                // Right child first on the stack so the left subtree is emitted next (at idx+1).
                stack.push_back(Work{mid, w.end, idx});
                stack.push_back(Work{w.begin, mid, -1});
            } else {
                node.prim_start = (int)order->size();
                node.prim_count = w.end - w.begin;
                for (int i = w.begin; i < w.end; ++i) order->push_back(ids_[i]);
                nodes->push_back(node);
            }
        }
        // Skip links top-down in preorder (parents precede children): the left child skips to
        // its right sibling, the right child inherits the parent's skip; the root's is -1.
        for (int i = 0; i < (int)nodes->size(); ++i) {
            const int r = right_child[i];
            if (r < 0) continue;
            (*nodes)[i + 1].skip = r;
            (*nodes)[r].skip = (*nodes)[i].skip;
        }
    }

private:
    // Bin index of centroid coordinate `x` on an axis spanning [lo, lo + range).
    int bin_of(float x, float lo, float range) const {
        int b = (int)((x - lo) / range * ((float)bins_ - 0.0001f));
        return b < 0 ? 0 : (b >= bins_ ? bins_ - 1 : b);
    }

    // Decides leaf vs split for ids_[begin, end); on a split, partitions the range stably and
    // returns the first index of the right part in *mid.
    bool make_leaf(int begin, int end, const Box& bounds, const Box& cbounds, int* mid) {
        const int n = end - begin;
        const bool compat = bins_ == 8;
        if (compat && n <= 4) return true;
        if (n <= 1) return true;
        const Vec3 ext = cbounds.hi - cbounds.lo;
        if (ext.x < 1e-6f && ext.y < 1e-6f && ext.z < 1e-6f) {
            if (n <= max_leaf_) return true;
            *mid = begin + n / 2;
            return false;
        }
        int best_axis = -1, best_split = 1;
        float best_cost = 1e9f;
        int compat_axis = 0;
        if (compat) {
            // Largest centroid extent; the reference partitions on it even if no cost wins.
            if (ext.y > ext.x) compat_axis = 1;
            if (ext.z > ext.x && ext.z > ext.y) compat_axis = 2;
            best_axis = compat_axis;
        }
        std::vector<Box> bin_box(bins_);
        std::vector<int> bin_cnt(bins_);
        for (int axis = 0; axis < 3; ++axis) {
            if (compat ? axis != compat_axis : axis_of(ext, axis) < 1e-6f) continue;
            const float lo = axis_of(cbounds.lo, axis);
            const float range = axis_of(cbounds.hi, axis) - lo;
            std::fill(bin_box.begin(), bin_box.end(), Box{});
            std::fill(bin_cnt.begin(), bin_cnt.end(), 0);
            for (int i = begin; i < end; ++i) {
                const PrimInfo& pi = info_[ids_[i]];
                const int b = bin_of(axis_of(pi.centroid, axis), lo, range);
                bin_box[b].grow(pi.box);
                bin_cnt[b] += 1;
            }
            // Right side of each split: bins grown in ascending order (the order only matters for
            // the sign of zero box coordinates, kept as the reference's for the compatible mode).
            std::vector<Box> right_box(bins_);
            std::vector<int> right_cnt(bins_);
            for (int split = 1; split < bins_; ++split) {
                Box acc;
                int cnt = 0;
                for (int b = split; b < bins_; ++b) {
                    acc.grow(bin_box[b]);
                    cnt += bin_cnt[b];
                }
                right_box[split] = acc;
                right_cnt[split] = cnt;
            }
            Box left;
            int lcnt = 0;
            for (int split = 1; split < bins_; ++split) {
                left.grow(bin_box[split - 1]);
                lcnt += bin_cnt[split - 1];
                const float cost = ((float)lcnt * left.area() +
                                    (float)right_cnt[split] * right_box[split].area()) /
                                   bounds.area();
                if (cost < best_cost) {
                    best_cost = cost;
                    best_split = split;
                    best_axis = axis;
                }
            }
        }
        if (!compat && n <= max_leaf_) {
            // SAH termination: a leaf costs n intersections; a split costs one more node visit
            // (traversal_cost) plus the area-weighted intersections of its children.
            if (best_axis < 0 || (float)n <= ct_ + best_cost) return true;
        }
        int m = begin;
        if (best_axis >= 0) {
            const float lo = axis_of(cbounds.lo, best_axis);
            const float range = axis_of(cbounds.hi, best_axis) - lo;
            int* first = ids_.data() + begin;
            int* last = ids_.data() + end;
            int* cut = std::stable_partition(first, last, [&](int p) {
                return bin_of(axis_of(info_[p].centroid, best_axis), lo, range) < best_split;
            });
            m = begin + (int)(cut - first);
        }
        if (m == begin || m == end) m = begin + n / 2;  // empty side: split by index
        *mid = m;
        return false;
    }

    std::vector<PrimInfo> info_;
    std::vector<int> ids_;
    int bins_;
    int max_leaf_;
    float ct_;
};

}  // namespace

void build_bvh_options(Scene& scene, int sah_bins, int max_leaf, float traversal_cost) {
    if (scene.spheres.empty() && scene.triangles.empty())
        throw std::runtime_error("Cannot build BVH: no primitives");
    if (sah_bins < 2 || sah_bins > 256) throw std::runtime_error("SAH bin count must be in [2, 256]");
    if (max_leaf < 1 || max_leaf > 15) throw std::runtime_error("max_leaf must be in [1, 15]");
    if (!(traversal_cost >= 0.0f)) throw std::runtime_error("traversal cost must be >= 0");
    Builder b(scene, sah_bins, sah_bins == 8 ? 4 : max_leaf, traversal_cost);
    b.run(&scene.nodes, &scene.prim_order);
}

void build_bvh_bins(Scene& scene, int sah_bins) { build_bvh_options(scene, sah_bins, 4, 0.5f); }

void build_bvh(Scene& scene) { build_bvh_bins(scene, 8); }

std::string validate_bvh(const Scene& scene) {
    const int n_prims = scene.n_prims();
    const int n_nodes = (int)scene.nodes.size();
    std::vector<int> seen(n_prims, 0);
    for (int p : scene.prim_order) {
        if (p < 0 || p >= n_prims) return "primitive index out of range";
        seen[p] += 1;
    }
    if ((int)scene.prim_order.size() != n_prims) return "not all primitives in BVH";
    for (int c : seen)
        if (c != 1) return "primitive appears multiple times or not at all";
    const std::vector<PrimInfo> info = prim_infos(scene);
    auto contains = [](Vec3 plo, Vec3 phi, Vec3 clo, Vec3 chi) {
        const float e = 1e-5f;
        return plo.x - e <= clo.x && chi.x <= phi.x + e && plo.y - e <= clo.y &&
               chi.y <= phi.y + e && plo.z - e <= clo.z && chi.z <= phi.z + e;
    };
    for (int i = 0; i < n_nodes; ++i) {
        const BvhNode& n = scene.nodes[i];
        if (n.skip < -1 || n.skip >= n_nodes) return "skip link out of bounds";
        if (n.skip != -1 && n.skip <= i) return "skip link does not point forward";
        if (n.prim_count > 0) {
            if (n.prim_count > 4) return "leaf has more than 4 primitives";
            if (n.prim_start < 0 || n.prim_start + n.prim_count > (int)scene.prim_order.size())
                return "leaf prim_start/count out of bounds";
            for (int k = 0; k < n.prim_count; ++k) {
                const Box& pb = info[scene.prim_order[n.prim_start + k]].box;
                if (!contains(n.lo, n.hi, pb.lo, pb.hi)) return "leaf box does not contain its primitive";
            }
            continue;
        }
        if (n.prim_start != -1) return "internal node has prim_start != -1";
        if (i + 1 >= n_nodes) return "left child (N+1) out of bounds";
        const int right = scene.nodes[i + 1].skip;
        if (right <= i + 1 || right >= n_nodes) return "right child index invalid";
        if (scene.nodes[right].skip != n.skip) return "right child does not share parent's skip";
        const BvhNode& l = scene.nodes[i + 1];
        const BvhNode& r = scene.nodes[right];
        if (!contains(n.lo, n.hi, l.lo, l.hi)) return "parent box does not contain left child";
        if (!contains(n.lo, n.hi, r.lo, r.hi)) return "parent box does not contain right child";
    }
    if (n_nodes > 0 && scene.nodes.back().skip != -1) return "last node skip is not -1";
    return "";
}

}  // namespace wf
