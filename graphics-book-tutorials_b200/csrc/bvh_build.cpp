// Binned-SAH BVH builder emitting the preorder skip-link layout, and its validator.
//
// Output format (API surface, WVM/include/wf/bvh.hpp:8-18): nodes in preorder, node 0 the root,
// the left child of an internal node N at N+1, `skip` of a left child = its right sibling, `skip`
// of a right child = its parent's skip, -1 past the last subtree; leaves hold <= 4 primitives as a
// range of prim_order, and prim_order lists leaf primitives in preorder.
//
// The tree is built depth-first over index ranges with an explicit work stack (no recursion, no
// per-node vector copies), writing nodes in preorder; skip links are set in one pass at the end.
//
// Parallel build: the top of the tree is built on the calling thread, in preorder; every range
// of at most `grain` primitives met there becomes an independent subtree task instead. Tasks run
// on a pool of threads, each into its own node / prim_order / right-child arrays, and are then
// stitched into the preorder layout (node and primitive offsets added). A range's split decision
// depends only on the primitives in it, and a task permutes only its own slice of the id array,
// so the tree is byte-identical to the single-threaded build for any thread count.
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
#include <atomic>
#include <stdexcept>
#include <thread>
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

// Runs fn(i) for i in [0, n) on `threads` threads (the calling thread is one of them).
template <class F>
void parallel_for(int n, int threads, F&& fn) {
    std::atomic<int> next{0};
    auto worker = [&] {
        for (int i; (i = next.fetch_add(1)) < n;) fn(i);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::min(threads, n); ++t) pool.emplace_back(worker);
    worker();
    for (std::thread& t : pool) t.join();
}

std::vector<PrimInfo> prim_infos(const Scene& scene, int threads) {
    const int ns = (int)scene.spheres.size();
    std::vector<PrimInfo> info(scene.n_prims());
    const int chunk = 1 << 16;
    parallel_for(((int)info.size() + chunk - 1) / chunk, threads, [&](int c) {
    for (int p = c * chunk; p < std::min((int)info.size(), (c + 1) * chunk); ++p) {
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
    });
    return info;
}

struct Work {
    int begin, end;  // range of `ids`
    int parent;      // internal node whose RIGHT child is built from this range (-1: none)
};

// Nodes of a subtree in preorder with local indices; right[i] is node i's right child (-1: leaf).
struct Subtree {
    std::vector<BvhNode> nodes;
    std::vector<int> order;
    std::vector<int> right;
};

class Builder {
public:
    Builder(const Scene& scene, int bins, int max_leaf, float traversal_cost, int threads)
        : info_(prim_infos(scene, threads)), bins_(bins), max_leaf_(max_leaf), ct_(traversal_cost), threads_(threads) {
        ids_.resize(info_.size());
        for (int i = 0; i < (int)ids_.size(); ++i) ids_[i] = i;
    }

    void run(std::vector<BvhNode>* nodes, std::vector<int>* order) {
        const int n = (int)ids_.size();
        // Ranges of at most `grain` primitives below the top become tasks (about 16 per thread).
        const int grain = threads_ > 1 ? std::max(2048, n / (16 * threads_)) : n + 1;
        // Top of the tree in preorder: each piece is a top node or a task placeholder.
        struct Piece {
            BvhNode node;
            int right_piece;  // top internal node: piece index of its right child, else -1
            int task;         // task index, or -1 for a top node
        };
        std::vector<Piece> pieces;
        std::vector<std::pair<int, int>> task_ranges;
        std::vector<Work> stack{{0, n, -1}};
        while (!stack.empty()) {
            const Work w = stack.back();
            stack.pop_back();
            const int me = (int)pieces.size();
            if (w.parent >= 0) pieces[w.parent].right_piece = me;
            if (w.end - w.begin <= grain && me > 0) {
                pieces.push_back(Piece{BvhNode{}, -1, (int)task_ranges.size()});
                task_ranges.emplace_back(w.begin, w.end);
                continue;
            }
            Subtree one;
            int mid = -1;
            const bool leaf = emit(w.begin, w.end, &one, &mid, threads_ > 1);
            if (leaf) one.nodes[0].prim_start = w.begin;  // top leaf: its slice of ids_
            pieces.push_back(Piece{one.nodes[0], -1, -1});
            if (!leaf) {
                stack.push_back(Work{mid, w.end, me});
                stack.push_back(Work{w.begin, mid, -1});
            }
        }
        std::vector<Subtree> tasks(task_ranges.size());
        parallel_for((int)tasks.size(), threads_, [&](int t) { build(task_ranges[t].first, task_ranges[t].second, &tasks[t]); });

        // Stitch: first node index of every piece, then the nodes, right children and prim_order.
        std::vector<int> base(pieces.size());
        int total = 0;
        for (size_t p = 0; p < pieces.size(); ++p) {
            base[p] = total;
            total += pieces[p].task < 0 ? 1 : (int)tasks[pieces[p].task].nodes.size();
        }
        nodes->assign((size_t)total, BvhNode{});
        std::vector<int> right((size_t)total, -1);
        order->clear();
        order->reserve((size_t)n);
        for (size_t p = 0; p < pieces.size(); ++p) {
            const Piece& pc = pieces[p];
            if (pc.task < 0) {
                BvhNode nd = pc.node;
                if (nd.prim_count > 0) {  // a leaf at the top (a tree of a few primitives)
                    const int first = nd.prim_start;
                    nd.prim_start = (int)order->size();
                    for (int i = 0; i < nd.prim_count; ++i) order->push_back(ids_[first + i]);
                } else {
                    right[base[p]] = base[pc.right_piece];
                }
                (*nodes)[base[p]] = nd;
            } else {
                const Subtree& st = tasks[pc.task];
                const int prim_base = (int)order->size();
                for (size_t i = 0; i < st.nodes.size(); ++i) {
                    BvhNode nd = st.nodes[i];
                    if (nd.prim_count > 0) nd.prim_start += prim_base;
                    (*nodes)[base[p] + i] = nd;
                    if (st.right[i] >= 0) right[base[p] + i] = base[p] + st.right[i];
                }
                order->insert(order->end(), st.order.begin(), st.order.end());
            }
        }
        // Skip links top-down in preorder (parents precede children): the left child skips to
        // its right sibling, the right child inherits the parent's skip; the root's is -1.
        for (int i = 0; i < total; ++i) {
            const int r = right[i];
            if (r < 0) continue;
            (*nodes)[i + 1].skip = r;
            (*nodes)[r].skip = (*nodes)[i].skip;
        }
    }

private:
    // Builds the subtree over ids_[begin, end) into `out` (local preorder).
    void build(int begin, int end, Subtree* out) {
        out->nodes.reserve(2 * (size_t)(end - begin));
        out->right.reserve(2 * (size_t)(end - begin));
        out->order.reserve((size_t)(end - begin));
        std::vector<Work> stack{{begin, end, -1}};
        while (!stack.empty()) {
            const Work w = stack.back();
            stack.pop_back();
            const int idx = (int)out->nodes.size();
            if (w.parent >= 0) out->right[w.parent] = idx;
            int mid = -1;
            if (!emit(w.begin, w.end, out, &mid, false)) {
                // Right child first on the stack so the left subtree is emitted next (at idx+1).
                stack.push_back(Work{mid, w.end, idx});
                stack.push_back(Work{w.begin, mid, -1});
            }
        }
    }

    // Appends the node for ids_[begin, end) to `out`: a leaf (its primitives appended to
    // out->order, prim_start local to it) or an internal node whose range is partitioned at *mid.
    // Returns true for a leaf. skip stays -1 until the final pass. `par`: large ranges spread their
    // passes over the thread pool (top of the tree only; tasks are already parallel).
    bool emit(int begin, int end, Subtree* out, int* mid, bool par) {
        Box bounds, cbounds;
        fold_chunks(begin, end, par, std::pair<Box, Box>{},
                    [&](int b, int e, std::pair<Box, Box>& acc) {
                        for (int i = b; i < e; ++i) {
                            acc.first.grow(info_[ids_[i]].box);
                            acc.second.grow(info_[ids_[i]].centroid);
                        }
                    },
                    [&](const std::pair<Box, Box>& acc) {
                        bounds.grow(acc.first);
                        cbounds.grow(acc.second);
                    });
        BvhNode node{};
        node.lo = bounds.lo;
        node.hi = bounds.hi;
        node.skip = -1;
        out->right.push_back(-1);
        if (!make_leaf(begin, end, bounds, cbounds, mid, par)) {
            node.prim_start = -1;
            node.prim_count = 0;
            out->nodes.push_back(node);
            return false;
        }
        node.prim_start = (int)out->order.size();
        node.prim_count = end - begin;
        for (int i = begin; i < end; ++i) out->order.push_back(ids_[i]);
        out->nodes.push_back(node);
        return true;
    }

private:
    // Bin index of centroid coordinate `x` on an axis spanning [lo, lo + range).
    int bin_of(float x, float lo, float range) const {
        int b = (int)((x - lo) / range * ((float)bins_ - 0.0001f));
        return b < 0 ? 0 : (b >= bins_ ? bins_ - 1 : b);
    }

    // Decides leaf vs split for ids_[begin, end); on a split, partitions the range stably and
    // returns the first index of the right part in *mid.
    bool make_leaf(int begin, int end, const Box& bounds, const Box& cbounds, int* mid, bool par) {
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
            if (!par || n < kParallelRange) {
                for (int i = begin; i < end; ++i) {
                    const PrimInfo& pi = info_[ids_[i]];
                    const int b = bin_of(axis_of(pi.centroid, axis), lo, range);
                    bin_box[b].grow(pi.box);
                    bin_cnt[b] += 1;
                }
            } else {
                using Bins = std::pair<std::vector<Box>, std::vector<int>>;
                fold_chunks(begin, end, par, Bins(std::vector<Box>(bins_), std::vector<int>(bins_, 0)),
                            [&](int b0, int e0, Bins& acc) {
                                for (int i = b0; i < e0; ++i) {
                                    const PrimInfo& pi = info_[ids_[i]];
                                    const int b = bin_of(axis_of(pi.centroid, axis), lo, range);
                                    acc.first[b].grow(pi.box);
                                    acc.second[b] += 1;
                                }
                            },
                            [&](const Bins& acc) {
                                for (int b = 0; b < bins_; ++b) {
                                    bin_box[b].grow(acc.first[b]);
                                    bin_cnt[b] += acc.second[b];
                                }
                            });
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
            auto left_of = [&](int p) { return bin_of(axis_of(info_[p].centroid, best_axis), lo, range) < best_split; };
            m = begin + stable_partition_ids(first, last, par, left_of);
        }
        if (m == begin || m == end) m = begin + n / 2;  // empty side: split by index
        *mid = m;
        return false;
    }

    // Folds [begin, end) chunk by chunk, each chunk into its own copy of `init`, and hands the
    // chunk results to `combine` in chunk order. Chunks run on the thread pool when `par` and the
    // range is large. With combine applied in order, the result equals one sequential fold: box
    // growth keeps the first of equal values (strict compare-select on finite coordinates, which
    // scene validation guarantees) and counts are integers.
    template <class Acc, class Fold, class Combine>
    void fold_chunks(int begin, int end, bool par, const Acc& init, Fold&& fold, Combine&& combine) const {
        const int n = end - begin;
        const int chunk = par && n >= kParallelRange ? std::max(kParallelRange / 4, n / (4 * threads_)) : n;
        const int nchunks = chunk > 0 ? (n + chunk - 1) / chunk : 0;
        if (nchunks <= 1) {
            Acc acc = init;
            fold(begin, end, acc);
            combine(acc);
            return;
        }
        std::vector<Acc> accs((size_t)nchunks, init);
        parallel_for(nchunks, threads_, [&](int c) { fold(begin + c * chunk, std::min(end, begin + (c + 1) * chunk), accs[(size_t)c]); });
        for (const Acc& a : accs) combine(a);
    }

    // std::stable_partition of [first, last) by `left`, spread over the pool for large ranges
    // (flags, per-chunk counts, then every chunk scatters its elements to their stable places).
    // Returns the size of the left part.
    template <class Pred>
    int stable_partition_ids(int* first, int* last, bool par, Pred&& left) const {
        const int n = (int)(last - first);
        if (!par || n < kParallelRange) return (int)(std::stable_partition(first, last, left) - first);
        const int chunk = std::max(kParallelRange / 4, n / (4 * threads_));
        const int nchunks = (n + chunk - 1) / chunk;
        std::vector<unsigned char> flag((size_t)n);
        std::vector<int> nleft((size_t)nchunks, 0);
        parallel_for(nchunks, threads_, [&](int c) {
            int k = 0;
            for (int i = c * chunk; i < std::min(n, (c + 1) * chunk); ++i) k += (flag[(size_t)i] = left(first[i]) ? 1 : 0);
            nleft[(size_t)c] = k;
        });
        std::vector<int> lbase((size_t)nchunks), rbase((size_t)nchunks);
        int total_left = 0;
        for (int c = 0; c < nchunks; ++c) {
            lbase[(size_t)c] = total_left;
            total_left += nleft[(size_t)c];
        }
        for (int c = 0, r = total_left; c < nchunks; ++c) {
            rbase[(size_t)c] = r;
            r += std::min(n, (c + 1) * chunk) - c * chunk - nleft[(size_t)c];
        }
        std::vector<int> out((size_t)n);
        parallel_for(nchunks, threads_, [&](int c) {
            int l = lbase[(size_t)c], r = rbase[(size_t)c];
            for (int i = c * chunk; i < std::min(n, (c + 1) * chunk); ++i) out[(size_t)(flag[(size_t)i] ? l++ : r++)] = first[i];
        });
        std::copy(out.begin(), out.end(), first);
        return total_left;
    }

    static constexpr int kParallelRange = 1 << 15;

    std::vector<PrimInfo> info_;
    std::vector<int> ids_;
    int bins_;
    int max_leaf_;
    float ct_;
    int threads_;
};

}  // namespace

void build_bvh_options(Scene& scene, int sah_bins, int max_leaf, float traversal_cost, int threads) {
    if (scene.spheres.empty() && scene.triangles.empty())
        throw std::runtime_error("Cannot build BVH: no primitives");
    if (sah_bins < 2 || sah_bins > 256) throw std::runtime_error("SAH bin count must be in [2, 256]");
    if (max_leaf < 1 || max_leaf > 15) throw std::runtime_error("max_leaf must be in [1, 15]");
    if (!(traversal_cost >= 0.0f)) throw std::runtime_error("traversal cost must be >= 0");
    if (threads <= 0) threads = (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()));
    Builder b(scene, sah_bins, sah_bins == 8 ? 4 : max_leaf, traversal_cost, threads);
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
    const std::vector<PrimInfo> info = prim_infos(scene, 1);
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
