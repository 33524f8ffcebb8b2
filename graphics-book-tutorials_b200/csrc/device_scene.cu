// Scene upload: validation and repacking into the device layout described in dev_scene.cuh.
// Host arithmetic in this file is compiled without contraction (-ffp-contract=off) so every
// precomputed float equals the one the reference computes per ray.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <functional>
#include <initializer_list>
#include <mutex>
#include <thread>
#include <string>
#include <vector>
#include "engine.hpp"
#include "../../include/wfb200.h"

namespace wfb {

void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int st = (e == cudaErrorMemoryAllocation) ? WFB_ERR_OUT_OF_MEMORY : WFB_ERR_CUDA;
    cudaGetLastError();  // clear a sticky launch error so the next call starts clean
    throw Error(st, std::string(what) + ": " + cudaGetErrorString(e));
}

ResidentScene::~ResidentScene() {
    if (arena) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (device >= 0 && cur != device) cudaSetDevice(device);
        // Renders and batch launches wait for their kernels before returning, and renderers and
        // batches hold the scene while they exist; work that returned without waiting (the
        // allocation-free entry, on the caller's stream) recorded `last_use`, which the release
        // waits for.
        if (last_use) cudaStreamWaitEvent(0, last_use, 0);
        cudaFreeAsync(arena, 0);
        if (device >= 0 && cur != device && cur >= 0) cudaSetDevice(cur);
    }
    if (last_use) cudaEventDestroy(last_use);
}

namespace {

inline float i2f(int i) {
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}

inline float4 f4(wf::Vec3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

DevScene with_camera(const DevScene& s, const wf::Camera& cam, int width, int height) {
    DevScene v = s;
    v.camera = wf::make_camera_rig(cam, width, height);  // host libm, as the reference does
    v.width = width;
    v.height = height;
    return v;
}

namespace {

// Pinned host staging for scene uploads, reused by every upload of the process (grown when a
// larger scene arrives, never returned): the packed arrays are written straight into it and cross
// PCIe in one copy, instead of being built in fresh pageable vectors (page faults) and copied by
// the driver through its own bounce buffer.
struct Staging {
    std::mutex mu;
    char* p = nullptr;
    size_t cap = 0;
};
Staging& staging() {
    static Staging* s = new Staging;  // not freed at exit: the CUDA runtime may be gone by then
    return *s;
}

// Cache key of a packed arena: 4 KB chunks hashed on the device 8 bytes at a time with a
// multiply-xorshift mix; the host folds the chunk hashes in order.
constexpr size_t kHashChunkWords = 512;
__global__ void hash_chunks(const unsigned long long* __restrict__ w, size_t n_words, unsigned long long* out) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t begin = c * kHashChunkWords;
    if (begin >= n_words) return;
    const size_t end = begin + kHashChunkWords < n_words ? begin + kHashChunkWords : n_words;
    unsigned long long h = 0x6A09E667F3BCC909ull ^ c;
    for (size_t i = begin; i < end; ++i) {
        h = (h ^ w[i]) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    out[c] = h;
}

uint64_t fold(uint64_t h, uint64_t w) {
    h = (h ^ w) * 0x9E3779B97F4A7C15ull;
    return h ^ (h >> 29);
}

// Runs the sections on up to `threads` threads (the caller's included), each thread taking the next
// section in order; rethrows the error of the first section (in order) that failed, as a serial
// pass would.
void run_sections(const std::vector<std::function<void()>>& fs, int threads) {
    std::vector<std::exception_ptr> errs(fs.size());
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t k; (k = next.fetch_add(1)) < fs.size();) {
            try {
                fs[k]();
            } catch (...) {
                errs[k] = std::current_exception();
            }
        }
    };
    std::vector<std::thread> pool;
    const int extra = std::min<int>(threads, (int)fs.size()) - 1;
    for (int t = 0; t < extra; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (const auto& e : errs)
        if (e) std::rethrow_exception(e);
}

// Splits [0, n) into ranges of at least `grain` items, at most `parts` of them, as sections.
void add_ranges(std::vector<std::function<void()>>& fs, int n, int grain, int parts,
                const std::function<void(int, int)>& body) {
    const int k = std::max(1, std::min(parts, n / std::max(1, grain)));
    for (int c = 0; c < k; ++c) {
        const int lo = (int)((long long)n * c / k), hi = (int)((long long)n * (c + 1) / k);
        fs.emplace_back([=, &body] { body(lo, hi); });
    }
}

}  // namespace

void pack_node(const wf::Scene& host, int i, float4* out) {
    // {lo, skip} {hi, leaf}
    const int nn = (int)host.nodes.size(), np = (int)host.prim_order.size();
    const wf::BvhNode& n = host.nodes[i];
    int leaf = -1;
    if (n.prim_count > 0) {
        if (n.prim_count > kMaxLeafPrims) throw Error(WFB_ERR_UNSUPPORTED, "BVH leaf holds more than 15 primitives");
        if (n.prim_start < 0 || (long long)n.prim_start + n.prim_count > np || n.prim_start > kMaxLeafStart)
            throw Error(WFB_ERR_INVALID_ARGUMENT, "BVH leaf prim_start/count out of bounds");
        leaf = (n.prim_start << kLeafCountBits) | n.prim_count;
    }
    if (n.skip < -1 || n.skip >= nn) throw Error(WFB_ERR_INVALID_ARGUMENT, "BVH skip link out of bounds");
    // Every traversal step moves forward (to N+1 or to a forward skip), so a traversal ends after at
    // most n_nodes steps; a backward skip could loop forever and is rejected.
    if (n.skip != -1 && n.skip <= i) throw Error(WFB_ERR_INVALID_ARGUMENT, "BVH skip link does not point forward");
    out[0] = f4(n.lo, i2f(n.skip));
    out[1] = f4(n.hi, i2f(leaf));
}

bool pack_wide(const wf::Scene& host, std::vector<float4>* records, std::vector<int>* code_of) {
    const int nn = (int)host.nodes.size();
    auto end_of = [&](int i) { return host.nodes[i].skip < 0 ? nn : host.nodes[i].skip; };
    auto is_leaf = [&](int i) { return host.nodes[i].prim_count > 0; };
    std::vector<int> code(nn);
    int n_wide = 0;
    for (int i = 0; i < nn; ++i) {
        const wf::BvhNode& n = host.nodes[i];
        code[i] = is_leaf(i) ? ((n.prim_start << kLeafCountBits) | n.prim_count) : ~n_wide++;
    }
    std::vector<float4> rec(8 * (size_t)n_wide);
    for (int i = 0; i < nn; ++i) {
        if (is_leaf(i)) continue;
        int cand[4], nc = 0;
        for (int c = i + 1; c < end_of(i); c = end_of(c)) {
            if (end_of(c) <= c) return false;
            if (is_leaf(c)) {
                if (nc == 4) return false;
                cand[nc++] = c;
                continue;
            }
            for (int g = c + 1; g < end_of(c); g = end_of(g)) {
                if (end_of(g) <= g || nc == 4) return false;
                cand[nc++] = g;
            }
        }
        float4* r = &rec[8 * (size_t)~code[i]];
        for (int k = 0; k < 4; ++k) {
            if (k < nc) {
                const wf::BvhNode& c = host.nodes[cand[k]];
                r[2 * k] = f4(c.lo, i2f(cand[k]));
                r[2 * k + 1] = f4(c.hi, i2f(code[cand[k]]));
            } else {
                r[2 * k] = make_float4(0, 0, 0, i2f(-1));
                r[2 * k + 1] = make_float4(0, 0, 0, i2f(0));
            }
        }
    }
    records->swap(rec);
    code_of->swap(code);
    return true;
}

void pack_prim(const wf::Scene& host, int j, float4* out) {
    const int ns = (int)host.spheres.size();
    const long long n_prims = (long long)ns + (long long)host.triangles.size();
    const int p = host.prim_order[j];
    if (p < 0 || p >= n_prims) throw Error(WFB_ERR_INVALID_ARGUMENT, "prim_order entry out of range");
    if (p < ns) {
        const wf::Sphere& s = host.spheres[p];
        out[0] = f4(s.center, i2f(p));
        out[1] = make_float4(s.radius, 0, 0, 0);
        out[2] = make_float4(0, 0, 0, 0);
    } else {
        const wf::Triangle& t = host.triangles[p - ns];
        const wf::Vec3 p0 = host.vertices[t.i0];
        out[0] = f4(p0, i2f(p));
        out[1] = f4(host.vertices[t.i1] - p0, 0.0f);
        out[2] = f4(host.vertices[t.i2] - p0, 0.0f);
    }
}

// Nesting check of the internal nodes in [lo, hi): each one's children -- i + 1, then the skip
// link of each child in turn, up to the node's own skip link (the end of the array when the link is
// -1) -- must lie inside its box, move forward, and end exactly at its skip link. By transitivity
// every node that traversal can reach only through a passed internal node then lies inside that
// node's box, and leaving a subtree lands on its skip link. In a well-formed tree each node is the
// child of one node, so the walks take fewer steps than there are nodes; more steps mean a tree that
// is not one, and fail.
bool boxes_nested_range(const wf::BvhNode* n, int nn, int lo, int hi) {
    long long budget = nn;
    for (int i = lo; i < hi; ++i) {
        const wf::BvhNode& q = n[i];
        if (q.prim_count != 0) continue;
        const int end_i = q.skip < 0 ? nn : q.skip;
        if (end_i <= i) return false;
        int c = i + 1;
        while (c < end_i) {
            if (--budget < 0) return false;
            const wf::BvhNode& k = n[c];
            const int end_c = k.skip < 0 ? nn : k.skip;
            if (end_c <= c || end_c > end_i) return false;
            if (!(k.lo.x >= q.lo.x && k.lo.y >= q.lo.y && k.lo.z >= q.lo.z && k.hi.x <= q.hi.x &&
                  k.hi.y <= q.hi.y && k.hi.z <= q.hi.z))
                return false;
            c = end_c;
        }
    }
    return true;
}

// 1 when the preorder skip-link tree is properly nested and every node's box lies inside the box
// of each internal node whose subtree holds it (the subtree of node i: the nodes after i and before
// its skip link). Speculative traversal is exact under this condition (dev_scene.cuh, box_step); a
// tree that fails it is traversed without speculation.
int check_boxes_nested(const std::vector<wf::BvhNode>& nodes) {
    return boxes_nested_range(nodes.data(), (int)nodes.size(), 0, (int)nodes.size()) ? 1 : 0;
}

uint64_t mix_key(uint64_t h, const void* data, size_t bytes) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    size_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = fold(h, w);
    }
    for (; i < bytes; ++i) h = (h ^ p[i]) * 0x100000001B3ull;
    return h ^ (uint64_t)bytes;
}

std::shared_ptr<ResidentScene> upload_scene(const wf::Scene& host) {
    if (host.nodes.empty()) throw Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
    if (host.width <= 0 || host.height <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "scene resolution must be positive");
    if (host.materials.empty()) throw Error(WFB_ERR_INVALID_ARGUMENT, "no materials");
    const int ns = (int)host.spheres.size();
    const int nt = (int)host.triangles.size();
    const int nv = (int)host.vertices.size();
    const int nm = (int)host.materials.size();
    const int nn = (int)host.nodes.size();
    const int np = (int)host.prim_order.size();
    const int nl = (int)host.lights.size();
    const long long n_prims = (long long)ns + nt;
    // node indices stay below kNodeHeld, the traversal's speculation mark (dev_scene.cuh)
    if (nn >= kNodeHeld) throw Error(WFB_ERR_UNSUPPORTED, "BVH has 2^30 nodes or more");
    for (const wf::Sphere& s : host.spheres)
        if (s.material < 0 || s.material >= nm) throw Error(WFB_ERR_INVALID_ARGUMENT, "sphere material index out of range");
    for (const wf::Triangle& t : host.triangles) {
        if (t.material < 0 || t.material >= nm) throw Error(WFB_ERR_INVALID_ARGUMENT, "triangle material index out of range");
        if (t.i0 < 0 || t.i0 >= nv || t.i1 < 0 || t.i1 >= nv || t.i2 < 0 || t.i2 >= nv)
            throw Error(WFB_ERR_INVALID_ARGUMENT, "triangle vertex index out of range");
    }

    // One arena of 256-byte aligned parts, packed in pinned staging and copied once.
    enum { kNodes, kPrims, kSpheres, kTriShade, kTriArea, kMaterials, kLights, kParts };
    const size_t bytes[kParts] = {(size_t)2 * nn * 16,          (size_t)3 * (np > 0 ? np : 1) * 16,
                                  (size_t)2 * (ns > 0 ? ns : 1) * 16, (size_t)(nt > 0 ? nt : 1) * 16,
                                  (size_t)(nt > 0 ? nt : 1) * 4,  (size_t)nm * sizeof(wf::Material),
                                  (size_t)4 * (nl > 0 ? nl : 1) * 16};
    size_t off[kParts], total = 0;
    for (int k = 0; k < kParts; ++k) {
        off[k] = total;
        total += align256(bytes[k]);
    }
    Staging& st = staging();
    std::lock_guard<std::mutex> lock(st.mu);
    if (st.cap < total) {
        if (st.p) cuda_check(cudaFreeHost(st.p), "cudaFreeHost staging");
        st.p = nullptr;
        st.cap = 0;
        const size_t cap = (total + (16u << 20) - 1) & ~(size_t)((16u << 20) - 1);
        cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&st.p), cap, cudaHostAllocPortable), "cudaHostAlloc staging");
        st.cap = cap;
    }
    char* stage = st.p;
    // Padding, placeholder records of empty parts and unused words are zero, so the arena (and its
    // hash) depends on the scene only.
    for (int k = 0; k < kParts; ++k) std::memset(stage + off[k] + bytes[k], 0, align256(bytes[k]) - bytes[k]);
    if (np == 0) std::memset(stage + off[kPrims], 0, bytes[kPrims]);
    if (ns == 0) std::memset(stage + off[kSpheres], 0, bytes[kSpheres]);
    if (nt == 0) {
        std::memset(stage + off[kTriShade], 0, bytes[kTriShade]);
        std::memset(stage + off[kTriArea], 0, bytes[kTriArea]);
    }
    if (nl == 0) std::memset(stage + off[kLights], 0, bytes[kLights]);
    float4* nodes = reinterpret_cast<float4*>(stage + off[kNodes]);
    float4* prims = reinterpret_cast<float4*>(stage + off[kPrims]);
    float4* tri_shade = reinterpret_cast<float4*>(stage + off[kTriShade]);
    float* tri_area = reinterpret_cast<float*>(stage + off[kTriArea]);
    float4* lights = reinterpret_cast<float4*>(stage + off[kLights]);

    int nested = 0;
    const std::function<void(int, int)> pack_nodes = [&](int lo, int hi) {
        for (int i = lo; i < hi; ++i) pack_node(host, i, nodes + 2 * i);
    };
    const std::function<void(int, int)> pack_prims = [&](int lo, int hi) {
        for (int j = lo; j < hi; ++j) pack_prim(host, j, prims + 3 * j);
    };
    const std::function<void(int, int)> pack_triangles = [&](int lo, int hi) {
        // Triangle shading records and areas.
        for (int i = lo; i < hi; ++i) {
            const wf::Triangle& t = host.triangles[i];
            const wf::Vec3 e1 = host.vertices[t.i1] - host.vertices[t.i0];
            const wf::Vec3 e2 = host.vertices[t.i2] - host.vertices[t.i0];
            tri_shade[i] = f4(wf::normalize(wf::cross(e1, e2)), i2f(t.material));
            tri_area[i] = 0.5f * wf::length(wf::cross(e1, e2));
        }
    };
    auto pack_rest = [&] {
        // Spheres (wf::Sphere bytes), materials and lights.
        if (ns) std::memcpy(stage + off[kSpheres], host.spheres.data(), sizeof(wf::Sphere) * ns);
        std::memcpy(stage + off[kMaterials], host.materials.data(), sizeof(wf::Material) * nm);
        // Lights: {a, prim} {b, area} {c, material} {n, radius}.
        for (int i = 0; i < nl; ++i) {
            const int p = host.lights[i].prim;
            if (p < 0 || p >= n_prims) throw Error(WFB_ERR_INVALID_ARGUMENT, "light primitive out of range");
            if (p < ns) {
                const wf::Sphere& s = host.spheres[p];
                const float area = 4.0f * wf::kPi * s.radius * s.radius;
                lights[4 * i] = f4(s.center, i2f(p));
                lights[4 * i + 1] = make_float4(0, 0, 0, area);
                lights[4 * i + 2] = make_float4(0, 0, 0, i2f(s.material));
                lights[4 * i + 3] = make_float4(0, 0, 0, s.radius);
            } else {
                const wf::Triangle& t = host.triangles[p - ns];
                const wf::Vec3 a = host.vertices[t.i0], b = host.vertices[t.i1], c = host.vertices[t.i2];
                const wf::Vec3 e1 = b - a, e2 = c - a;
                lights[4 * i] = f4(a, i2f(p));
                lights[4 * i + 1] = f4(b, 0.5f * wf::length(wf::cross(e1, e2)));
                lights[4 * i + 2] = f4(c, i2f(t.material));
                lights[4 * i + 3] = f4(wf::normalize(wf::cross(b - a, c - a)), 0.0f);
            }
        }
    };
    // Sections in the order a serial pass would take: node ranges, the nesting check, primitive
    // ranges, triangle ranges, the rest; large scenes spread them over up to 8 threads.
    const int threads = (size_t)nn + np + nt > (1u << 16) ? (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    std::vector<std::function<void()>> sections;
    add_ranges(sections, nn, 1 << 14, threads, pack_nodes);
    std::atomic<int> nested_ok{1};
    const std::function<void(int, int)> check_nested = [&](int lo, int hi) {
        if (!boxes_nested_range(host.nodes.data(), nn, lo, hi)) nested_ok = 0;
    };
    add_ranges(sections, nn, 1 << 14, threads, check_nested);
    add_ranges(sections, np, 1 << 14, threads, pack_prims);
    add_ranges(sections, nt, 1 << 14, threads, pack_triangles);
    sections.emplace_back(pack_rest);
    run_sections(sections, threads);
    nested = nested_ok.load();

    auto rs = std::make_shared<ResidentScene>();
    cuda_check(cudaGetDevice(&rs->device), "cudaGetDevice");
    cuda_check(cudaEventCreateWithFlags(&rs->last_use, cudaEventDisableTiming), "cudaEventCreate scene use");
    const size_t n_chunks = (total / 8 + kHashChunkWords - 1) / kHashChunkWords;
    // From the stream-ordered pool (on the legacy stream, which orders the copy, the hash and the
    // read-back below): a scene created per frame reuses the memory of the one before it.
    cuda_check(cudaMallocAsync(&rs->arena, total + n_chunks * 8, 0), "allocate scene");
    rs->bytes = total;
    char* base = static_cast<char*>(rs->arena);
    cuda_check(cudaMemcpyAsync(base, stage, total, cudaMemcpyHostToDevice, 0), "cudaMemcpy scene");
    // Content key: chunk hashes of the arena (in the tail of the same allocation), folded here.
    unsigned long long* chunk_hash = reinterpret_cast<unsigned long long*>(base + total);
    (void)cudaGetLastError();  // the check below is for this launch only
    hash_chunks<<<(unsigned)((n_chunks + 255) / 256), 256, 0, 0>>>(
        reinterpret_cast<const unsigned long long*>(base), total / 8, chunk_hash);
    cuda_check(cudaGetLastError(), "hash_chunks launch");
    std::vector<unsigned long long> hashes(n_chunks);
    cuda_check(cudaMemcpy(hashes.data(), chunk_hash, n_chunks * 8, cudaMemcpyDeviceToHost), "cudaMemcpy hashes");
    uint64_t key = 0x6A09E667F3BCC909ull ^ total;
    for (unsigned long long h : hashes) key = fold(key, h);
    key = mix_key(key, &host.env, sizeof(host.env));
    rs->content_key = mix_key(key, &host.camera, sizeof(host.camera));

    DevScene& d = rs->dev;
    d.nodes = reinterpret_cast<const float4*>(base + off[kNodes]);
    d.prims = reinterpret_cast<const float4*>(base + off[kPrims]);
    d.spheres = reinterpret_cast<const float4*>(base + off[kSpheres]);
    d.tri_shade = reinterpret_cast<const float4*>(base + off[kTriShade]);
    d.tri_area = reinterpret_cast<const float*>(base + off[kTriArea]);
    d.materials = reinterpret_cast<const float4*>(base + off[kMaterials]);
    d.lights = reinterpret_cast<const float4*>(base + off[kLights]);
    d.n_spheres = ns;
    d.n_triangles = nt;
    d.n_materials = nm;
    d.n_nodes = nn;
    d.n_lights = nl;
    d.env = host.env;
    d.camera = wf::make_camera_rig(host.camera, host.width, host.height);
    d.width = host.width;
    d.height = host.height;
    d.boxes_nested = nested;
    return rs;
}

}  // namespace wfb
