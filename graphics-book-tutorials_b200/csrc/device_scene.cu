// Scene upload: validation and repacking into the device layout described in dev_scene.cuh.
// Host arithmetic in this file is compiled without contraction (-ffp-contract=off) so every
// precomputed float equals the one the reference computes per ray.
#include <cstring>
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
        cudaFree(arena);
        if (device >= 0 && cur != device && cur >= 0) cudaSetDevice(cur);
    }
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

std::shared_ptr<ResidentScene> upload_scene(wf::Scene host) {
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
    for (const wf::Sphere& s : host.spheres)
        if (s.material < 0 || s.material >= nm) throw Error(WFB_ERR_INVALID_ARGUMENT, "sphere material index out of range");
    for (const wf::Triangle& t : host.triangles) {
        if (t.material < 0 || t.material >= nm) throw Error(WFB_ERR_INVALID_ARGUMENT, "triangle material index out of range");
        if (t.i0 < 0 || t.i0 >= nv || t.i1 < 0 || t.i1 >= nv || t.i2 < 0 || t.i2 >= nv)
            throw Error(WFB_ERR_INVALID_ARGUMENT, "triangle vertex index out of range");
    }

    // Nodes: {lo, skip} {hi, leaf}.
    std::vector<float4> nodes((size_t)2 * nn);
    for (int i = 0; i < nn; ++i) {
        const wf::BvhNode& n = host.nodes[i];
        int leaf = -1;
        if (n.prim_count > 0) {
            if (n.prim_count > kMaxLeafPrims)
                throw Error(WFB_ERR_UNSUPPORTED, "BVH leaf holds more than 15 primitives");
            if (n.prim_start < 0 || (long long)n.prim_start + n.prim_count > np || n.prim_start > kMaxLeafStart)
                throw Error(WFB_ERR_INVALID_ARGUMENT, "BVH leaf prim_start/count out of bounds");
            leaf = (n.prim_start << kLeafCountBits) | n.prim_count;
        }
        if (n.skip < -1 || n.skip >= nn) throw Error(WFB_ERR_INVALID_ARGUMENT, "BVH skip link out of bounds");
        // Every traversal step moves forward (to N+1 or to a forward skip), so a traversal ends
        // after at most n_nodes steps; a backward skip could loop forever and is rejected.
        if (n.skip != -1 && n.skip <= i) throw Error(WFB_ERR_INVALID_ARGUMENT, "BVH skip link does not point forward");
        nodes[2 * i] = f4(n.lo, i2f(n.skip));
        nodes[2 * i + 1] = f4(n.hi, i2f(leaf));
    }
    // Leaf primitive records in prim_order order.
    std::vector<float4> prims((size_t)3 * (np > 0 ? np : 1), make_float4(0, 0, 0, 0));
    for (int j = 0; j < np; ++j) {
        const int p = host.prim_order[j];
        if (p < 0 || p >= n_prims) throw Error(WFB_ERR_INVALID_ARGUMENT, "prim_order entry out of range");
        if (p < ns) {
            const wf::Sphere& s = host.spheres[p];
            prims[3 * j] = f4(s.center, i2f(p));
            prims[3 * j + 1] = make_float4(s.radius, 0, 0, 0);
        } else {
            const wf::Triangle& t = host.triangles[p - ns];
            const wf::Vec3 p0 = host.vertices[t.i0];
            prims[3 * j] = f4(p0, i2f(p));
            prims[3 * j + 1] = f4(host.vertices[t.i1] - p0, 0.0f);
            prims[3 * j + 2] = f4(host.vertices[t.i2] - p0, 0.0f);
        }
    }
    // Spheres (wf::Sphere bytes), triangle shading records and areas, materials.
    std::vector<float4> spheres((size_t)2 * (ns > 0 ? ns : 1), make_float4(0, 0, 0, 0));
    if (ns) std::memcpy(spheres.data(), host.spheres.data(), sizeof(wf::Sphere) * ns);
    std::vector<float4> tri_shade(nt > 0 ? nt : 1, make_float4(0, 0, 0, 0));
    std::vector<float> tri_area(nt > 0 ? nt : 1, 0.0f);
    for (int i = 0; i < nt; ++i) {
        const wf::Triangle& t = host.triangles[i];
        const wf::Vec3 e1 = host.vertices[t.i1] - host.vertices[t.i0];
        const wf::Vec3 e2 = host.vertices[t.i2] - host.vertices[t.i0];
        tri_shade[i] = f4(wf::normalize(wf::cross(e1, e2)), i2f(t.material));
        tri_area[i] = 0.5f * wf::length(wf::cross(e1, e2));
    }
    std::vector<float4> materials((size_t)3 * nm);
    std::memcpy(materials.data(), host.materials.data(), sizeof(wf::Material) * nm);
    // Lights: {a, prim} {b, area} {c, material} {n, radius}.
    std::vector<float4> lights((size_t)4 * (nl > 0 ? nl : 1), make_float4(0, 0, 0, 0));
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

    // One arena, 256-byte aligned sub-buffers.
    struct Part {
        const void* src;
        size_t bytes;
        size_t off;
    };
    Part parts[] = {{nodes.data(), nodes.size() * 16, 0},       {prims.data(), prims.size() * 16, 0},
                    {spheres.data(), spheres.size() * 16, 0},   {tri_shade.data(), tri_shade.size() * 16, 0},
                    {tri_area.data(), tri_area.size() * 4, 0},  {materials.data(), materials.size() * 16, 0},
                    {lights.data(), lights.size() * 16, 0}};
    size_t total = 0;
    for (Part& p : parts) {
        p.off = total;
        total += align256(p.bytes);
    }
    auto rs = std::make_shared<ResidentScene>();
    cuda_check(cudaGetDevice(&rs->device), "cudaGetDevice");
    cuda_check(cudaMalloc(&rs->arena, total), "cudaMalloc scene");
    rs->bytes = total;
    char* base = static_cast<char*>(rs->arena);
    for (const Part& p : parts)
        cuda_check(cudaMemcpy(base + p.off, p.src, p.bytes, cudaMemcpyHostToDevice), "cudaMemcpy scene");
    DevScene& d = rs->dev;
    d.nodes = reinterpret_cast<const float4*>(base + parts[0].off);
    d.prims = reinterpret_cast<const float4*>(base + parts[1].off);
    d.spheres = reinterpret_cast<const float4*>(base + parts[2].off);
    d.tri_shade = reinterpret_cast<const float4*>(base + parts[3].off);
    d.tri_area = reinterpret_cast<const float*>(base + parts[4].off);
    d.materials = reinterpret_cast<const float4*>(base + parts[5].off);
    d.lights = reinterpret_cast<const float4*>(base + parts[6].off);
    d.n_spheres = ns;
    d.n_triangles = nt;
    d.n_materials = nm;
    d.n_nodes = nn;
    d.n_lights = nl;
    d.env = host.env;
    d.camera = wf::make_camera_rig(host.camera, host.width, host.height);
    d.width = host.width;
    d.height = host.height;
    rs->host = std::move(host);
    return rs;
}

}  // namespace wfb
