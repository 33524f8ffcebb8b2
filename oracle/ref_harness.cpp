// ORACLE -- test infrastructure only.
//
// extern "C" access to the REFERENCE implementation, compiled from its own sources (see
// oracle/Makefile; nothing here is shipped with the engine). It lets the parity tests feed the
// reference the same scene arrays the engine renders:
//   ref_render_cpu    wf::render_cpu        (WVM/src/cpu_renderer.cpp:13)
//   ref_render_gpu    wf::GpuRenderer::render for both GPU arms (WVM/src/gpu/gpu_renderer.cu:355)
//   ref_build_bvh     wf::build_bvh         (WVM/src/bvh_build.cpp:228)
//   ref_scene_hash    wf::scene_hash        (WVM/src/scene.cpp:107)
//   ref_make_scene    wf::make_scene        (WVM/src/scenes.cpp:29), exported as arrays
//   ref_scan / ref_compact / ref_queue_push   wf::gpu queue primitives (WVM/src/gpu/queues.cu)
// The scene struct below has the same field order as the engine's wfb_scene_desc.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "wf/bvh.hpp"
#include "wf/renderer.hpp"
#include "wf/scene.hpp"

// Host-side interface of the reference queue primitives (WVM/src/gpu/queues.cuh:30-55), declared
// here so this file stays host-only C++ (the header also carries device code).
namespace wf::gpu {
struct ScanWorkspace {
    uint32_t* block_sums = nullptr;
    int capacity = 0;
};
cudaError_t scan_workspace_create(ScanWorkspace* ws, int capacity);
void scan_workspace_destroy(ScanWorkspace* ws);
cudaError_t scan_exclusive_u32(const uint32_t* d_in, uint32_t* d_out, int n, uint32_t* d_total, ScanWorkspace& ws,
                               cudaStream_t stream);
cudaError_t compact_u32(const uint32_t* d_values, const uint32_t* d_flags, uint32_t* d_out, uint32_t* d_count,
                        uint32_t* d_scratch, int n, ScanWorkspace& ws, cudaStream_t stream);
cudaError_t test_queue_push(const uint32_t* d_flags, int n, uint32_t* d_items, uint32_t capacity, uint32_t* d_counter,
                            uint32_t* d_overflow, cudaStream_t stream);
}  // namespace wf::gpu

namespace {

struct RefSceneDesc {
    const void* spheres; int n_spheres;
    const float* vertices; int n_vertices;
    const int* triangles; int n_triangles;
    const void* materials; int n_materials;
    const void* nodes; int n_nodes;
    const int* prim_order; int n_prim_order;
    const void* lights; int n_lights;
    float env[3];
    float cam_position[3], cam_look_at[3], cam_up[3], cam_vfov_deg;
    int width, height;
};

template <class T>
void fill(std::vector<T>& v, const void* src, int n) {
    v.resize((size_t)n);
    if (n > 0) std::memcpy(v.data(), src, sizeof(T) * (size_t)n);
}

wf::Scene to_scene(const RefSceneDesc* d) {
    wf::Scene s;
    fill(s.spheres, d->spheres, d->n_spheres);
    fill(s.vertices, d->vertices, d->n_vertices);
    fill(s.triangles, d->triangles, d->n_triangles);
    fill(s.materials, d->materials, d->n_materials);
    fill(s.nodes, d->nodes, d->n_nodes);
    fill(s.prim_order, d->prim_order, d->n_prim_order);
    fill(s.lights, d->lights, d->n_lights);
    s.env = wf::Vec3{d->env[0], d->env[1], d->env[2]};
    s.camera.position = wf::Vec3{d->cam_position[0], d->cam_position[1], d->cam_position[2]};
    s.camera.look_at = wf::Vec3{d->cam_look_at[0], d->cam_look_at[1], d->cam_look_at[2]};
    s.camera.up = wf::Vec3{d->cam_up[0], d->cam_up[1], d->cam_up[2]};
    s.camera.vfov_deg = d->cam_vfov_deg;
    s.width = d->width;
    s.height = d->height;
    return s;
}

std::string g_err;

wf::RenderParams params(int spp, uint32_t seed, int max_depth, int threads) {
    wf::RenderParams p;
    p.spp = spp;
    p.seed = seed;
    p.max_depth = max_depth;
    p.threads = threads;
    return p;
}

void copy_out(const wf::RenderResult& r, float* rgb, float* lum_var) {
    if (rgb) std::memcpy(rgb, r.rgb.data(), r.rgb.size() * sizeof(float));
    if (lum_var) std::memcpy(lum_var, r.lum_var.data(), r.lum_var.size() * sizeof(float));
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// stats_out (optional, 8 doubles): render_ms, ext rays, shadow rays, invalid hits, overflows,
// high_water[0..2].
int ref_render_cpu(const RefSceneDesc* d, int spp, uint32_t seed, int max_depth, int threads, float* rgb,
                   float* lum_var, double* render_ms) {
    try {
        const wf::Scene s = to_scene(d);
        wf::RenderStats st{};
        const wf::RenderResult r = wf::render_cpu(s, params(spp, seed, max_depth, threads), &st);
        copy_out(r, rgb, lum_var);
        if (render_ms) *render_ms = st.render_ms;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ref_render_gpu(const RefSceneDesc* d, int mode, int spp, uint32_t seed, int max_depth, int count_rays,
                   int queue_capacity, float* rgb, float* lum_var, double* stats_out) {
    try {
        const wf::Scene s = to_scene(d);
        wf::GpuRenderer r(s, mode == 1 ? wf::GpuMode::Wavefront : wf::GpuMode::Megakernel);
        wf::RenderParams p = params(spp, seed, max_depth, 0);
        p.count_rays = count_rays != 0;
        p.queue_capacity = queue_capacity;
        wf::RenderStats st{};
        const wf::RenderResult out = r.render(p, &st);
        copy_out(out, rgb, lum_var);
        if (stats_out) {
            stats_out[0] = st.render_ms;
            stats_out[1] = (double)st.extension_rays;
            stats_out[2] = (double)st.shadow_rays;
            stats_out[3] = (double)st.invalid_hits;
            stats_out[4] = (double)st.queue_overflows;
            for (int i = 0; i < 3; ++i) stats_out[5 + i] = (double)st.queue_high_water[i];
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Builds the reference BVH (8-bin SAH) for the scene; nodes (48 B each) and prim_order are
// written to caller buffers of capacity cap_nodes / cap_prims; counts returned in *n_nodes, *n_prims.
int ref_build_bvh(const RefSceneDesc* d, void* nodes, int cap_nodes, int* prim_order, int cap_prims, int* n_nodes,
                  int* n_prims) {
    try {
        wf::Scene s = to_scene(d);
        wf::build_bvh(s);
        *n_nodes = (int)s.nodes.size();
        *n_prims = (int)s.prim_order.size();
        if (*n_nodes > cap_nodes || *n_prims > cap_prims) return 2;
        std::memcpy(nodes, s.nodes.data(), s.nodes.size() * sizeof(wf::BvhNode));
        std::memcpy(prim_order, s.prim_order.data(), s.prim_order.size() * sizeof(int));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

uint64_t ref_scene_hash(const RefSceneDesc* d) { return wf::scene_hash(to_scene(d)); }

// Procedural reference scene, handed out as a heap object plus array accessors.
void* ref_make_scene(const char* name, int width, int height) {
    try {
        return new wf::Scene(wf::make_scene(name, width, height));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_scene_counts(const void* h, int* counts /* 7 */) {
    const wf::Scene* s = static_cast<const wf::Scene*>(h);
    counts[0] = (int)s->spheres.size();
    counts[1] = (int)s->vertices.size();
    counts[2] = (int)s->triangles.size();
    counts[3] = (int)s->materials.size();
    counts[4] = (int)s->nodes.size();
    counts[5] = (int)s->prim_order.size();
    counts[6] = (int)s->lights.size();
}

// Fills a RefSceneDesc whose array pointers point into the heap scene (valid until ref_scene_free).
void ref_scene_view(const void* h, RefSceneDesc* d) {
    const wf::Scene* s = static_cast<const wf::Scene*>(h);
    d->spheres = s->spheres.data(); d->n_spheres = (int)s->spheres.size();
    d->vertices = reinterpret_cast<const float*>(s->vertices.data()); d->n_vertices = (int)s->vertices.size();
    d->triangles = reinterpret_cast<const int*>(s->triangles.data()); d->n_triangles = (int)s->triangles.size();
    d->materials = s->materials.data(); d->n_materials = (int)s->materials.size();
    d->nodes = s->nodes.data(); d->n_nodes = (int)s->nodes.size();
    d->prim_order = s->prim_order.data(); d->n_prim_order = (int)s->prim_order.size();
    d->lights = s->lights.data(); d->n_lights = (int)s->lights.size();
    const float env[3] = {s->env.x, s->env.y, s->env.z};
    std::memcpy(d->env, env, sizeof(env));
    const wf::Camera& c = s->camera;
    const float pos[3] = {c.position.x, c.position.y, c.position.z};
    const float at[3] = {c.look_at.x, c.look_at.y, c.look_at.z};
    const float up[3] = {c.up.x, c.up.y, c.up.z};
    std::memcpy(d->cam_position, pos, sizeof(pos));
    std::memcpy(d->cam_look_at, at, sizeof(at));
    std::memcpy(d->cam_up, up, sizeof(up));
    d->cam_vfov_deg = c.vfov_deg;
    d->width = s->width;
    d->height = s->height;
}

void ref_scene_free(void* h) { delete static_cast<wf::Scene*>(h); }

// Queue primitives on device pointers; each call makes its own workspace and synchronises.
int ref_scan(const uint32_t* d_in, uint32_t* d_out, int n, uint32_t* d_total, int capacity) {
    wf::gpu::ScanWorkspace ws;
    cudaError_t e = wf::gpu::scan_workspace_create(&ws, capacity);
    if (e != cudaSuccess) return (int)e;
    e = wf::gpu::scan_exclusive_u32(d_in, d_out, n, d_total, ws, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    wf::gpu::scan_workspace_destroy(&ws);
    return (int)e;
}

int ref_compact(const uint32_t* d_values, const uint32_t* d_flags, uint32_t* d_out, uint32_t* d_count,
                uint32_t* d_scratch, int n, int capacity) {
    wf::gpu::ScanWorkspace ws;
    cudaError_t e = wf::gpu::scan_workspace_create(&ws, capacity);
    if (e != cudaSuccess) return (int)e;
    e = wf::gpu::compact_u32(d_values, d_flags, d_out, d_count, d_scratch, n, ws, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    wf::gpu::scan_workspace_destroy(&ws);
    return (int)e;
}

int ref_queue_push(const uint32_t* d_flags, int n, uint32_t* d_items, uint32_t capacity, uint32_t* d_counter,
                   uint32_t* d_overflow) {
    cudaError_t e = wf::gpu::test_queue_push(d_flags, n, d_items, capacity, d_counter, d_overflow, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

}  // extern "C"
