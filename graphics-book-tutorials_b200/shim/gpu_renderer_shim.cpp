// wf::GpuRenderer and wf::query_cuda_device over the C ABI: the drop-in for the reference's GPU
// library (WVM/src/gpu/gpu_renderer.cu). Code written against WVM/include/wf/renderer.hpp -- the
// reference's CLI, bench and GPU tests -- links against libwf_gpu.so (+ libwfb200.so) instead of
// the reference's libwfgpu.a and renders through this engine, with the same bits.
//
// Contract kept from the reference:
//   - the constructor uploads the scene and throws std::runtime_error for a scene without BVH
//     nodes (gpu_renderer.cu:100-104) or on any engine/CUDA error;
//   - render() = reset(); run_passes(0, spp) into fresh stats; download(spp) (gpu_renderer.cu:356-365);
//   - run_passes adds ray counts, overflows and invalid hits to *stats, keeps the queue high-water
//     maxima, adds stage times, and sets render_ms and peak_vram_bytes (gpu_renderer.cu:249-304);
//   - download / download_mean use the reference film convention (mean = sum * (1/spp), variance
//     in double clamped at 0, gpu_renderer.cu:306-341).
// Differences: download(spp_done <= 0) throws instead of returning a non-finite image, and the
// renderer runs on its own stream (synchronous to the caller, like the reference's stream 0).
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include "wf/renderer.hpp"
#include "../../include/wfb200.h"

namespace wf {
namespace {

void check(int status, const char* what) {
    if (status != WFB_OK) throw std::runtime_error(std::string(what) + ": " + wfb_last_error());
}

std::string version_string(int v) { return std::to_string(v / 1000) + "." + std::to_string((v % 1000) / 10); }

}  // namespace

CudaDeviceFacts query_cuda_device() {
    wfb_device_facts f{};
    check(wfb_device_facts_get(&f), "query_cuda_device");
    CudaDeviceFacts out;
    out.name = f.name;
    out.driver_version = version_string(f.driver_version);
    out.runtime_version = version_string(f.runtime_version);
    out.driver_api_version = std::to_string(f.driver_version);
    out.compute_capability = std::to_string(f.cc_major) + "." + std::to_string(f.cc_minor);
    out.total_memory_bytes = f.total_memory_bytes;
    out.free_memory_bytes = f.free_memory_bytes;
    return out;
}

struct GpuRenderer::Impl {
    wfb_scene_t scene = nullptr;
    wfb_renderer_t r = nullptr;
    int width = 0, height = 0;
    ~Impl() {
        if (r) wfb_renderer_destroy(r);
        if (scene) wfb_scene_destroy(scene);
    }
};

GpuRenderer::GpuRenderer(const Scene& scene, GpuMode mode) : impl_(std::make_unique<Impl>()) {
    if (scene.nodes.empty()) throw std::runtime_error("Scene not finalized (no BVH nodes)");
    wfb_scene_desc d{};
    d.spheres = scene.spheres.data();
    d.n_spheres = (int)scene.spheres.size();
    d.vertices = reinterpret_cast<const float*>(scene.vertices.data());
    d.n_vertices = (int)scene.vertices.size();
    d.triangles = reinterpret_cast<const int*>(scene.triangles.data());
    d.n_triangles = (int)scene.triangles.size();
    d.materials = scene.materials.data();
    d.n_materials = (int)scene.materials.size();
    d.nodes = scene.nodes.data();
    d.n_nodes = (int)scene.nodes.size();
    d.prim_order = scene.prim_order.data();
    d.n_prim_order = (int)scene.prim_order.size();
    d.lights = scene.lights.data();
    d.n_lights = (int)scene.lights.size();
    const Vec3 env = scene.env, pos = scene.camera.position, at = scene.camera.look_at, up = scene.camera.up;
    const float f[4][3] = {{env.x, env.y, env.z}, {pos.x, pos.y, pos.z}, {at.x, at.y, at.z}, {up.x, up.y, up.z}};
    for (int k = 0; k < 3; ++k) {
        d.env[k] = f[0][k];
        d.cam_position[k] = f[1][k];
        d.cam_look_at[k] = f[2][k];
        d.cam_up[k] = f[3][k];
    }
    d.cam_vfov_deg = scene.camera.vfov_deg;
    d.width = scene.width;
    d.height = scene.height;
    check(wfb_scene_create(&d, 0, &impl_->scene), "scene upload");
    check(wfb_renderer_create(impl_->scene, mode == GpuMode::Wavefront ? WFB_MODE_WAVEFRONT : WFB_MODE_MEGAKERNEL,
                              &impl_->r),
          "GpuRenderer");
    impl_->width = scene.width;
    impl_->height = scene.height;
}

GpuRenderer::~GpuRenderer() = default;

void GpuRenderer::reset() { check(wfb_renderer_reset(impl_->r), "reset"); }

void GpuRenderer::run_passes(int first_sample, int count, const RenderParams& p, RenderStats* stats) {
    wfb_render_params cp{};
    cp.spp = count;
    cp.seed = p.seed;
    cp.max_depth = p.max_depth;
    cp.count_rays = p.count_rays ? 1 : 0;
    cp.stage_timing = p.stage_timing ? 1 : 0;
    cp.queue_capacity = p.queue_capacity;
    wfb_render_stats cs{};
    check(wfb_renderer_run_passes(impl_->r, first_sample, count, &cp, &cs), "run_passes");
    if (!stats) return;
    stats->extension_rays += cs.extension_rays;
    stats->shadow_rays += cs.shadow_rays;
    stats->invalid_hits += cs.invalid_hits;
    stats->queue_overflows += cs.queue_overflows;
    for (int j = 0; j < 5; ++j)
        if (cs.queue_high_water[j] > stats->queue_high_water[j]) stats->queue_high_water[j] = cs.queue_high_water[j];
    StageTimes& s = stats->stages;
    s.extend += cs.stage_ms[0];
    s.classify += cs.stage_ms[1];
    s.shade_lambert += cs.stage_ms[2];
    s.shade_metal += cs.stage_ms[3];
    s.shade_dielectric += cs.stage_ms[4];
    s.shadow += cs.stage_ms[5];
    s.compact += cs.stage_ms[6];
    s.other += cs.stage_ms[7];
    stats->render_ms = cs.render_ms;
    stats->peak_vram_bytes = cs.peak_vram_bytes;
}

RenderResult GpuRenderer::download(int spp_done) {
    RenderResult res;
    res.width = impl_->width;
    res.height = impl_->height;
    res.spp = spp_done;
    const size_t pixels = (size_t)impl_->width * (size_t)impl_->height;
    res.rgb.resize(3 * pixels);
    res.lum_var.resize(pixels);
    check(wfb_renderer_download(impl_->r, spp_done, res.rgb.data(), res.lum_var.data()), "download");
    return res;
}

void GpuRenderer::download_mean(int spp_done, std::vector<float>* rgb) {
    if (!rgb) return;
    rgb->resize(3 * (size_t)impl_->width * (size_t)impl_->height);
    check(wfb_renderer_download_mean(impl_->r, spp_done, rgb->data()), "download_mean");
}

RenderResult GpuRenderer::render(const RenderParams& p, RenderStats* stats) {
    reset();
    RenderStats local{};
    run_passes(0, p.spp, p, &local);
    if (stats) *stats = local;
    return download(p.spp);
}

uint64_t GpuRenderer::device_bytes() const { return wfb_renderer_device_bytes(impl_->r); }

const std::string& GpuRenderer::device_name() const {
    static const std::string name = [] {
        wfb_device_facts f{};
        return wfb_device_facts_get(&f) == WFB_OK ? std::string(f.name) : std::string("unknown");
    }();
    return name;
}

}  // namespace wf
