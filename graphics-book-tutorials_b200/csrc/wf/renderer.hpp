// C++ renderer interface: the reference's GpuRenderer class (WVM/include/wf/renderer.hpp:11-74),
// declared identically so code written against the reference (its CLI, its GPU tests) links
// against this engine. The implementation (shim/gpu_renderer_shim.cpp, built as libwf_gpu.so) forwards every call to
// the engine's C ABI (include/wfb200.h).
#pragma once
#include <cstdint>
#include <memory>
#include <vector>
#include "wf/film.hpp"
#include "wf/scene.hpp"

namespace wf {

struct RenderParams {
    int spp = 64;
    uint32_t seed = 1234;
    int max_depth = 8;
    int threads = 0;            // CPU arm only
    bool count_rays = false;    // also count extension and shadow rays
    bool stage_timing = false;  // wavefront: per-stage times (adds synchronisation)
    int queue_capacity = 0;     // wavefront test hook: 0 = no limit; smaller values make
                                // dropped pushes counted in stats.queue_overflows
};

struct StageTimes {  // milliseconds summed over a render, wavefront only
    double extend = 0, classify = 0, shade_lambert = 0, shade_metal = 0, shade_dielectric = 0,
           shadow = 0, compact = 0, other = 0;
};

struct RenderStats {
    double render_ms = 0.0;
    double total_ms = 0.0;
    uint64_t extension_rays = 0, shadow_rays = 0;
    long long queue_high_water[5] = {0, 0, 0, 0, 0};  // lambert, metal, dielectric, shadow, active
    long long queue_overflows = 0;
    long long invalid_hits = 0;
    uint64_t peak_vram_bytes = 0;
    StageTimes stages;
};

RenderResult render_cpu(const Scene& scene, const RenderParams& p, RenderStats* stats);

enum class GpuMode { Megakernel, Wavefront };

class GpuRenderer {
public:
    GpuRenderer(const Scene& scene, GpuMode mode);
    ~GpuRenderer();
    GpuRenderer(const GpuRenderer&) = delete;
    GpuRenderer& operator=(const GpuRenderer&) = delete;

    RenderResult render(const RenderParams& p, RenderStats* stats);
    void reset();
    void run_passes(int first_sample, int count, const RenderParams& p, RenderStats* stats);
    RenderResult download(int spp_done);
    void download_mean(int spp_done, std::vector<float>* rgb);

    uint64_t device_bytes() const;
    const std::string& device_name() const;

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

struct CudaDeviceFacts {
    std::string name, driver_version, runtime_version, driver_api_version, compute_capability;
    uint64_t total_memory_bytes = 0, free_memory_bytes = 0;
};
CudaDeviceFacts query_cuda_device();

}  // namespace wf
