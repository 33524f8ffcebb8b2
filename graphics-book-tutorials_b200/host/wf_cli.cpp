// `wf render ...`: the reference's command line (flags: WVM/include/wf/config.hpp:30-34; flow:
// WVM/src/main.cpp:34-203) on this engine's GPU arms.
//
// Scenes: the reference's procedural names (cornell, divergence, trianglehv, furnace), a path to an
// .obj file, or one of this engine's benchmark generators (cornell36, icospheres, heightfield;
// generator seed 1234, 16-bin SAH). --mode megakernel | wavefront render on the GPU through
// wf::GpuRenderer; --mode cpu is refused (this engine has no CPU arm: there is no fallback).
// Timed repetitions reuse one renderer (the scene is uploaded once); each run's render_ms is the
// CUDA-event time of its passes, as in the reference. --out writes PREFIX.png (tone-mapped) and
// PREFIX.pfm; --report writes report.json (schema 1) after one untimed ray-counting render.
// Exit status: 0 on success, 1 on an error (message on stderr).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
#include "scene_gen.hpp"
#include "wf/config.hpp"
#include "wf/film.hpp"
#include "wf/image_io.hpp"
#include "wf/renderer.hpp"
#include "wf/report.hpp"
#include "wf/scene.hpp"

namespace {

std::string git_revision() {
    FILE* p = popen("git rev-parse HEAD 2>/dev/null", "r");
    if (!p) return "";
    char buf[96] = {0};
    const size_t n = fread(buf, 1, sizeof buf - 1, p);
    pclose(p);
    std::string rev(buf, n);
    while (!rev.empty() && (rev.back() == '\n' || rev.back() == '\r' || rev.back() == ' ')) rev.pop_back();
    return rev;
}

bool ends_with(const std::string& s, const std::string& suffix) {
    return s.size() >= suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0;
}

wf::Scene load_scene(const wf::Config& c) {
    if (ends_with(c.scene, ".obj")) return wf::load_obj(c.scene, c.width, c.height);
    if (c.scene == "cornell36" || c.scene == "icospheres" || c.scene == "heightfield")
        return wfb::make_config_scene(c.scene, c.width, c.height, 1234u, 16);
    return wf::make_scene(c.scene, c.width, c.height);
}

int run(const wf::Config& c) {
    if (c.mode == wf::Mode::Cpu) {
        std::cerr << "Error: --mode cpu: this engine renders on the GPU only (megakernel or wavefront)\n";
        return 1;
    }
    const wf::Scene scene = load_scene(c);
    const wf::GpuMode gm = c.mode == wf::Mode::Megakernel ? wf::GpuMode::Megakernel : wf::GpuMode::Wavefront;
    wf::RenderParams p;
    p.spp = c.spp;
    p.seed = c.seed;
    p.max_depth = c.max_depth;
    p.threads = c.threads;
    wf::GpuRenderer renderer(scene, gm);
    for (int i = 0; i < c.warmup; ++i) renderer.render(p, nullptr);
    std::vector<double> runs;
    wf::RenderResult result;
    wf::RenderStats stats;
    for (int i = 0; i < c.reps; ++i) {
        stats = wf::RenderStats{};
        result = renderer.render(p, &stats);
        runs.push_back(stats.render_ms);
    }
    std::string png, pfm;
    if (!c.out_prefix.empty()) {
        png = c.out_prefix + ".png";
        pfm = c.out_prefix + ".pfm";
        wf::write_png(png, result.width, result.height, wf::tonemap_to_srgb8(result.rgb));
        wf::write_pfm(pfm, result.width, result.height, result.rgb);
    }
    const double median_ms = wf::percentile(runs, 0.5);
    const double samples = (double)c.width * (double)c.height * (double)c.spp;
    std::printf("%s %s %dx%d %d spp: median %.3f ms, %.2f Msamples/s\n", c.scene.c_str(), wf::mode_name(c.mode).c_str(),
                c.width, c.height, c.spp, median_ms, median_ms > 0.0 ? samples / median_ms / 1e3 : 0.0);
    if (c.report_path.empty()) return 0;

    wf::Report r;
    r.git_revision = git_revision();
    r.scene_name = c.scene;
    r.scene_hash = wf::scene_hash(scene);
    r.width = c.width;
    r.height = c.height;
    r.spp = c.spp;
    r.max_depth = c.max_depth;
    r.seed = c.seed;
    r.mode = wf::mode_name(c.mode);
    r.run_ms = runs;
    if (median_ms > 0.0) r.samples_per_second = samples / (median_ms / 1e3);
    for (int i = 0; i < 5; ++i) r.queue_high_water[i] = stats.queue_high_water[i];
    r.queue_overflows = stats.queue_overflows;
    r.invalid_hits = stats.invalid_hits;
    r.peak_vram_bytes = stats.peak_vram_bytes;
    r.image_png = png;
    r.image_pfm = pfm;
    r.pfm_hash = wf::fnv1a64(result.rgb.data(), result.rgb.size() * sizeof(float));
    r.nonfinite_pixels = wf::count_nonfinite(result.rgb);
    {
        // rays per second: one separate, untimed counting render (counting never touches the timings)
        wf::RenderParams counting = p;
        counting.count_rays = true;
        wf::RenderStats cs;
        renderer.render(counting, &cs);
        const double rays = (double)cs.extension_rays + (double)cs.shadow_rays;
        if (median_ms > 0.0 && rays > 0.0) r.rays_per_second = rays / (median_ms / 1e3);
    }
    const wf::CudaDeviceFacts f = wf::query_cuda_device();
    r.device.name = f.name;
    r.device.driver_version = f.driver_version;
    r.device.cuda_runtime_version = f.runtime_version;
    r.device.cuda_driver_version = f.driver_api_version;
    r.device.compute_capability = f.compute_capability;
    r.device.total_memory_bytes = f.total_memory_bytes;
    const std::string text = wf::report_to_json(r);
    const std::string problem = wf::validate_report_json(text);
    if (!problem.empty()) {
        std::cerr << "Error: report failed validation: " << problem << "\n";
        return 1;
    }
    std::ofstream out(c.report_path, std::ios::binary | std::ios::trunc);
    out << text;
    out.close();
    if (!out) {
        std::cerr << "Error: cannot write " << c.report_path << "\n";
        return 1;
    }
    return 0;
}

}  // namespace

int main(int argc, const char* argv[]) {
    try {
        return run(wf::parse_args(argc, argv));
    } catch (const wf::ConfigError& e) {
        std::cerr << "Error: " << e.what() << "\n" << wf::usage();
        return 1;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 1;
    }
}
