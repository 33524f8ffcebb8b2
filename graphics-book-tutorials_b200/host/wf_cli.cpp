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
//
// `wf batch` and `wf serve` (no reference counterpart) render a job list through the C ABI:
//   wf batch --jobs FILE.json [--mode megakernel|wavefront] [--reps N] [--out-dir DIR]
//     every job in one persistent launch (the megakernel replayed as a CUDA graph); prints one JSON
//     line: median device time over --reps runs, Msamples/s and each job's FNV-1a rgb hash;
//     --out-dir writes DIR/job_NNN.pfm.
//   wf serve --jobs FILE.json [--lambda JOBS_PER_S] [--duration S] [--drain S] [--seed N]
//            [--mode megakernel|wavefront] [--plain]
//     open-loop Poisson arrivals drawn uniformly from the list into the continuous-batching
//     server (--plain: one job per launch); prints one JSON line with p50/p95/p99 latency
//     (submit -> film on the host) and Msamples/s.
// A job list is {"jobs": [{"scene", "width", "height", "spp", "max_depth", "seed", "cam_position",
// "cam_look_at", "cam_up", "cam_vfov_deg"}, ...]} with scenes from the benchmark generators
// (tests/golden/job_mix_64_seed1234.json is the 64-job benchmark mix).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include "../../include/wfb200.h"
#include "wf/json.hpp"
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

// ---- wf batch / wf serve ----------------------------------------------------------------------

const char* kJobsUsage =
    "Usage: batch --jobs FILE.json [--mode megakernel|wavefront] [--reps N] [--out-dir DIR]\n"
    "       serve --jobs FILE.json [--lambda JOBS_PER_S] [--duration S] [--drain S] [--seed N]\n"
    "             [--mode megakernel|wavefront] [--plain]\n";

struct JobArgs {
    std::string jobs_path, out_dir, mode = "megakernel";
    int reps = 3;
    double lambda = 10.0, duration = 10.0, drain = 30.0;
    unsigned long long seed = 1234;
    bool plain = false;
};

struct JobEntry {
    std::string scene;
    wfb_job_desc desc{};
};

void check(int status, const char* what) {
    if (status != WFB_OK) {
        const char* e = wfb_last_error();
        throw std::runtime_error(std::string(what) + ": " + (e ? e : "error"));
    }
}

double number_arg(const std::string& flag, const char* text) {
    char* end = nullptr;
    const double v = std::strtod(text, &end);
    if (end == text || *end != '\0') throw wf::ConfigError(flag + " expects a number, got '" + text + "'");
    return v;
}

JobArgs parse_job_args(int argc, const char* argv[]) {
    JobArgs a;
    const bool serve = std::string(argv[1]) == "serve";
    for (int i = 2; i < argc; ++i) {
        const std::string f = argv[i];
        if (f == "--plain" && serve) {
            a.plain = true;
            continue;
        }
        if (i + 1 >= argc) throw wf::ConfigError("missing value for " + f);
        const char* v = argv[++i];
        if (f == "--jobs") a.jobs_path = v;
        else if (f == "--mode") a.mode = v;
        else if (f == "--reps" && !serve) a.reps = (int)number_arg(f, v);
        else if (f == "--out-dir" && !serve) a.out_dir = v;
        else if (f == "--lambda" && serve) a.lambda = number_arg(f, v);
        else if (f == "--duration" && serve) a.duration = number_arg(f, v);
        else if (f == "--drain" && serve) a.drain = number_arg(f, v);
        else if (f == "--seed" && serve) a.seed = (unsigned long long)number_arg(f, v);
        else throw wf::ConfigError("unknown flag " + f);
    }
    if (a.jobs_path.empty()) throw wf::ConfigError("--jobs is required");
    if (a.mode != "megakernel" && a.mode != "wavefront") throw wf::ConfigError("--mode must be megakernel or wavefront");
    if (a.reps < 1 || a.reps > 1000) throw wf::ConfigError("--reps must be in 1..1000");
    if (!(a.lambda > 0.0) || !(a.duration > 0.0) || !(a.drain >= 0.0))
        throw wf::ConfigError("--lambda and --duration must be positive, --drain non-negative");
    return a;
}

float f32_of(const wf::Json& j, const char* key) {
    const wf::Json& v = j.at(key);
    if (v.type != wf::Json::Number) throw std::runtime_error(std::string("job field ") + key + " must be a number");
    return (float)v.num;
}

int int_of(const wf::Json& j, const char* key, int lo, int hi) {
    const wf::Json& v = j.at(key);
    if (v.type != wf::Json::Number || v.num != (double)(long long)v.num || v.num < lo || v.num > hi)
        throw std::runtime_error(std::string("job field ") + key + " must be an integer in " + std::to_string(lo) +
                                 ".." + std::to_string(hi));
    return (int)v.num;
}

void vec3_of(const wf::Json& j, const char* key, float out[3]) {
    const wf::Json& v = j.at(key);
    if (v.type != wf::Json::Array || v.arr.size() != 3) throw std::runtime_error(std::string("job field ") + key + " must be 3 numbers");
    for (int k = 0; k < 3; ++k) {
        if (v.arr[k].type != wf::Json::Number) throw std::runtime_error(std::string("job field ") + key + " must be 3 numbers");
        out[k] = (float)v.arr[k].num;
    }
}

std::vector<JobEntry> load_jobs(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot read " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    const wf::Json root = wf::json_parse(ss.str());
    if (!root.has("jobs") || root.at("jobs").type != wf::Json::Array) throw std::runtime_error(path + ": no \"jobs\" array");
    std::vector<JobEntry> jobs;
    for (const wf::Json& j : root.at("jobs").arr) {
        try {
            if (j.type != wf::Json::Object) throw std::runtime_error("a job must be an object");
            JobEntry e;
            const wf::Json& sc = j.at("scene");
            if (sc.type != wf::Json::String) throw std::runtime_error("job field scene must be a string");
            e.scene = sc.str;
            if (e.scene != "cornell36" && e.scene != "icospheres" && e.scene != "heightfield")
                throw std::runtime_error("scene '" + e.scene + "' is not a benchmark generator");
            e.desc.width = int_of(j, "width", 1, 16384);
            e.desc.height = int_of(j, "height", 1, 16384);
            e.desc.spp = int_of(j, "spp", 1, 1 << 20);
            e.desc.max_depth = int_of(j, "max_depth", 0, 1024);
            e.desc.seed = (uint32_t)int_of(j, "seed", 0, 2147483647);
            vec3_of(j, "cam_position", e.desc.cam_position);
            vec3_of(j, "cam_look_at", e.desc.cam_look_at);
            vec3_of(j, "cam_up", e.desc.cam_up);
            e.desc.cam_vfov_deg = f32_of(j, "cam_vfov_deg");
            jobs.push_back(e);
        } catch (const std::out_of_range&) {
            throw std::runtime_error(path + ": job " + std::to_string(jobs.size()) + " misses a field");
        } catch (const std::runtime_error& e) {
            throw std::runtime_error(path + ": job " + std::to_string(jobs.size()) + ": " + e.what());
        }
    }
    if (jobs.empty()) throw std::runtime_error(path + ": the job list is empty");
    return jobs;
}

// The benchmark scenes the jobs name, generated once (seed 1234, 16-bin SAH) and shared.
struct SceneSet {
    std::map<std::string, wfb_scene_t> by_name;
    explicit SceneSet(const std::vector<JobEntry>& jobs) {
        for (const JobEntry& j : jobs)
            if (!by_name.count(j.scene)) {
                wfb_scene_t s = nullptr;
                check(wfb_scene_generate(j.scene.c_str(), 64, 64, 1234u, 16, &s), "generate scene");
                by_name[j.scene] = s;
            }
    }
    ~SceneSet() {
        for (auto& kv : by_name) wfb_scene_destroy(kv.second);
    }
};

wfb_launch_config launch_config(const JobArgs& a) {
    wfb_launch_config c{};
    c.mode = a.mode == "wavefront" ? WFB_MODE_WAVEFRONT : WFB_MODE_MEGAKERNEL;
    c.use_graph = 1;
    c.occupancy = -1;
    return c;
}

double samples_of(const wfb_job_desc& d) { return (double)d.width * d.height * d.spp; }

int run_batch(const JobArgs& a) {
    const std::vector<JobEntry> jobs = load_jobs(a.jobs_path);
    SceneSet scenes(jobs);
    const wfb_launch_config cfg = launch_config(a);
    wfb_batch_t b = nullptr;
    check(wfb_batch_create((int)jobs.size(), &cfg, &b), "create batch");
    std::unique_ptr<wfb_batch, int (*)(wfb_batch_t)> guard(b, wfb_batch_destroy);
    double samples = 0.0;
    for (const JobEntry& j : jobs) {
        int id = 0;
        check(wfb_batch_add(b, scenes.by_name.at(j.scene), &j.desc, &id), "add job");
        samples += samples_of(j.desc);
    }
    check(wfb_batch_run(b, 0, nullptr), "run batch");  // warm-up: graph capture, module load
    std::vector<double> runs;
    for (int r = 0; r < a.reps; ++r) {
        wfb_render_stats st{};
        check(wfb_batch_run(b, 0, &st), "run batch");
        runs.push_back(st.render_ms);
    }
    std::string hashes;
    for (size_t k = 0; k < jobs.size(); ++k) {
        const wfb_job_desc& d = jobs[k].desc;
        std::vector<float> rgb((size_t)3 * d.width * d.height);
        check(wfb_batch_download(b, (int)k, rgb.data(), nullptr), "download job");
        hashes += std::string(k ? ", " : "") + "\"" + wf::hex64(wf::fnv1a64(rgb.data(), rgb.size() * sizeof(float))) + "\"";
        if (!a.out_dir.empty()) {
            char name[32];
            std::snprintf(name, sizeof name, "/job_%03zu.pfm", k);
            wf::write_pfm(a.out_dir + name, d.width, d.height, rgb);
        }
    }
    const double median = wf::percentile(runs, 0.5);
    std::printf("{\"mode\": \"batch\", \"arm\": \"%s\", \"jobs\": %zu, \"samples\": %.0f, \"reps\": %d, "
                "\"median_ms\": %.3f, \"msamples_s\": %.2f, \"rgb_fnv1a64\": [%s]}\n",
                a.mode.c_str(), jobs.size(), samples, a.reps, median, median > 0 ? samples / median / 1e3 : 0.0,
                hashes.c_str());
    return 0;
}

int run_serve(const JobArgs& a) {
    using clock = std::chrono::steady_clock;
    const std::vector<JobEntry> jobs = load_jobs(a.jobs_path);
    SceneSet scenes(jobs);
    wfb_server_config sc{};
    sc.one_job_per_launch = a.plain ? 1 : 0;
    sc.launch = launch_config(a);
    wfb_server_t srv = nullptr;
    check(wfb_server_create(&sc, &srv), "create server");
    std::unique_ptr<wfb_server, int (*)(wfb_server_t)> guard(srv, wfb_server_destroy);
    // warm-up: the smallest job (graph capture, module load), then the statistics start afresh
    size_t small = 0;
    for (size_t k = 1; k < jobs.size(); ++k)
        if (samples_of(jobs[k].desc) < samples_of(jobs[small].desc)) small = k;
    uint64_t t = 0;
    check(wfb_server_submit(srv, scenes.by_name.at(jobs[small].scene), &jobs[small].desc, &t), "submit");
    check(wfb_server_wait(srv, t, 600000), "wait");
    check(wfb_server_result(srv, t, nullptr, nullptr, nullptr), "result");
    check(wfb_server_reset_stats(srv), "reset stats");
    // open-loop Poisson arrivals
    std::mt19937_64 rng(a.seed);
    std::exponential_distribution<double> gap(a.lambda);
    std::uniform_int_distribution<size_t> pick(0, jobs.size() - 1);
    std::vector<uint64_t> tickets;
    const auto t0 = clock::now();
    double t_next = 0.0;
    for (;;) {
        t_next += gap(rng);
        if (t_next > a.duration) break;
        std::this_thread::sleep_until(t0 + std::chrono::duration_cast<clock::duration>(std::chrono::duration<double>(t_next)));
        const JobEntry& j = jobs[pick(rng)];
        check(wfb_server_submit(srv, scenes.by_name.at(j.scene), &j.desc, &t), "submit");
        tickets.push_back(t);
    }
    const auto deadline = clock::now() + std::chrono::duration_cast<clock::duration>(std::chrono::duration<double>(a.drain));
    size_t completed = 0;
    for (uint64_t tk : tickets) {
        const auto left = std::chrono::duration_cast<std::chrono::milliseconds>(deadline - clock::now()).count();
        if (wfb_server_wait(srv, tk, (int)std::max<long long>(0, left)) == WFB_OK) {
            check(wfb_server_result(srv, tk, nullptr, nullptr, nullptr), "result");
            ++completed;
        }
    }
    wfb_server_stats st{};
    check(wfb_server_stats_get(srv, &st), "server stats");
    std::printf("{\"mode\": \"serve\", \"policy\": \"%s\", \"arm\": \"%s\", \"lambda\": %g, \"duration_s\": %g, "
                "\"submitted\": %zu, \"completed\": %zu, \"incomplete\": %zu, \"p50_ms\": %.2f, \"p95_ms\": %.2f, "
                "\"p99_ms\": %.2f, \"mean_ms\": %.2f, \"msamples_s\": %.2f, \"launches\": %llu}\n",
                a.plain ? "one-job-per-launch" : "continuous-batching", a.mode.c_str(), a.lambda, a.duration,
                tickets.size(), completed, tickets.size() - completed, st.p50_ms, st.p95_ms, st.p99_ms, st.mean_ms,
                st.wall_s > 0 ? (double)st.samples_done / st.wall_s / 1e6 : 0.0, (unsigned long long)st.launches);
    return 0;
}

}  // namespace

int main(int argc, const char* argv[]) {
    const bool jobs_cmd = argc >= 2 && (std::string(argv[1]) == "batch" || std::string(argv[1]) == "serve");
    try {
        if (jobs_cmd) {
            const JobArgs a = parse_job_args(argc, argv);
            return std::string(argv[1]) == "batch" ? run_batch(a) : run_serve(a);
        }
        return run(wf::parse_args(argc, argv));
    } catch (const wf::ConfigError& e) {
        std::cerr << "Error: " << e.what() << "\n" << (jobs_cmd ? kJobsUsage : wf::usage());
        return 1;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 1;
    }
}
