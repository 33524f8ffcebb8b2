// extern "C" boundary (include/wfb200.h): status codes instead of exceptions, opaque handles.
#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include "engine.hpp"
#include "autotune.hpp"
#include "noalloc.hpp"
#include "queues.hpp"
#include "server.hpp"
#include "wavefront.hpp"
#include "scene_gen.hpp"
#include "../../include/wfb200.h"

struct wfb_scene {
    wf::Scene host;
    std::shared_ptr<wfb::ResidentScene> resident;  // uploaded on first use
    std::mutex mu;
    std::shared_ptr<wfb::ResidentScene> get_resident() {
        std::lock_guard<std::mutex> lock(mu);
        if (!resident) resident = wfb::upload_scene(host);
        return resident;
    }
};

struct wfb_renderer {
    std::unique_ptr<wfb::Renderer> r;
};

struct wfb_scan_workspace {
    std::unique_ptr<wfb::ScanWorkspace> ws;
};

struct wfb_batch {
    std::unique_ptr<wfb::BatchRenderer> b;
    std::vector<std::shared_ptr<wfb::ResidentScene>> scenes;  // keeps job scenes resident
};

struct wfb_server {
    std::unique_ptr<wfb::Server> s;
};

namespace {
wfb::JobSpec job_spec(wfb_scene_t scene, const wfb_job_desc* d) {
    wfb::JobSpec j;
    j.scene = scene->get_resident();
    j.camera.position = wf::Vec3{d->cam_position[0], d->cam_position[1], d->cam_position[2]};
    j.camera.look_at = wf::Vec3{d->cam_look_at[0], d->cam_look_at[1], d->cam_look_at[2]};
    j.camera.up = wf::Vec3{d->cam_up[0], d->cam_up[1], d->cam_up[2]};
    j.camera.vfov_deg = d->cam_vfov_deg;
    j.width = d->width;
    j.height = d->height;
    j.first_sample = 0;
    j.sample_count = d->spp;
    j.seed = d->seed;
    j.max_depth = d->max_depth;
    return j;
}
}  // namespace

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

template <class F>
int guarded(F&& f) {
    try {
        g_last_error.clear();
        f();
        return WFB_OK;
    } catch (const wfb::Error& e) {
        return fail(e.status, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(WFB_ERR_INVALID_ARGUMENT, e.what());
    } catch (const std::bad_alloc&) {
        return fail(WFB_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(WFB_ERR_INVALID_ARGUMENT, e.what());
    } catch (...) {
        return fail(WFB_ERR_INTERNAL, "unknown exception");
    }
}

wfb::PassParams pass_params(const wfb_render_params* p, int first, int count) {
    wfb::PassParams q;
    q.first_sample = first;
    q.sample_count = count;
    q.seed = p->seed;
    q.max_depth = p->max_depth;
    q.count_rays = p->count_rays != 0;
    q.stage_timing = p->stage_timing != 0;
    q.queue_capacity = p->queue_capacity;
    return q;
}

void to_c_stats(const wf::RenderStats& s, wfb_render_stats* out) {
    out->render_ms = s.render_ms;
    out->total_ms = s.total_ms;
    out->extension_rays = s.extension_rays;
    out->shadow_rays = s.shadow_rays;
    for (int i = 0; i < 5; ++i) out->queue_high_water[i] = s.queue_high_water[i];
    out->queue_overflows = s.queue_overflows;
    out->invalid_hits = s.invalid_hits;
    out->peak_vram_bytes = s.peak_vram_bytes;
    const double st[8] = {s.stages.extend, s.stages.classify, s.stages.shade_lambert, s.stages.shade_metal,
                          s.stages.shade_dielectric, s.stages.shadow, s.stages.compact, s.stages.other};
    for (int i = 0; i < 8; ++i) out->stage_ms[i] = st[i];
    out->node_visits = 0;
    out->prim_tests = 0;
    out->kernel_launches = 0;
    out->kernel_ms = 0.0;
}

void need(bool ok, const char* msg) {
    if (!ok) throw wfb::Error(WFB_ERR_INVALID_ARGUMENT, msg);
}

// Register-cap occupancy targets compiled for block 128 (CTAs per SM).
bool occupancy_target(int occ) { return occ == 6 || occ == 8 || occ == 10; }

// wfb_launch_config -> LaunchConfig; NULL or values <= 0 (occupancy < 0) keep the defaults.
wfb::LaunchConfig launch_config(const wfb_launch_config* c) {
    wfb::LaunchConfig l;
    if (c == nullptr) return l;
    need(c->mode == WFB_MODE_MEGAKERNEL || c->mode == WFB_MODE_WAVEFRONT, "mode must be megakernel or wavefront");
    l.mode = c->mode == WFB_MODE_WAVEFRONT ? wf::GpuMode::Wavefront : wf::GpuMode::Megakernel;
    l.use_graph = c->use_graph != 0;
    if (c->block > 0) l.mk.block = c->block;
    need(l.mk.block == 64 || l.mk.block == 128 || l.mk.block == 256, "block must be 64, 128 or 256");
    if (c->occupancy >= 0) l.mk.occupancy = l.wf.occupancy = c->occupancy;
    else if (l.mk.block != 128) l.mk.occupancy = 0;  // the register-cap targets exist for block 128 only
    need(l.mk.occupancy == 0 || (occupancy_target(l.mk.occupancy) && l.mk.block == 128),
         "occupancy target must be 0, 6, 8 or 10 (block 128)");
    need(c->min_active <= 32 && c->leaf_batch <= 32, "min_active and leaf_batch must be in 1..32");
    if (c->min_active > 0) l.mk.min_active = l.wf.min_active = c->min_active;
    if (c->leaf_batch > 0) l.mk.leaf_batch = l.wf.leaf_batch = c->leaf_batch;
    if (c->paths_in_flight > 0) l.wf.paths_in_flight = c->paths_in_flight;
    if (c->split_chunks > 0) l.mk.split_chunks = c->split_chunks;
    return l;
}

}  // namespace

extern "C" {

int wfb_abi_version(void) { return WFB_ABI_VERSION; }

const char* wfb_last_error(void) { return g_last_error.c_str(); }

int wfb_device_name(char* buf, int len) {
    return guarded([&] {
        need(buf && len > 0, "null buffer");
        int dev = 0;
        wfb::cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cudaDeviceProp prop;
        wfb::cuda_check(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
        std::strncpy(buf, prop.name, (size_t)len - 1);
        buf[len - 1] = '\0';
    });
}

int wfb_device_facts_get(wfb_device_facts* out) {
    return guarded([&] {
        need(out != nullptr, "null argument");
        int dev = 0;
        wfb::cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cudaDeviceProp prop;
        wfb::cuda_check(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
        size_t free_b = 0, total_b = 0;
        wfb::cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        std::memset(out, 0, sizeof(*out));
        std::memcpy(out->name, prop.name, std::min(sizeof(out->name) - 1, std::strlen(prop.name)));
        cudaDriverGetVersion(&out->driver_version);
        cudaRuntimeGetVersion(&out->runtime_version);
        out->cc_major = prop.major;
        out->cc_minor = prop.minor;
        out->sm_count = prop.multiProcessorCount;
        out->total_memory_bytes = total_b;
        out->free_memory_bytes = free_b;
        out->l2_bytes = (uint64_t)prop.l2CacheSize;
        out->persisting_l2_max_bytes = (uint64_t)prop.persistingL2CacheMaxSize;
        out->access_window_max_bytes = (uint64_t)prop.accessPolicyMaxWindowSize;
        out->wavefront_l2_resident_paths = (int)wfb::wavefront_l2_resident_paths(dev);
        out->wavefront_slot_bytes = (int)wfb::wavefront_slot_bytes();
        size_t set_aside = 0;
        wfb::cuda_check(cudaDeviceGetLimit(&set_aside, cudaLimitPersistingL2CacheSize), "persisting L2 set-aside");
        out->persisting_l2_set_aside_bytes = set_aside;
    });
}

int wfb_scene_create(const wfb_scene_desc* d, int finalize_bins, wfb_scene_t* out) {
    return guarded([&] {
        need(d && out, "null argument");
        need(d->n_spheres >= 0 && d->n_vertices >= 0 && d->n_triangles >= 0 && d->n_materials >= 0 &&
                 d->n_nodes >= 0 && d->n_prim_order >= 0 && d->n_lights >= 0,
             "negative array size");
        auto s = std::make_unique<wfb_scene>();
        wf::Scene& h = s->host;
        auto copy = [](auto& vec, const void* src, int n) {  // one pass: no zero-fill before the copy
            using T = typename std::decay_t<decltype(vec)>::value_type;
            const T* p = static_cast<const T*>(src);
            if (n) vec.assign(p, p + n);
            else vec.clear();
        };
        need((d->n_spheres == 0 || d->spheres) && (d->n_vertices == 0 || d->vertices) &&
                 (d->n_triangles == 0 || d->triangles) && (d->n_materials == 0 || d->materials) &&
                 (d->n_nodes == 0 || d->nodes) && (d->n_prim_order == 0 || d->prim_order) &&
                 (d->n_lights == 0 || d->lights),
             "null array with a nonzero size");
        copy(h.spheres, d->spheres, d->n_spheres);
        copy(h.vertices, d->vertices, d->n_vertices);
        copy(h.triangles, d->triangles, d->n_triangles);
        copy(h.materials, d->materials, d->n_materials);
        copy(h.nodes, d->nodes, d->n_nodes);
        copy(h.prim_order, d->prim_order, d->n_prim_order);
        copy(h.lights, d->lights, d->n_lights);
        h.env = wf::Vec3{d->env[0], d->env[1], d->env[2]};
        h.camera.position = wf::Vec3{d->cam_position[0], d->cam_position[1], d->cam_position[2]};
        h.camera.look_at = wf::Vec3{d->cam_look_at[0], d->cam_look_at[1], d->cam_look_at[2]};
        h.camera.up = wf::Vec3{d->cam_up[0], d->cam_up[1], d->cam_up[2]};
        h.camera.vfov_deg = d->cam_vfov_deg;
        need(d->width > 0 && d->height > 0, "resolution must be positive");
        h.width = d->width;
        h.height = d->height;
        if (finalize_bins > 0) wf::finalize_scene_bins(h, finalize_bins);
        *out = s.release();
    });
}

int wfb_scene_generate(const char* name, int width, int height, uint32_t seed, int sah_bins,
                       wfb_scene_t* out) {
    return guarded([&] {
        need(name && out, "null argument");
        auto s = std::make_unique<wfb_scene>();
        s->host = wfb::make_config_scene(name, width, height, seed, sah_bins > 0 ? sah_bins : 16);
        *out = s.release();
    });
}

int wfb_scene_info_get(wfb_scene_t s, wfb_scene_info* info) {
    return guarded([&] {
        need(s && info, "null argument");
        const wf::Scene& h = s->host;
        info->n_spheres = (int)h.spheres.size();
        info->n_vertices = (int)h.vertices.size();
        info->n_triangles = (int)h.triangles.size();
        info->n_materials = (int)h.materials.size();
        info->n_nodes = (int)h.nodes.size();
        info->n_prim_order = (int)h.prim_order.size();
        info->n_lights = (int)h.lights.size();
        info->width = h.width;
        info->height = h.height;
        const float env[3] = {h.env.x, h.env.y, h.env.z};
        std::memcpy(info->env, env, sizeof(env));
        const float pos[3] = {h.camera.position.x, h.camera.position.y, h.camera.position.z};
        const float at[3] = {h.camera.look_at.x, h.camera.look_at.y, h.camera.look_at.z};
        const float up[3] = {h.camera.up.x, h.camera.up.y, h.camera.up.z};
        std::memcpy(info->cam_position, pos, sizeof(pos));
        std::memcpy(info->cam_look_at, at, sizeof(at));
        std::memcpy(info->cam_up, up, sizeof(up));
        info->cam_vfov_deg = h.camera.vfov_deg;
    });
}

int wfb_test_traverse(wfb_scene_t s, const void* rays, int n, int anyhit, int speculate, int box_steps,
                      int leaf_batch, void* hits) {
    return guarded([&] {
        need(s && (n == 0 || (rays && hits)), "null argument");
        wfb::traverse_check(s->host, static_cast<const float*>(rays), n, anyhit != 0, speculate != 0, box_steps,
                            leaf_batch, static_cast<float*>(hits));
    });
}

int wfb_test_traverse_wide(wfb_scene_t s, const void* rays, int n, int anyhit, void* hits, int64_t* counts) {
    return guarded([&] {
        need(s && counts && (n == 0 || (rays && hits)), "null argument");
        long long c[4] = {0, 0, 0, 0};
        wfb::traverse_wide_check(s->host, static_cast<const float*>(rays), n, anyhit != 0, static_cast<float*>(hits), c);
        for (int k = 0; k < 4; ++k) counts[k] = (int64_t)c[k];
    });
}

int wfb_scene_boxes_nested(wfb_scene_t s, int* nested) {
    return guarded([&] {
        need(s && nested, "null argument");
        *nested = wfb::check_boxes_nested(s->host.nodes);
    });
}

int wfb_scene_export(wfb_scene_t s, void* spheres, float* vertices, int* triangles, void* materials,
                     void* nodes, int* prim_order, void* lights) {
    return guarded([&] {
        need(s != nullptr, "null scene");
        const wf::Scene& h = s->host;
        auto put = [](void* dst, const auto& vec) {
            if (dst && !vec.empty()) std::memcpy(dst, vec.data(), sizeof(vec[0]) * vec.size());
        };
        put(spheres, h.spheres);
        put(vertices, h.vertices);
        put(triangles, h.triangles);
        put(materials, h.materials);
        put(nodes, h.nodes);
        put(prim_order, h.prim_order);
        put(lights, h.lights);
    });
}

uint64_t wfb_scene_hash(wfb_scene_t s) { return s ? wf::scene_hash(s->host) : 0; }

int wfb_scene_rebuild_bvh(wfb_scene_t s, int bins, int max_leaf, float traversal_cost, int threads) {
    return guarded([&] {
        need(s != nullptr, "null scene");
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->resident) throw wfb::Error(WFB_ERR_INVALID_ARGUMENT, "scene is already uploaded; rebuild before use");
        wf::build_bvh_options(s->host, bins, max_leaf, traversal_cost, threads);
    });
}

int wfb_scene_validate_bvh(wfb_scene_t s, char* msg, int len) {
    return guarded([&] {
        need(s && msg && len > 0, "null argument");
        const std::string m = wf::validate_bvh(s->host);
        std::strncpy(msg, m.c_str(), (size_t)len - 1);
        msg[len - 1] = '\0';
    });
}

int wfb_scene_destroy(wfb_scene_t s) {
    delete s;
    return WFB_OK;
}

uint64_t wfb_scene_device_bytes(wfb_scene_t s) {
    if (!s) return 0;
    std::lock_guard<std::mutex> lock(s->mu);
    return s->resident ? s->resident->bytes : 0;
}

int wfb_renderer_create(wfb_scene_t s, int mode, wfb_renderer_t* out) {
    return guarded([&] {
        need(s && out, "null argument");
        need(mode == WFB_MODE_MEGAKERNEL || mode == WFB_MODE_WAVEFRONT, "unknown mode");
        if (s->host.nodes.empty()) throw wfb::Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
        auto r = std::make_unique<wfb_renderer>();
        r->r = std::make_unique<wfb::Renderer>(s->get_resident(),
                                               mode == WFB_MODE_WAVEFRONT ? wf::GpuMode::Wavefront : wf::GpuMode::Megakernel);
        *out = r.release();
    });
}

int wfb_renderer_set_camera(wfb_renderer_t r, const float position[3], const float look_at[3],
                            const float up[3], float vfov_deg, int width, int height) {
    return guarded([&] {
        need(r && position && look_at && up, "null argument");
        wf::Camera c;
        c.position = wf::Vec3{position[0], position[1], position[2]};
        c.look_at = wf::Vec3{look_at[0], look_at[1], look_at[2]};
        c.up = wf::Vec3{up[0], up[1], up[2]};
        c.vfov_deg = vfov_deg;
        r->r->set_camera(c, width, height);
    });
}

int wfb_renderer_reset(wfb_renderer_t r) {
    return guarded([&] {
        need(r != nullptr, "null renderer");
        r->r->reset();
    });
}

int wfb_renderer_run_passes(wfb_renderer_t r, int first_sample, int count, const wfb_render_params* p,
                            wfb_render_stats* stats) {
    return guarded([&] {
        need(r && p, "null argument");
        wf::RenderStats st{};
        r->r->run_passes(pass_params(p, first_sample, count), &st);
        if (stats) {
            to_c_stats(st, stats);
            stats->node_visits = r->r->last_node_visits();
            stats->prim_tests = r->r->last_prim_tests();
            stats->kernel_launches = (uint64_t)r->r->last_kernel_launches();
            stats->kernel_ms = r->r->last_kernel_ms();
        }
    });
}

int wfb_renderer_download(wfb_renderer_t r, int spp_done, float* rgb, float* lum_var) {
    return guarded([&] {
        need(r != nullptr, "null renderer");
        r->r->download(spp_done, rgb, lum_var);
    });
}

int wfb_renderer_download_mean(wfb_renderer_t r, int spp_done, float* rgb) {
    return guarded([&] {
        need(r && rgb, "null argument");
        r->r->download_mean(spp_done, rgb);
    });
}

int wfb_renderer_download_sums(wfb_renderer_t r, float* rgb_sum, float* lum_sum, float* lum2_sum) {
    return guarded([&] {
        need(r != nullptr, "null renderer");
        r->r->download_sums(rgb_sum, lum_sum, lum2_sum);
    });
}

int wfb_renderer_render(wfb_renderer_t r, const wfb_render_params* p, wfb_render_stats* stats, float* rgb,
                        float* lum_var) {
    return guarded([&] {
        need(r && p, "null argument");
        need(p->spp > 0, "spp must be positive");
        r->r->reset();
        wf::RenderStats st{};
        r->r->run_passes(pass_params(p, 0, p->spp), &st);
        r->r->download(p->spp, rgb, lum_var);
        if (stats) {
            to_c_stats(st, stats);
            stats->node_visits = r->r->last_node_visits();
            stats->prim_tests = r->r->last_prim_tests();
            stats->kernel_launches = (uint64_t)r->r->last_kernel_launches();
            stats->kernel_ms = r->r->last_kernel_ms();
        }
    });
}

uint64_t wfb_renderer_device_bytes(wfb_renderer_t r) { return r ? r->r->device_bytes() : 0; }

int wfb_renderer_configure(wfb_renderer_t r, int block, int blocks_per_sm, int min_active, int split_chunks,
                           int paths_in_flight, int occupancy, int leaf_batch) {
    return guarded([&] {
        need(r != nullptr, "null renderer");
        need(block <= 0 || block == 64 || block == 128 || block == 256, "block must be 64, 128 or 256");
        need(min_active <= 32, "min_active must be in 1..32");
        need(occupancy < 0 || occupancy == 0 || (occupancy_target(occupancy) && (block <= 0 || block == 128)),
             "occupancy target must be 0, 6, 8 or 10 (block 128)");
        need(leaf_batch <= 32, "leaf_batch must be in 1..32");
        r->r->configure(block, blocks_per_sm, min_active, split_chunks, paths_in_flight, occupancy, leaf_batch);
    });
}
int wfb_renderer_set_l2_residency(wfb_renderer_t r, int mode) {
    return guarded([&] {
        need(r != nullptr, "null renderer");
        need(mode >= -1 && mode <= 1, "L2 residency mode must be -1, 0 or 1");
        r->r->set_l2_residency(mode);
    });
}

int wfb_renderer_set_speculation(wfb_renderer_t r, int on) {
    return guarded([&] {
        need(r != nullptr, "null renderer");
        r->r->set_speculation(on != 0);
    });
}

uint64_t wfb_renderer_l2_window_bytes(wfb_renderer_t r) { return r ? r->r->l2_window_bytes() : 0; }

int wfb_renderer_width(wfb_renderer_t r) { return r ? r->r->width() : 0; }
int wfb_renderer_height(wfb_renderer_t r) { return r ? r->r->height() : 0; }

int wfb_renderer_destroy(wfb_renderer_t r) {
    delete r;
    return WFB_OK;
}

int wfb_autotune(wfb_scene_t scene, int width, int height, int probe_spp, int max_depth, int try_wavefront,
                 wfb_tune_result* out) {
    return guarded([&] {
        need(scene && out, "null argument");
        if (scene->host.nodes.empty()) throw wfb::Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
        const wfb::TuneResult t = wfb::autotune(scene->get_resident(), scene->host.camera, width, height, probe_spp,
                                                max_depth, try_wavefront != 0);
        out->mode = t.mode;
        out->block = t.block;
        out->occupancy = t.occupancy;
        out->min_active = t.min_active;
        out->leaf_batch = t.leaf_batch;
        out->paths_in_flight = t.paths_in_flight;
        out->wf_min_active = t.wf_min_active;
        out->wf_occupancy = t.wf_occupancy;
        out->msamples_s = t.msamples_s;
        out->megakernel_msamples_s = t.megakernel_msamples_s;
        out->wavefront_msamples_s = t.wavefront_msamples_s;
        out->candidates = t.candidates;
    });
}

int wfb_renderer_apply_tuning(wfb_renderer_t r, const wfb_tune_result* t) {
    return guarded([&] {
        need(r && t, "null argument");
        wfb::TuneResult tr;
        tr.mode = t->mode;
        tr.block = t->block;
        tr.occupancy = t->occupancy;
        tr.min_active = t->min_active;
        tr.leaf_batch = t->leaf_batch;
        tr.paths_in_flight = t->paths_in_flight;
        tr.wf_min_active = t->wf_min_active;
        tr.wf_occupancy = t->wf_occupancy;
        wfb::apply_tuning(*r->r, tr);
    });
}

int wfb_batch_create(int max_jobs, const wfb_launch_config* cfg, wfb_batch_t* out) {
    return guarded([&] {
        need(out != nullptr, "null argument");
        auto b = std::make_unique<wfb_batch>();
        b->b = std::make_unique<wfb::BatchRenderer>(max_jobs, launch_config(cfg));
        *out = b.release();
    });
}

int wfb_batch_add(wfb_batch_t b, wfb_scene_t scene, const wfb_job_desc* job, int* job_id) {
    return guarded([&] {
        need(b && scene && job, "null argument");
        if (scene->host.nodes.empty()) throw wfb::Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
        wfb::JobSpec j = job_spec(scene, job);
        const int id = b->b->add(j);
        b->scenes.push_back(j.scene);
        if (job_id) *job_id = id;
    });
}

int wfb_batch_clear(wfb_batch_t b) {
    return guarded([&] {
        need(b != nullptr, "null batch");
        b->b->clear();
        b->scenes.clear();
    });
}

int wfb_batch_run(wfb_batch_t b, int count_rays, wfb_render_stats* stats) {
    return guarded([&] {
        need(b != nullptr, "null batch");
        wf::RenderStats st{};
        b->b->run(count_rays != 0, &st);
        if (stats) {
            to_c_stats(st, stats);
            stats->kernel_launches = (uint64_t)b->b->launcher().last_launches();
        }
    });
}

int wfb_batch_download(wfb_batch_t b, int job_id, float* rgb, float* lum_var) {
    return guarded([&] {
        need(b != nullptr, "null batch");
        b->b->download(job_id, b->b->job(job_id).sample_count, rgb, lum_var);
    });
}

int wfb_batch_download_sums(wfb_batch_t b, int job_id, float* rgb_sum, float* lum_sum, float* lum2_sum) {
    return guarded([&] {
        need(b != nullptr, "null batch");
        b->b->download_sums(job_id, rgb_sum, lum_sum, lum2_sum);
    });
}

int wfb_batch_destroy(wfb_batch_t b) {
    delete b;
    return WFB_OK;
}

int wfb_server_create(const wfb_server_config* c, wfb_server_t* out) {
    return guarded([&] {
        need(c && out, "null argument");
        wfb::ServerConfig cfg;
        if (c->budget_bytes > 0) cfg.budget_bytes = c->budget_bytes;
        if (c->max_jobs > 0) cfg.max_jobs = c->max_jobs;
        if (c->launch_target_ms > 0) cfg.launch_target_ms = c->launch_target_ms;
        cfg.fixed_slice = c->fixed_slice;
        cfg.one_job_per_launch = c->one_job_per_launch != 0;
        need(c->schedule == WFB_SCHEDULE_EXPRESS || c->schedule == WFB_SCHEDULE_SHARED, "unknown schedule");
        cfg.schedule = c->schedule == WFB_SCHEDULE_SHARED ? wfb::kScheduleShared : wfb::kScheduleExpress;
        cfg.launch = launch_config(&c->launch);
        if (c->launch.split_chunks <= 0) cfg.launch.mk.split_chunks = wfb::kServerSplitChunks;
        auto s = std::make_unique<wfb_server>();
        s->s = std::make_unique<wfb::Server>(cfg);
        *out = s.release();
    });
}

int wfb_server_submit(wfb_server_t s, wfb_scene_t scene, const wfb_job_desc* job, uint64_t* ticket) {
    return guarded([&] {
        need(s && scene && job && ticket, "null argument");
        if (scene->host.nodes.empty()) throw wfb::Error(WFB_ERR_NOT_FINALIZED, "Scene not finalized (no BVH nodes)");
        *ticket = s->s->submit(job_spec(scene, job));
    });
}

int wfb_server_poll(wfb_server_t s, uint64_t ticket, int* state) {
    return guarded([&] {
        need(s && state, "null argument");
        *state = s->s->state(ticket);
    });
}

int wfb_server_wait(wfb_server_t s, uint64_t ticket, int timeout_ms) {
    return guarded([&] {
        need(s != nullptr, "null server");
        if (!s->s->wait(ticket, timeout_ms)) throw wfb::Error(WFB_ERR_TIMEOUT, "job not finished before the timeout");
    });
}

int wfb_server_result(wfb_server_t s, uint64_t ticket, float* rgb, float* lum_var, double* latency_ms) {
    return guarded([&] {
        need(s != nullptr, "null server");
        s->s->result(ticket, rgb, lum_var, latency_ms);
    });
}

int wfb_server_cancel(wfb_server_t s, uint64_t ticket) {
    return guarded([&] {
        need(s != nullptr, "null server");
        if (!s->s->cancel(ticket)) throw wfb::Error(WFB_ERR_INVALID_ARGUMENT, "job is finished or unknown");
    });
}

int wfb_server_stats_get(wfb_server_t s, wfb_server_stats* out) {
    return guarded([&] {
        need(s && out, "null argument");
        const wfb::ServerStats st = s->s->stats();
        out->submitted = st.submitted;
        out->completed = st.completed;
        out->cancelled = st.cancelled;
        out->failed = st.failed;
        out->launches = st.launches;
        out->samples_done = st.samples_done;
        out->busy_ms = st.busy_ms;
        out->wall_s = st.wall_s;
        out->p50_ms = st.p50_ms;
        out->p95_ms = st.p95_ms;
        out->p99_ms = st.p99_ms;
        out->mean_ms = st.mean_ms;
        out->max_ms = st.max_ms;
        out->bytes_in_use = st.bytes_in_use;
        out->peak_bytes = st.peak_bytes;
        out->queued = st.queued;
        out->active = st.active;
    });
}

int wfb_server_reset_stats(wfb_server_t s) {
    return guarded([&] {
        need(s != nullptr, "null server");
        s->s->reset_stats();
    });
}

int wfb_server_destroy(wfb_server_t s) {
    delete s;
    return WFB_OK;
}

int wfb_scan_workspace_create(int capacity, wfb_scan_workspace_t* out) {
    return guarded([&] {
        need(out != nullptr, "null argument");
        auto w = std::make_unique<wfb_scan_workspace>();
        w->ws = wfb::scan_workspace_create(capacity);
        *out = w.release();
    });
}

int wfb_scan_workspace_destroy(wfb_scan_workspace_t ws) {
    delete ws;
    return WFB_OK;
}

int wfb_scan_exclusive_u32(const uint32_t* d_in, uint32_t* d_out, int n, uint32_t* d_total, wfb_scan_workspace_t ws,
                           void* stream) {
    return guarded([&] {
        need(ws != nullptr, "null workspace");
        need(n == 0 || (d_in && d_out), "null buffer");
        wfb::scan_exclusive_u32(d_in, d_out, n, d_total, *ws->ws, static_cast<cudaStream_t>(stream));
    });
}

int wfb_compact_u32(const uint32_t* d_values, const uint32_t* d_flags, uint32_t* d_out, uint32_t* d_count,
                    uint32_t* d_scratch, int n, wfb_scan_workspace_t ws, void* stream) {
    (void)d_scratch;
    return guarded([&] {
        need(ws != nullptr, "null workspace");
        need(n == 0 || (d_values && d_flags && d_out), "null buffer");
        wfb::compact_u32(d_values, d_flags, d_out, d_count, n, *ws->ws, static_cast<cudaStream_t>(stream));
    });
}

int wfb_test_queue_push(const uint32_t* d_flags, int n, uint32_t* d_items, uint32_t capacity, uint32_t* d_counter,
                        uint32_t* d_overflow, void* stream) {
    return guarded([&] {
        need(n == 0 || (d_flags && d_counter && d_overflow && (capacity == 0 || d_items)), "null buffer");
        wfb::test_queue_push(d_flags, n, d_items, capacity, d_counter, d_overflow, static_cast<cudaStream_t>(stream));
    });
}

int wfb_scan_workspace_check(wfb_scan_workspace_t ws, void* stream) {
    return guarded([&] {
        need(ws != nullptr, "null workspace");
        if (wfb::scan_workspace_failed(*ws->ws, static_cast<cudaStream_t>(stream)))
            throw wfb::Error(WFB_ERR_DEVICE_WAIT, "a scan look-back wait gave up");
    });
}

int wfb_test_bounded_wait(uint64_t limit_ns, int unsatisfiable) {
    return guarded([&] { wfb::set_device_wait_test(limit_ns, unsatisfiable != 0); });
}

int wfb_render_passes_noalloc(wfb_scene_t s, int first_sample, int count, uint32_t seed, int max_depth,
                              float* rgb_sum, float* lum_sum, float* lum2_sum, void* stream) {
    return guarded([&] {
        need(s != nullptr, "null scene");
        std::shared_ptr<wfb::ResidentScene> rs;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            rs = s->resident;  // never uploads here: uploading allocates
        }
        if (!rs)
            throw wfb::Error(WFB_ERR_INVALID_ARGUMENT,
                             "scene is not resident on the device; create a renderer on it first (that uploads it)");
        wfb::render_passes_noalloc(*rs, first_sample, count, seed, max_depth, rgb_sum, lum_sum, lum2_sum,
                                   static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
