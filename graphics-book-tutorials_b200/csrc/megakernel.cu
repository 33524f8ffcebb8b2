// Persistent megakernel: one lane per path, register-resident state, one launch per render.
//
// Replaces megakernel_kernel / run_megakernel_pass (WVM/src/gpu/megakernel.cu:11-104), which
// launches one thread per pixel per sample and synchronises the host after every sample. Here:
//   * The grid is sized to the number of CTAs that are resident at once (persistent threads).
//   * A lane owns one pixel at a time and traces that pixel's samples in ascending order, adding
//     each finished path to register copies of the pixel's film sums. The per-pixel sum order is
//     therefore the reference's (one film_add per sample, WVM/src/gpu/engine.cuh:25-32) and the
//     film is bit-identical, with one film read and one film write per pixel per render.
//   * Work is handed out by a global counter with warp-aggregated fetches (one atomic per warp
//     per refill), so lanes that finish early take the next pixel instead of idling.
//   * A loop iteration traces ONE ray per lane -- the extension ray or the pending shadow ray of
//     the previous Lambertian bounce -- through the same traversal code, then does the matching
//     shading step. Lanes of a warp therefore stay together in the traversal loop whichever ray
//     kind they hold, and a path that ends regenerates the next sample at once.
//   * Ray counts are kept in registers and folded with one atomic per warp at exit.
// The shadow-ray origin equals the next extension-ray origin (both are p + n * eps after
// shade_lambert), so a pending shadow ray costs only its direction, tmax and contribution.
#include "engine.hpp"
#include "../../include/wfb200.h"

namespace wfb {
namespace {

constexpr unsigned kFull = 0xffffffffu;

struct MkArgs {
    DevScene s;
    DevFilm film;
    DevCounters* counters;
    unsigned int* work;
    int pixels;
    int first_sample;
    int sample_end;
    uint32_t seed;
    int max_depth;
    int count_rays;
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) megakernel_persistent(const MkArgs a) {
    const DevScene& s = a.s;
    const int lane = threadIdx.x & 31;

    int pixel = -1, px = 0, py = 0, sample = 0;
    bool out_of_work = false;
    wf::PathState ps;
    float acc_r = 0.f, acc_g = 0.f, acc_b = 0.f, acc_l = 0.f, acc_l2 = 0.f;
    bool shadow_pending = false, alive_after_shadow = false;
    wf::Vec3 sh_dir{0.f, 0.f, 0.f}, sh_contrib{0.f, 0.f, 0.f};
    float sh_tmax = 0.f;
    unsigned long long n_ext = 0, n_shadow = 0;
    unsigned int n_invalid = 0;

    for (;;) {
        // ---- refill: lanes without a pixel take the next ones (one atomic per warp) ----
        const bool need = pixel < 0 && !out_of_work;
        const unsigned need_mask = __ballot_sync(kFull, need);
        if (need_mask) {
            const int leader = __ffs(need_mask) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(a.work, (unsigned)__popc(need_mask));
            base = __shfl_sync(kFull, base, leader);
            if (need) {
                const unsigned idx = base + __popc(need_mask & ((1u << lane) - 1u));
                if (idx < (unsigned)a.pixels) {
                    pixel = (int)idx;
                    px = pixel % s.width;
                    py = pixel / s.width;
                    sample = a.first_sample;
                    acc_r = a.film.rgb[3 * pixel];
                    acc_g = a.film.rgb[3 * pixel + 1];
                    acc_b = a.film.rgb[3 * pixel + 2];
                    acc_l = a.film.lum[pixel];
                    acc_l2 = a.film.lum2[pixel];
                    ps = wf::init_path(s, px, py, (uint32_t)sample, a.seed);
                    shadow_pending = false;
                } else {
                    out_of_work = true;
                }
            }
        }
        const bool active = pixel >= 0;
        if (__ballot_sync(kFull, active) == 0) break;

        // ---- trace one ray per active lane (extension, or the pending shadow ray) ----
        wf::HitRecord h;
        h.prim = -1;
        if (active) {
            wf::Ray r = ps.ray;
            if (shadow_pending) {
                r.d = sh_dir;
                r.tmin = wf::kRayEps;
                r.tmax = sh_tmax;
            }
            intersect_dev(s, r, &h, shadow_pending);
        }
        if (!active) continue;

        // ---- shading step for the ray just traced ----
        bool path_done = false;
        if (shadow_pending) {
            ++n_shadow;
            if (h.prim < 0) ps.L += sh_contrib;  // unoccluded
            shadow_pending = false;
            path_done = !alive_after_shadow;
        } else {
            ++n_ext;
            if (!hit_is_valid(s, h)) {
                ++n_invalid;
                ps.L += ps.throughput * s.env;  // invalid hit is treated as a miss
                path_done = true;
            } else {
                wf::Surface f;
                const int mat = wf::classify(s, ps, h, a.max_depth, &f);
                if (mat < 0) {
                    path_done = true;
                } else if (mat == wf::kLambert) {
                    wf::Ray sh;
                    wf::Vec3 c;
                    int has = 0;
                    const bool alive = wf::shade_lambert(s, ps, f, &sh, &c, &has);
                    if (has) {
                        shadow_pending = true;
                        alive_after_shadow = alive;
                        sh_dir = sh.d;
                        sh_tmax = sh.tmax;
                        sh_contrib = c;
                    } else {
                        path_done = !alive;
                    }
                } else if (mat == wf::kMetal) {
                    path_done = !wf::shade_metal(s, ps, f);
                } else {
                    path_done = !wf::shade_dielectric(s, ps, f);
                }
            }
        }
        if (!path_done) continue;

        // ---- film_add in registers, then the next sample of this pixel or a new pixel ----
        acc_r += ps.L.x;
        acc_g += ps.L.y;
        acc_b += ps.L.z;
        const float l = wf::luminance(ps.L);
        acc_l += l;
        acc_l2 += l * l;
        ++sample;
        if (sample < a.sample_end) {
            ps = wf::init_path(s, px, py, (uint32_t)sample, a.seed);
        } else {
            a.film.rgb[3 * pixel] = acc_r;
            a.film.rgb[3 * pixel + 1] = acc_g;
            a.film.rgb[3 * pixel + 2] = acc_b;
            a.film.lum[pixel] = acc_l;
            a.film.lum2[pixel] = acc_l2;
            pixel = -1;
        }
    }

    // ---- fold counters: one atomic per warp ----
    for (int off = 16; off > 0; off >>= 1) {
        n_ext += __shfl_down_sync(kFull, n_ext, off);
        n_shadow += __shfl_down_sync(kFull, n_shadow, off);
        n_invalid += __shfl_down_sync(kFull, n_invalid, off);
    }
    if (lane == 0) {
        if (a.count_rays) {
            if (n_ext) atomicAdd(&a.counters->extension_rays, n_ext);
            if (n_shadow) atomicAdd(&a.counters->shadow_rays, n_shadow);
        }
        if (n_invalid) atomicAdd(&a.counters->invalid_hits, n_invalid);
    }
}

template <int BLOCK>
void launch_block(const MkArgs& args, int blocks_per_sm, cudaStream_t stream) {
    int dev = 0, sms = 0, occ = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, megakernel_persistent<BLOCK>, BLOCK, 0),
               "occupancy");
    if (blocks_per_sm > 0 && blocks_per_sm < occ) occ = blocks_per_sm;
    if (occ < 1) occ = 1;
    long long grid = (long long)sms * occ;
    const long long needed = ((long long)args.pixels + BLOCK - 1) / BLOCK;
    if (grid > needed) grid = needed;
    if (grid < 1) grid = 1;
    megakernel_persistent<BLOCK><<<(unsigned)grid, BLOCK, 0, stream>>>(args);
    cuda_check(cudaGetLastError(), "megakernel launch");
}

}  // namespace

void launch_megakernel(const DevScene& s, const DevFilm& film, DevCounters* counters,
                       unsigned int* work_counter, const PassParams& p, const MegakernelConfig& cfg,
                       cudaStream_t stream) {
    if (p.sample_count <= 0 || film.pixels <= 0) return;
    MkArgs args;
    args.s = s;
    args.film = film;
    args.counters = counters;
    args.work = work_counter;
    args.pixels = film.pixels;
    args.first_sample = p.first_sample;
    args.sample_end = p.first_sample + p.sample_count;
    args.seed = p.seed;
    args.max_depth = p.max_depth;
    args.count_rays = p.count_rays ? 1 : 0;
    cuda_check(cudaMemsetAsync(work_counter, 0, sizeof(unsigned int), stream), "memset work counter");
    switch (cfg.block) {
        case 64: launch_block<64>(args, cfg.blocks_per_sm, stream); break;
        case 256: launch_block<256>(args, cfg.blocks_per_sm, stream); break;
        case 128: launch_block<128>(args, cfg.blocks_per_sm, stream); break;
        default: throw Error(WFB_ERR_INVALID_ARGUMENT, "megakernel block size must be 64, 128 or 256");
    }
}

}  // namespace wfb
