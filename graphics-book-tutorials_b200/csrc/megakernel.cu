// Persistent megakernel: one lane per path, register-resident state, one launch per render -- or
// per batch of render jobs.
//
// Replaces megakernel_kernel / run_megakernel_pass (WVM/src/gpu/megakernel.cu:11-104), which
// launches one thread per pixel per sample, traces each path to completion and synchronises the
// host after every sample (lane efficiency 7-12 of 32 in the reference's own profiles). Here:
//
//  * Persistent threads: the grid is the set of CTAs resident at once; work units are handed out
//    by a global counter with warp-aggregated fetches (one atomic per warp per refill).
//  * Jobs: a work unit belongs to one job (scene, camera, resolution, seed, depth, film). A single
//    render is a batch of one job passed in parameter space; a batch of many jobs is a device-side
//    job table whose units are numbered consecutively, so paths of different jobs share one launch
//    and the tail of one job overlaps the others. Per-job pixel ids stay job-local (the RNG key
//    uses py * width + px of the job, WVM/include/wf/path_core.hpp:74), so a job renders the same
//    bits alone and inside any batch.
//  * Resumable traversal: a ray's traversal state is the next node index, a pending leaf and the
//    best hit (box_step / prim_step, dev_scene.cuh). A warp runs rounds of box steps (lanes without
//    a pending leaf test their next node) and rounds of primitive steps (lanes with a pending leaf
//    test its next primitive), choosing a primitive round once `leaf_batch` lanes hold a pending
//    leaf or they outnumber the box lanes, so leaf work is done by many lanes at once instead of
//    by the one or two lanes that reach a leaf in a given box round. It keeps going while at least
//    `min_active` lanes traverse; only then does it shade the lanes whose ray finished and give
//    them their next ray (extension, the pending shadow ray of a Lambertian bounce, or the camera
//    ray of the next sample) -- the "dynamic ray fetch" of Aila and Laine (HPG 2009) with
//    one-lane-per-path shading. A lane holding a pending leaf also takes part in box rounds until
//    it reaches its next leaf (speculation, made exact in box_step), so box rounds stay full while
//    leaves gather for a primitive round.
//  * Film order: a unit is one pixel and a run of its samples in ascending order. Direct mode: a
//    unit covers all samples of the pixel; the lane adds every finished path to register copies of
//    the film sums (film_add order, WVM/src/gpu/engine.cuh:25-32). Split mode (a job with fewer
//    pixels than resident lanes): a pixel's samples are cut into chunks on different lanes; each
//    path's radiance goes to its (pixel, sample) slot of a buffer and film_commit adds the slots
//    in sample order. Both produce bit-identical films.
//  * The shadow ray of a Lambertian bounce starts at the next extension ray's origin
//    (p + n * eps, WVM/include/wf/path_core.hpp:197,210,226); only direction, tmax and
//    contribution are kept.
//  * Ray counters live in registers and are folded with one atomic per warp at exit.
#include <algorithm>
#include <type_traits>
#include "engine.hpp"
#include "../../include/wfb200.h"

namespace wfb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
// Box steps per box round: a lane that can still step after one takes up to this many in a row
// before the warp votes again, so the round's ballots and choice are paid once per several steps
// (B200, 1280x720x64, against one step per round: icospheres +12%, heightfield +14%; 6 and 8 were
// slower than 4 on icospheres). Each lane's steps are the same ones, in the same order.
constexpr int kBoxSteps = 4;
// The same for batch launches (64-job mix: 1 step 1,384 ms, 2 steps 1,263, 4 steps 1,214; on another
// box 4 steps 1,167 against 1,182 at 6).
constexpr int kBatchBoxSteps = 4;

struct MkArgs {
    JobDesc job0;              // single-job launch
    const JobDesc* jobs;       // batch launch: device job table
    const BatchHeader* hdr;    // batch launch: job count and total units (device)
    DevCounters* counters;
    unsigned int* work;
    int count_rays;
    int min_active;
    int leaf_batch;
    int speculate;  // speculative traversal (box_step): 1 on, 0 off
};

template <bool MULTI>
__device__ __forceinline__ const JobDesc& job_at(const MkArgs& a, int j) {
    return MULTI ? a.jobs[j] : a.job0;
}

// MINB > 1 caps registers so that MINB CTAs fit an SM (__launch_bounds__ minimum blocks).
// COUNT adds node-visit and primitive-test counters (used by count_rays runs only).
// SPLIT: every job of the launch is in split mode (chunks > 1), so the per-lane film accumulators
// of direct mode and their branches are compiled out (5 registers fewer under the register cap).
template <int BLOCK, bool MULTI, int MINB, bool COUNT, bool SPLIT>
__global__ void __launch_bounds__(BLOCK, MINB) megakernel_persistent(const MkArgs a) {
    const int lane = threadIdx.x & 31;
    const unsigned total_units = MULTI ? a.hdr->total_units : a.job0.units;
    const int n_jobs = MULTI ? (int)a.hdr->n_jobs : 1;

    // ---- per-lane work and path state ----
    int job = 0;
    int pixel = -1, sample = 0, s_end = 0;
    bool out_of_work = false;
    wf::PathState ps{};
    float acc_r = 0.f, acc_g = 0.f, acc_b = 0.f, acc_l = 0.f, acc_l2 = 0.f;
    bool shadow_ray = false, alive_after_shadow = false;
    wf::Vec3 sh_dir{0.f, 0.f, 0.f}, sh_contrib{0.f, 0.f, 0.f};
    float sh_tmax = 0.f;
    // The state that only shading reads is parked in shared memory while the lane's ray traverses
    // (one word per field per lane, field-major so a warp's words are consecutive), so that the
    // traversal loop keeps only the ray, its origin and the traversal state in registers: 1-3% on
    // one scene, about 1% on the 64-job batch (whose several BVHs share what is left of L1; with one
    // box step per round parking cost batches up to 13%, with kBoxSteps it gains).
    constexpr int kParked = SPLIT ? 22 : 27;
    __shared__ float parked[kParked * BLOCK];
    auto P = [&](int f) -> float& { return parked[f * BLOCK + threadIdx.x]; };
    auto park = [&]() {
        P(0) = ps.throughput.x; P(1) = ps.throughput.y; P(2) = ps.throughput.z;
        P(3) = ps.L.x; P(4) = ps.L.y; P(5) = ps.L.z;
        P(6) = __int_as_float(ps.depth); P(7) = __int_as_float(ps.specular); P(8) = ps.prev_pdf;
        P(9) = __uint_as_float(ps.key.k0); P(10) = __uint_as_float(ps.key.k1);
        P(11) = ps.ray.d.x; P(12) = ps.ray.d.y; P(13) = ps.ray.d.z; P(14) = ps.ray.tmin; P(15) = ps.ray.tmax;
        P(16) = sh_contrib.x; P(17) = sh_contrib.y; P(18) = sh_contrib.z;
        P(19) = __int_as_float(alive_after_shadow ? 1 : 0);
        P(20) = __int_as_float(sample); P(21) = __int_as_float(s_end);
        if (!SPLIT) { P(22) = acc_r; P(23) = acc_g; P(24) = acc_b; P(25) = acc_l; P(26) = acc_l2; }
    };
    auto unpark = [&]() {
        ps.throughput = wf::Vec3{P(0), P(1), P(2)};
        ps.L = wf::Vec3{P(3), P(4), P(5)};
        ps.depth = __float_as_int(P(6)); ps.specular = __float_as_int(P(7)); ps.prev_pdf = P(8);
        ps.key.k0 = __float_as_uint(P(9)); ps.key.k1 = __float_as_uint(P(10));
        ps.ray.d = wf::Vec3{P(11), P(12), P(13)}; ps.ray.tmin = P(14); ps.ray.tmax = P(15);
        sh_contrib = wf::Vec3{P(16), P(17), P(18)};
        alive_after_shadow = __float_as_int(P(19)) != 0;
        sample = __float_as_int(P(20)); s_end = __float_as_int(P(21));
        if (!SPLIT) { acc_r = P(22); acc_g = P(23); acc_b = P(24); acc_l = P(25); acc_l2 = P(26); }
    };
    // ---- traversal state of the lane's current ray. Every ray starts at ps.ray.o (the camera,
    // or p + n * eps for both the next extension ray and the shadow ray) with tmin = kRayEps. ----
    int node = -1;
    int pend = 0;  // pending leaf (box_step / prim_step)
    bool spec = false;  // this ray may take box steps while it holds a pending leaf (box_step)
    TravRay ray;
    wf::HitRecord h;
    h.t = 0.f;
    h.prim = -1;
    h.u = h.v = 0.f;
    // batch launches cache the lane's job BVH; a single job reads it from parameter space
    const float4* jnodes = nullptr;
    const float4* jprims = nullptr;
    int jn_nodes = 0, jn_spheres = 0;
    unsigned n_ext = 0, n_shadow = 0, n_invalid = 0, n_steps = 0, n_prims = 0;

    auto start_ray = [&](int boxes_nested) {
        const int nn = MULTI ? jn_nodes : a.job0.s.n_nodes;
        if (shadow_ray) traversal_begin(nn, sh_dir, sh_tmax, &ray, &node, &h);
        else traversal_begin(nn, ps.ray.d, ps.ray.tmax, &ray, &node, &h);
        pend = 0;
        spec = a.speculate && (shadow_ray || (boxes_nested && finite_inv(ray)));
    };
    auto new_path = [&](const DevScene& s, uint32_t seed) {
        ps = wf::init_path(s, pixel % s.width, pixel / s.width, (uint32_t)sample, seed);
    };

    for (;;) {
        // ================= traversal: rounds of box steps or of primitive steps =================
        for (;;) {
            const bool in_leaf = pend != 0;
            const bool at_box = can_box_step(node, pend, spec);
            const unsigned pmask = __ballot_sync(kFull, in_leaf);
            const unsigned bmask = __ballot_sync(kFull, at_box);
            const unsigned tmask = pmask | bmask;
            if (tmask == 0) break;
            if (__popc(tmask) < a.min_active) {
                // few lanes left traversing: stop if some other lane has shading or refill to do
                const bool waiting = !(in_leaf || at_box) && (pixel >= 0 || !out_of_work);
                if (__ballot_sync(kFull, waiting) != 0) break;
            }
            // primitive round once enough lanes hold a pending leaf (or they outnumber the box lanes)
            const int np = __popc(pmask);
            if (np != 0 && (np >= a.leaf_batch || np >= __popc(bmask))) {
                if (in_leaf) {
                    if (COUNT) ++n_prims;
                    if (MULTI) prim_step(jprims, jn_spheres, ps.ray.o, ray, shadow_ray, node, pend, h);
                    else prim_step(a.job0.s.prims, a.job0.s.n_spheres, ps.ray.o, ray, shadow_ray, node, pend, h);
                }
            } else if (at_box) {
#pragma unroll
                for (int k = 0; k < (MULTI ? kBatchBoxSteps : kBoxSteps); ++k) {
                    if (k == 0 || can_box_step(node, pend, spec)) {
                        if (COUNT) ++n_steps;
                        if (MULTI) box_step(jnodes, jn_nodes, ps.ray.o, ray, h.t, node, pend);
                        else box_step(a.job0.s.nodes, a.job0.s.n_nodes, ps.ray.o, ray, h.t, node, pend);
                    }
                }
            }
        }

        // ================= shading: lanes whose ray has finished =================
        if (node < 0 && pend == 0 && pixel >= 0) {
            unpark();
            const JobDesc& J = job_at<MULTI>(a, job);
            const DevScene& s = J.s;
            bool path_done = false;
            if (shadow_ray) {
                ++n_shadow;
                if (h.prim < 0) ps.L += sh_contrib;  // unoccluded
                shadow_ray = false;
                path_done = !alive_after_shadow;
            } else {
                ++n_ext;
                if (!hit_is_valid(s, h)) {
                    ++n_invalid;
                    ps.L += ps.throughput * s.env;  // an invalid hit is treated as a miss
                    path_done = true;
                } else {
                    wf::Surface f;
                    const int mat = wf::classify(s, ps, h, J.max_depth, &f);
                    if (mat < 0) {
                        path_done = true;
                    } else if (mat == wf::kLambert) {
                        wf::Ray sh;
                        wf::Vec3 c;
                        int has = 0;
                        const bool alive = wf::shade_lambert(s, ps, f, &sh, &c, &has);
                        if (has) {
                            shadow_ray = true;
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
            if (path_done) {
                if (SPLIT || J.chunks > 1) {
                    float* slot = J.lbuf + sample_slot(pixel, sample - J.first_sample, J.film.pixels);
                    slot[0] = ps.L.x;
                    slot[1] = ps.L.y;
                    slot[2] = ps.L.z;
                } else {
                    acc_r += ps.L.x;
                    acc_g += ps.L.y;
                    acc_b += ps.L.z;
                    const float l = wf::luminance(ps.L);
                    acc_l += l;
                    acc_l2 += l * l;
                }
                ++sample;
                if (sample < s_end) {
                    new_path(s, J.seed);
                } else {
                    if (!SPLIT && J.chunks == 1) {
                        J.film.rgb[3 * pixel] = acc_r;
                        J.film.rgb[3 * pixel + 1] = acc_g;
                        J.film.rgb[3 * pixel + 2] = acc_b;
                        J.film.lum[pixel] = acc_l;
                        J.film.lum2[pixel] = acc_l2;
                    }
                    pixel = -1;
                }
            }
            if (pixel >= 0) {
                start_ray(s.boxes_nested);
                park();
            }
        }

        // ================= refill: lanes without a unit take the next ones =================
        const bool need = pixel < 0 && !out_of_work;
        const unsigned need_mask = __ballot_sync(kFull, need);
        if (need_mask) {
            const int leader = __ffs(need_mask) - 1;
            unsigned base = 0;
            // batch: the leader finds the job of the warp's first unit and where the next job
            // starts; a lane searches the table itself only when its unit crosses that boundary
            int j0 = 0;
            unsigned next_begin = 0xffffffffu;
            if (lane == leader) {
                base = atomicAdd(a.work, (unsigned)__popc(need_mask));
                if (MULTI && base < total_units) {
                    j0 = job_of_unit(a.jobs, n_jobs, base);
                    if (j0 + 1 < n_jobs) next_begin = a.jobs[j0 + 1].unit_begin;
                }
            }
            base = __shfl_sync(kFull, base, leader);
            if (MULTI) {
                j0 = __shfl_sync(kFull, j0, leader);
                next_begin = __shfl_sync(kFull, next_begin, leader);
            }
            if (need) {
                const unsigned u = base + __popc(need_mask & ((1u << lane) - 1u));
                if (u < total_units) {
                    if (MULTI) job = u < next_begin ? j0 : job_of_unit(a.jobs, n_jobs, u);
                    const JobDesc& J = job_at<MULTI>(a, job);
                    const DevScene& s = J.s;
                    if (MULTI) {
                        jnodes = s.nodes;
                        jprims = s.prims;
                        jn_nodes = s.n_nodes;
                        jn_spheres = s.n_spheres;
                    }
                    // unit -> pixel (u mod P) and chunk (u div P): neighbouring lanes, neighbouring pixels
                    const unsigned local = u - J.unit_begin;
                    const int pixels = J.film.pixels;
                    pixel = (int)(local % (unsigned)pixels);
                    const int c = (int)(local / (unsigned)pixels);
                    sample = J.first_sample + c * J.chunk;
                    s_end = min(sample + J.chunk, J.first_sample + J.sample_count);
                    if (!SPLIT && J.chunks == 1) {
                        acc_r = J.film.rgb[3 * pixel];
                        acc_g = J.film.rgb[3 * pixel + 1];
                        acc_b = J.film.rgb[3 * pixel + 2];
                        acc_l = J.film.lum[pixel];
                        acc_l2 = J.film.lum2[pixel];
                    }
                    new_path(s, J.seed);
                    shadow_ray = false;
                    start_ray(s.boxes_nested);
                    park();
                } else {
                    out_of_work = true;
                }
            }
        }
        if (__ballot_sync(kFull, pixel >= 0) == 0) break;
    }

    // ---- fold counters: one atomic per warp ----
    unsigned long long ext = n_ext, shd = n_shadow, steps = n_steps, prims = n_prims;
    for (int off = 16; off > 0; off >>= 1) {
        ext += __shfl_down_sync(kFull, ext, off);
        shd += __shfl_down_sync(kFull, shd, off);
        n_invalid += __shfl_down_sync(kFull, n_invalid, off);
        if (COUNT) {
            steps += __shfl_down_sync(kFull, steps, off);
            prims += __shfl_down_sync(kFull, prims, off);
        }
    }
    if (lane == 0) {
        if (a.count_rays) {
            if (ext) atomicAdd(&a.counters->extension_rays, ext);
            if (shd) atomicAdd(&a.counters->shadow_rays, shd);
            if (COUNT) {
                atomicAdd(&a.counters->node_visits, steps);
                atomicAdd(&a.counters->prim_tests, prims);
            }
        }
        if (n_invalid) atomicAdd(&a.counters->invalid_hits, n_invalid);
    }
}

__device__ __forceinline__ void commit_pixel(const DevFilm& film, const float* __restrict__ lbuf, int p, int count) {
    float r = film.rgb[3 * p], g = film.rgb[3 * p + 1], b = film.rgb[3 * p + 2];
    float l1 = film.lum[p], l2 = film.lum2[p];
    for (int k = 0; k < count; ++k) {
        const float* slot = lbuf + sample_slot(p, k, film.pixels);
        const wf::Vec3 L{slot[0], slot[1], slot[2]};
        r += L.x;
        g += L.y;
        b += L.z;
        const float l = wf::luminance(L);
        l1 += l;
        l2 += l * l;
    }
    film.rgb[3 * p] = r;
    film.rgb[3 * p + 1] = g;
    film.rgb[3 * p + 2] = b;
    film.lum[p] = l1;
    film.lum2[p] = l2;
}

// Split mode: film_add of every (pixel, sample) slot in ascending sample order.
__global__ void film_commit(DevFilm film, const float* __restrict__ lbuf, int pixels, int count) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < pixels) commit_pixel(film, lbuf, p, count);
}

// Batch form: blockIdx.y is the job; jobs in direct mode have nothing to commit.
__global__ void film_commit_jobs(const JobDesc* jobs, const BatchHeader* hdr) {
    const int j = blockIdx.y;
    if (j >= (int)hdr->n_jobs) return;
    const JobDesc& J = jobs[j];
    if (J.chunks <= 1) return;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < J.film.pixels; p += gridDim.x * blockDim.x)
        commit_pixel(J.film, J.lbuf, p, J.sample_count);
}

template <int BLOCK, bool MULTI, int MINB, bool COUNT, bool SPLIT>
int resident_ctas(int blocks_per_sm) {
    int dev = 0, sms = 0, occ = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &occ, megakernel_persistent<BLOCK, MULTI, MINB, COUNT, SPLIT>, BLOCK, 0),
               "occupancy");
    if (blocks_per_sm > 0 && blocks_per_sm < occ) occ = blocks_per_sm;
    if (occ < 1) occ = 1;
    return sms * occ;
}

template <int BLOCK, bool MULTI, int MINB, bool COUNT, bool SPLIT>
void launch_block(const MkArgs& args, long long units, int blocks_per_sm, cudaStream_t stream) {
    long long grid = resident_ctas<BLOCK, MULTI, MINB, COUNT, SPLIT>(blocks_per_sm);
    if (units > 0) {
        const long long needed = (units + BLOCK - 1) / BLOCK;
        if (grid > needed) grid = needed;
    }
    if (grid < 1) grid = 1;
    megakernel_persistent<BLOCK, MULTI, MINB, COUNT, SPLIT><<<(unsigned)grid, BLOCK, 0, stream>>>(args);
    cuda_check(cudaGetLastError(), "megakernel launch");
}

// Dispatch over the compiled (block, occupancy) variants.
template <bool MULTI, class F>
auto dispatch(const MegakernelConfig& cfg, F&& f) {
    if (cfg.block == 64) return f(std::integral_constant<int, 64>{}, std::integral_constant<int, 1>{});
    if (cfg.block == 256) return f(std::integral_constant<int, 256>{}, std::integral_constant<int, 1>{});
    if (cfg.block != 128) throw Error(WFB_ERR_INVALID_ARGUMENT, "megakernel block size must be 64, 128 or 256");
    if (cfg.occupancy == 6) return f(std::integral_constant<int, 128>{}, std::integral_constant<int, 6>{});
    if (cfg.occupancy == 8) return f(std::integral_constant<int, 128>{}, std::integral_constant<int, 8>{});
    if (cfg.occupancy == 10) return f(std::integral_constant<int, 128>{}, std::integral_constant<int, 10>{});
    if (cfg.occupancy > 1) throw Error(WFB_ERR_INVALID_ARGUMENT, "megakernel occupancy target must be 0, 6, 8 or 10");
    return f(std::integral_constant<int, 128>{}, std::integral_constant<int, 1>{});
}

// `all_split`: every job of the launch has chunks > 1 (selects the SPLIT variant).
template <bool MULTI>
void launch_any(const MkArgs& args, long long units, const MegakernelConfig& cfg, bool all_split,
                cudaStream_t stream) {
    if (args.count_rays) {  // counting runs use the instrumented 128-thread variant (both modes)
        launch_block<128, MULTI, 1, true, false>(args, units, cfg.blocks_per_sm, stream);
        return;
    }
    dispatch<MULTI>(cfg, [&](auto block, auto minb) {
        constexpr int B = decltype(block)::value, O = decltype(minb)::value;
        if (all_split) launch_block<B, MULTI, O, false, true>(args, units, cfg.blocks_per_sm, stream);
        else launch_block<B, MULTI, O, false, false>(args, units, cfg.blocks_per_sm, stream);
        return 0;
    });
}

}  // namespace

void launch_film_commit(const DevFilm& film, const float* lbuf, int count, cudaStream_t stream) {
    if (film.pixels <= 0 || count <= 0) return;
    film_commit<<<(film.pixels + 255) / 256, 256, 0, stream>>>(film, lbuf, film.pixels, count);
    cuda_check(cudaGetLastError(), "film commit launch");
}

int megakernel_resident_threads(const MegakernelConfig& cfg) {
    return dispatch<false>(cfg, [&](auto block, auto minb) {
        return decltype(block)::value *
               resident_ctas<decltype(block)::value, false, decltype(minb)::value, false, true>(cfg.blocks_per_sm);
    });
}

int megakernel_split_chunks(int pixels, int sample_count, const MegakernelConfig& cfg) {
    if (cfg.split_chunks > 0) return std::min(cfg.split_chunks, std::max(1, sample_count));
    // One sample per unit whenever the per-sample buffer fits: a warp then traces one sample of 32
    // neighbouring pixels (coherent camera rays), every lane takes new work after each path, and
    // the tail is one path long instead of a pixel's whole run of samples. Measured on B200:
    // +61% on icospheres 1280x720x64, +16% on heightfield, over one pixel per unit.
    if (sample_count <= 1 || pixels <= 0) return 1;
    if (split_buffer_bytes(pixels, sample_count) > kSplitBufferBytes) return 1;
    return sample_count;
}

JobDesc make_job(const DevScene& s, const DevFilm& film, float* lbuf, int first_sample, int sample_count, int chunks,
                 uint32_t seed, int max_depth) {
    JobDesc j{};
    j.s = s;
    j.film = film;
    j.lbuf = lbuf;
    j.first_sample = first_sample;
    j.sample_count = sample_count;
    j.chunks = chunks < 1 ? 1 : chunks;
    j.chunk = sample_count > 0 ? (sample_count + j.chunks - 1) / j.chunks : 0;
    j.chunks = j.chunk > 0 ? (sample_count + j.chunk - 1) / j.chunk : 1;  // no empty trailing chunk
    j.seed = seed;
    j.max_depth = max_depth;
    j.unit_begin = 0;
    j.units = sample_count > 0 ? (unsigned)film.pixels * (unsigned)j.chunks : 0u;
    return j;
}

int launch_megakernel(const DevScene& s, const DevFilm& film, DevCounters* counters, unsigned int* work_counter,
                      float* lbuf, const PassParams& p, const MegakernelConfig& cfg, int chunks,
                      cudaStream_t stream, KernelTimer* timer) {
    if (p.sample_count <= 0 || film.pixels <= 0) return 0;
    if (chunks > 1 && lbuf == nullptr) throw Error(WFB_ERR_INTERNAL, "split megakernel needs a sample buffer");
    MkArgs args{};
    args.job0 = make_job(s, film, lbuf, p.first_sample, p.sample_count, chunks, p.seed, p.max_depth);
    args.jobs = nullptr;
    args.hdr = nullptr;
    args.counters = counters;
    args.work = work_counter;
    args.count_rays = p.count_rays ? 1 : 0;
    args.min_active = cfg.min_active;
    args.leaf_batch = cfg.leaf_batch;
    args.speculate = cfg.speculate ? 1 : 0;
    cuda_check(cudaMemsetAsync(work_counter, 0, sizeof(unsigned int), stream), "memset work counter");
    if (timer) timer->begin(stream);
    launch_any<false>(args, args.job0.units, cfg, args.job0.chunks > 1, stream);
    if (timer) timer->end(stream);
    if (args.job0.chunks > 1) {
        launch_film_commit(film, lbuf, p.sample_count, stream);
        return 2;
    }
    return 1;
}

void launch_megakernel_batch(const JobDesc* d_jobs, const BatchHeader* d_hdr, int max_jobs, DevCounters* counters,
                             unsigned int* work_counter, bool count_rays, const MegakernelConfig& cfg,
                             bool all_split, cudaStream_t stream) {
    MkArgs args{};
    args.jobs = d_jobs;
    args.hdr = d_hdr;
    args.counters = counters;
    args.work = work_counter;
    args.count_rays = count_rays ? 1 : 0;
    args.min_active = cfg.min_active;
    args.leaf_batch = cfg.leaf_batch;
    args.speculate = cfg.speculate ? 1 : 0;
    cuda_check(cudaMemsetAsync(work_counter, 0, sizeof(unsigned int), stream), "memset work counter");
    launch_any<true>(args, 0, cfg, all_split, stream);  // full persistent grid: the unit count lives on the device
    launch_film_commit_jobs(d_jobs, d_hdr, max_jobs, stream);
}

void launch_film_commit_jobs(const JobDesc* d_jobs, const BatchHeader* d_hdr, int max_jobs, cudaStream_t stream) {
    int dev = 0, sms = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    film_commit_jobs<<<dim3((unsigned)sms, (unsigned)std::max(1, max_jobs)), 256, 0, stream>>>(d_jobs, d_hdr);
    cuda_check(cudaGetLastError(), "film commit launch");
}

KernelTimer::~KernelTimer() {
    for (cudaEvent_t e : ev_) cudaEventDestroy(e);
}

void KernelTimer::begin(cudaStream_t stream) {
    while ((int)ev_.size() < used_ + 2) {
        cudaEvent_t e = nullptr;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        ev_.push_back(e);
    }
    cuda_check(cudaEventRecord(ev_[used_], stream), "cudaEventRecord");
}

void KernelTimer::end(cudaStream_t stream) {
    cuda_check(cudaEventRecord(ev_[used_ + 1], stream), "cudaEventRecord");
    used_ += 2;
}

double KernelTimer::total_ms() const {
    double ms = 0.0;
    for (int i = 0; i + 1 < used_; i += 2) {
        float t = 0.f;
        cuda_check(cudaEventElapsedTime(&t, ev_[i], ev_[i + 1]), "cudaEventElapsedTime");
        ms += t;
    }
    return ms;
}

}  // namespace wfb
