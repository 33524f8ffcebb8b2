// Persistent megakernel: one lane per path, register-resident state, one launch per render.
//
// Replaces megakernel_kernel / run_megakernel_pass (WVM/src/gpu/megakernel.cu:11-104), which
// launches one thread per pixel per sample, traces each path to completion and synchronises the
// host after every sample (lane efficiency 7-12 of 32 in the reference's own profiles). Here:
//
//  * Persistent threads: the grid is the set of CTAs resident at once; work units are handed out
//    by a global counter with warp-aggregated fetches (one atomic per warp per refill).
//  * Resumable traversal: the stackless skip-link traversal state of a ray is just the next node
//    index plus the best hit so far, so it survives across loop iterations. A warp keeps stepping
//    the traversal of all its lanes while at least `min_active` lanes are still traversing; only
//    then does it run the shading code, for exactly the lanes whose ray has finished, and gives
//    them their next ray (the extension ray, the pending shadow ray of a Lambertian bounce, or
//    the camera ray of the next sample). Lanes that are mid-traversal keep their state. This is
//    the "dynamic ray fetch" of Aila and Laine (HPG 2009) adapted to one-lane-per-path shading.
//  * Film order: a work unit is one pixel and a run of its samples in ascending order. In direct
//    mode a unit covers all samples of the pixel and the lane adds every finished path to register
//    copies of the pixel's film sums (film_add order of WVM/src/gpu/engine.cuh:25-32), writing the
//    film once. In split mode (images with fewer pixels than resident lanes) a pixel's samples are
//    cut into chunks handed to different lanes; each path's radiance goes to its (pixel, sample)
//    slot of a scratch buffer and a second kernel adds the slots to the film in sample order.
//    Both modes produce bit-identical films.
//  * The shadow ray of a Lambertian bounce starts at the next extension ray's origin
//    (p + n * eps, WVM/include/wf/path_core.hpp:197,210,226); only its direction, tmax and
//    contribution are kept.
//  * Ray counters live in registers and are folded with one atomic per warp at exit.
// Every per-path float operation is the reference's (see wf/path_core.hpp), so the film is
// bit-identical to the reference arms for the same scene arrays and seed.
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
    float* lbuf;        // split mode: radiance per (pixel, sample - first), 3 floats each
    int pixels;
    int first_sample;
    int sample_count;
    int chunk;          // samples per work unit (== sample_count in direct mode)
    int chunks;         // work units per pixel
    uint32_t seed;
    int max_depth;
    int count_rays;
    int min_active;     // keep traversing while at least this many lanes of the warp traverse
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) megakernel_persistent(const MkArgs a) {
    const DevScene& s = a.s;
    const int lane = threadIdx.x & 31;
    const bool split = a.chunks > 1;
    const unsigned total_units = (unsigned)a.pixels * (unsigned)a.chunks;

    // ---- per-lane work and path state ----
    int pixel = -1, px = 0, py = 0, sample = 0, s_end = 0;
    bool out_of_work = false;
    wf::PathState ps{};
    float acc_r = 0.f, acc_g = 0.f, acc_b = 0.f, acc_l = 0.f, acc_l2 = 0.f;
    bool shadow_ray = false, alive_after_shadow = false;
    wf::Vec3 sh_dir{0.f, 0.f, 0.f}, sh_contrib{0.f, 0.f, 0.f};
    float sh_tmax = 0.f;
    // ---- traversal state of the lane's current ray ----
    int node = -1;  // next node to visit; -1: no ray in flight
    wf::Vec3 rd{0.f, 0.f, 1.f}, inv_d{0.f, 0.f, 1.f};
    float r_tmin = 0.f;
    wf::HitRecord h;
    h.t = 0.f;
    h.prim = -1;
    h.u = h.v = 0.f;
    unsigned long long n_ext = 0, n_shadow = 0;
    unsigned int n_invalid = 0;

    auto start_ray = [&]() {
        // intersect() prologue (WVM/include/wf/bvh.hpp:92-94) for the extension or shadow ray.
        rd = shadow_ray ? sh_dir : ps.ray.d;
        r_tmin = shadow_ray ? wf::kRayEps : ps.ray.tmin;
        h.t = shadow_ray ? sh_tmax : ps.ray.tmax;
        h.prim = -1;
        h.u = 0.0f;
        h.v = 0.0f;
        inv_d = wf::Vec3{1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z};
        node = s.n_nodes > 0 ? 0 : -1;
    };

    for (;;) {
        // ================= traversal: step all traversing lanes, one node each =================
        for (;;) {
            const bool trav = node >= 0;
            const unsigned tmask = __ballot_sync(kFull, trav);
            if (tmask == 0) break;
            if (__popc(tmask) < a.min_active) {
                // few lanes left traversing: stop if some other lane has shading or refill to do
                const bool waiting = !trav && (pixel >= 0 || !out_of_work);
                if (__ballot_sync(kFull, waiting) != 0) break;
            }
            if (!trav) continue;
            const float4 na = __ldg(&s.nodes[2 * node]);
            const float4 nb = __ldg(&s.nodes[2 * node + 1]);
            const int skip = __float_as_int(na.w);
            wf::Ray r;
            r.o = ps.ray.o;
            r.d = rd;
            r.tmin = r_tmin;
            r.tmax = h.t;  // the best hit so far bounds the ray (r.tmax = t on every hit)
            if (!wf::hit_box(wf::Vec3{na.x, na.y, na.z}, wf::Vec3{nb.x, nb.y, nb.z}, r.o, inv_d, r.tmin, r.tmax)) {
                node = skip;
            } else {
                const int leaf = __float_as_int(nb.w);
                if (leaf < 0) {
                    node = node + 1;
                } else {
                    node = skip;
                    const int count = leaf & kLeafCountMask;
                    const float4* rec = s.prims + 3 * (leaf >> kLeafCountBits);
                    for (int i = 0; i < count; ++i, rec += 3) {
                        const float4 q0 = __ldg(rec);
                        const float4 q1 = __ldg(rec + 1);
                        const int p = __float_as_int(q0.w);
                        float t, u = 0.0f, v = 0.0f;
                        bool hit;
                        if (p < s.n_spheres) {
                            hit = wf::hit_sphere_core(wf::Vec3{q0.x, q0.y, q0.z}, q1.x, r, &t);
                        } else {
                            const float4 q2 = __ldg(rec + 2);
                            hit = wf::hit_triangle_core(wf::Vec3{q0.x, q0.y, q0.z}, wf::Vec3{q1.x, q1.y, q1.z},
                                                        wf::Vec3{q2.x, q2.y, q2.z}, r, &t, &u, &v);
                        }
                        if (hit) {
                            r.tmax = t;
                            h.t = t;
                            h.prim = p;
                            h.u = u;
                            h.v = v;
                            if (shadow_ray) {  // any-hit: the first hit ends the query
                                node = -1;
                                break;
                            }
                        }
                    }
                }
            }
            if (node >= s.n_nodes) node = -1;
        }

        // ================= shading: lanes whose ray has finished =================
        if (node < 0 && pixel >= 0) {
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
                    const int mat = wf::classify(s, ps, h, a.max_depth, &f);
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
                if (split) {
                    float* slot = a.lbuf + 3 * ((size_t)pixel * a.sample_count + (sample - a.first_sample));
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
                    ps = wf::init_path(s, px, py, (uint32_t)sample, a.seed);
                } else {
                    if (!split) {
                        a.film.rgb[3 * pixel] = acc_r;
                        a.film.rgb[3 * pixel + 1] = acc_g;
                        a.film.rgb[3 * pixel + 2] = acc_b;
                        a.film.lum[pixel] = acc_l;
                        a.film.lum2[pixel] = acc_l2;
                    }
                    pixel = -1;
                }
            }
            if (pixel >= 0) start_ray();
        }

        // ================= refill: lanes without a unit take the next ones =================
        const bool need = pixel < 0 && !out_of_work;
        const unsigned need_mask = __ballot_sync(kFull, need);
        if (need_mask) {
            const int leader = __ffs(need_mask) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(a.work, (unsigned)__popc(need_mask));
            base = __shfl_sync(kFull, base, leader);
            if (need) {
                const unsigned u = base + __popc(need_mask & ((1u << lane) - 1u));
                if (u < total_units) {
                    // unit u: pixel u mod P, chunk u div P (neighbouring lanes, neighbouring pixels)
                    pixel = (int)(u % (unsigned)a.pixels);
                    const int c = (int)(u / (unsigned)a.pixels);
                    px = pixel % s.width;
                    py = pixel / s.width;
                    sample = a.first_sample + c * a.chunk;
                    s_end = min(sample + a.chunk, a.first_sample + a.sample_count);
                    if (!split) {
                        acc_r = a.film.rgb[3 * pixel];
                        acc_g = a.film.rgb[3 * pixel + 1];
                        acc_b = a.film.rgb[3 * pixel + 2];
                        acc_l = a.film.lum[pixel];
                        acc_l2 = a.film.lum2[pixel];
                    }
                    ps = wf::init_path(s, px, py, (uint32_t)sample, a.seed);
                    shadow_ray = false;
                    start_ray();
                } else {
                    out_of_work = true;
                }
            }
        }
        if (__ballot_sync(kFull, pixel >= 0) == 0) break;
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

// Split mode: film_add of every (pixel, sample) slot in ascending sample order.
__global__ void film_commit(DevFilm film, const float* __restrict__ lbuf, int pixels, int count) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    float r = film.rgb[3 * p], g = film.rgb[3 * p + 1], b = film.rgb[3 * p + 2];
    float l1 = film.lum[p], l2 = film.lum2[p];
    const float* slot = lbuf + 3 * (size_t)p * count;
    for (int k = 0; k < count; ++k, slot += 3) {
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

template <int BLOCK>
int resident_lanes(int blocks_per_sm) {
    int dev = 0, sms = 0, occ = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, megakernel_persistent<BLOCK>, BLOCK, 0),
               "occupancy");
    if (blocks_per_sm > 0 && blocks_per_sm < occ) occ = blocks_per_sm;
    if (occ < 1) occ = 1;
    return sms * occ;  // resident CTAs
}

template <int BLOCK>
void launch_block(const MkArgs& args, int blocks_per_sm, cudaStream_t stream) {
    long long grid = resident_lanes<BLOCK>(blocks_per_sm);
    const long long units = (long long)args.pixels * args.chunks;
    const long long needed = (units + BLOCK - 1) / BLOCK;
    if (grid > needed) grid = needed;
    if (grid < 1) grid = 1;
    megakernel_persistent<BLOCK><<<(unsigned)grid, BLOCK, 0, stream>>>(args);
    cuda_check(cudaGetLastError(), "megakernel launch");
}

}  // namespace

void launch_film_commit(const DevFilm& film, const float* lbuf, int count, cudaStream_t stream) {
    if (film.pixels <= 0 || count <= 0) return;
    film_commit<<<(film.pixels + 255) / 256, 256, 0, stream>>>(film, lbuf, film.pixels, count);
    cuda_check(cudaGetLastError(), "film commit launch");
}

int megakernel_resident_threads(const MegakernelConfig& cfg) {
    switch (cfg.block) {
        case 64: return 64 * resident_lanes<64>(cfg.blocks_per_sm);
        case 256: return 256 * resident_lanes<256>(cfg.blocks_per_sm);
        default: return 128 * resident_lanes<128>(cfg.blocks_per_sm);
    }
}

int megakernel_split_chunks(int pixels, int sample_count, const MegakernelConfig& cfg) {
    if (cfg.split_chunks > 0) return std::min(cfg.split_chunks, std::max(1, sample_count));
    // Enough units to keep every resident lane busy through the tail: aim for 4 units per lane.
    const long long lanes = megakernel_resident_threads(cfg);
    if ((long long)pixels >= 4 * lanes || sample_count <= 1) return 1;
    long long k = (4 * lanes + pixels - 1) / pixels;
    if (k > sample_count) k = sample_count;
    return (int)k;
}

void launch_megakernel(const DevScene& s, const DevFilm& film, DevCounters* counters, unsigned int* work_counter,
                       float* lbuf, const PassParams& p, const MegakernelConfig& cfg, int chunks,
                       cudaStream_t stream) {
    if (p.sample_count <= 0 || film.pixels <= 0) return;
    if (chunks > 1 && lbuf == nullptr) throw Error(WFB_ERR_INTERNAL, "split megakernel needs a sample buffer");
    MkArgs args;
    args.s = s;
    args.film = film;
    args.counters = counters;
    args.work = work_counter;
    args.lbuf = lbuf;
    args.pixels = film.pixels;
    args.first_sample = p.first_sample;
    args.sample_count = p.sample_count;
    args.chunks = chunks < 1 ? 1 : chunks;
    args.chunk = (p.sample_count + args.chunks - 1) / args.chunks;
    args.chunks = (p.sample_count + args.chunk - 1) / args.chunk;  // no empty trailing chunk
    args.seed = p.seed;
    args.max_depth = p.max_depth;
    args.count_rays = p.count_rays ? 1 : 0;
    args.min_active = cfg.min_active;
    cuda_check(cudaMemsetAsync(work_counter, 0, sizeof(unsigned int), stream), "memset work counter");
    switch (cfg.block) {
        case 64: launch_block<64>(args, cfg.blocks_per_sm, stream); break;
        case 256: launch_block<256>(args, cfg.blocks_per_sm, stream); break;
        case 128: launch_block<128>(args, cfg.blocks_per_sm, stream); break;
        default: throw Error(WFB_ERR_INVALID_ARGUMENT, "megakernel block size must be 64, 128 or 256");
    }
    if (args.chunks > 1) {
        film_commit<<<(film.pixels + 255) / 256, 256, 0, stream>>>(film, lbuf, film.pixels, p.sample_count);
        cuda_check(cudaGetLastError(), "film commit launch");
    }
}

}  // namespace wfb
