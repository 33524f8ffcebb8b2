// Persistent-threads wavefront: the whole render is ONE cooperative launch that iterates bounces on
// the device. Replaces the reference's wavefront (WVM/src/gpu/wavefront.cu:30-601), which launches
// 12+ kernels per bounce and synchronises the host 3 times per bounce.
//
// Path pool: `capacity` slots, structure of arrays (one array per field, coalesced by slot id),
// in one arena. A pool that fits the device's persisting L2 set-aside (about 180 B per slot, so a
// few hundred thousand paths on a B200; wavefront_l2_resident_paths) runs under a persisting
// access-policy window on every launch, so its state stays in L2 across bounces; larger pools (up
// to 16M paths, the default) stream through HBM. A slot owns a work unit (a pixel and a run of its samples, as in
// the megakernel) and, when its path ends, regenerates the next sample of the same pixel or takes a
// new unit: paths in flight stay constant until the work runs out. Film sums are kept per slot in
// sample order (direct mode) or per (pixel, sample) in a buffer committed in order afterwards
// (split mode), so the film is bit-identical to every arm.
//
// One bounce = five phases separated by grid barriers (bounded spins, error flag on timeout):
//   R  regenerate + compact: ended slots commit their sample and start the next one (or fetch a
//      unit, or go idle); a decoupled-look-back scan over the active list writes the next active
//      list, stable, and its length.
//   E  extend: closest-hit traversal of every active path, lanes fetching rays dynamically from
//      the active list (one atomic per warp per refill) and stepping a resumable stackless
//      traversal, so a warp never waits for its longest ray.
//   C  classify: validity check, emission/MIS/termination; slots pushed to the Lambertian, metal or
//      dielectric queue with warp-aggregated pushes (drop-and-count past the test capacity).
//   S  shade: the three material queues (shade_lambert pushes shadow records).
//   H  shadow: any-hit traversal of the shadow queue with dynamic fetch; unoccluded contributions
//      are added to the path radiance (a slot has at most one shadow record per bounce).
// Stage times come from %globaltimer at the barriers (no host synchronisation).
#include <algorithm>
#include <cstring>
#include <mutex>
#include "engine.hpp"
#include "queues.cuh"
#include "wavefront.hpp"
#include "../../include/wfb200.h"

namespace wfb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWfBlock = 128;
// Box steps per box round of the traversal phases (as kBoxSteps in the megakernel): a lane that can
// still step takes up to this many before the warp votes again (B200, 1280x720x64, against one:
// icospheres +8%, heightfield +11%; 8 beat 4).
constexpr int kWfBoxSteps = 8;
constexpr int kStages = 8;  // extend, classify, lambert, metal, dielectric, shadow, compact, other

struct Control {
    unsigned bar_count;
    unsigned bar_gen;
    unsigned n_active;
    unsigned n_next;
    unsigned qcount[4];  // lambert, metal, dielectric, shadow
    unsigned fetch[2];   // extend, shadow dynamic-fetch cursors
    unsigned unit_next;
    unsigned ticket;
    unsigned retired;    // extension rays finished in the current E phase
    unsigned suspended;  // extension rays carried over to the next iteration (all phases)
    unsigned err;
    unsigned overflow;
    unsigned invalid;
    unsigned high_water[5];
    unsigned long long ext_rays;
    unsigned long long shadow_rays;
    unsigned long long stage_ns[kStages];
};

struct Pool {
    float4* ray_o;   // origin, tmin
    float4* ray_d;   // direction, tmax
    float4* thr;     // throughput, prev_pdf
    float4* rad;     // L, depth | specular << 30
    uint2* key;
    int4* unit;      // pixel (-1: none), sample, end sample, 0
    float4* acc;     // film sums of the unit (direct mode only; outside the pool arena): rgb, lum
    float* acc2;     // lum2
    float4* hit;     // t, prim, u, v (a suspended ray: its best hit so far)
    int2* trav;      // a suspended ray's traversal state: next node, pending leaf
    uint32_t* alive;  // 0: no path, 1: path with a ray to trace, 2: extension ray suspended mid-traversal
    uint32_t* list[2];
    uint32_t* queue[4];  // lambert, metal, dielectric, shadow slots
    float4* sh_dir;      // shadow records: direction, tmax
    float4* sh_c;        // contribution, owner slot
    unsigned long long* status;
    Control* ctl;
};

struct WfArgs {
    JobDesc job0;             // single render: the one job, in parameter space
    const JobDesc* jobs;      // batch: device job table (units numbered across jobs)
    const BatchHeader* hdr;   // batch: job count and total units
    Pool pool;
    int capacity;
    uint32_t qcap;  // queue capacity (test hook); capacity otherwise
    int min_active;
    int leaf_batch;
    int split_shading;  // stage timing: a barrier between material queues
    int suspend;        // extension stragglers may be suspended to the next iteration
    int speculate;      // speculative traversal (box_step)
    unsigned long long wait_ns;  // limit of every bounded wait (grid barriers, look-backs)
    unsigned bar_extra;          // CTAs a barrier waits for beyond the launch's own (0; 1 only in the
                                 // wait-timeout test, where no barrier can complete)
};

// The job a slot's path belongs to (its unit's .w); a single render has only job0.
template <bool MULTI>
__device__ __forceinline__ const JobDesc& job_at(const WfArgs& a, int j) {
    return MULTI ? a.jobs[j] : a.job0;
}

__device__ __forceinline__ wf::PathState load_path(const Pool& P, int slot) {
    const float4 o = P.ray_o[slot], d = P.ray_d[slot], t = P.thr[slot], l = P.rad[slot];
    const uint2 k = P.key[slot];
    wf::PathState ps;
    ps.ray.o = wf::Vec3{o.x, o.y, o.z};
    ps.ray.tmin = o.w;
    ps.ray.d = wf::Vec3{d.x, d.y, d.z};
    ps.ray.tmax = d.w;
    ps.throughput = wf::Vec3{t.x, t.y, t.z};
    ps.prev_pdf = t.w;
    ps.L = wf::Vec3{l.x, l.y, l.z};
    const int bits = __float_as_int(l.w);
    ps.depth = bits & 0x3fffffff;
    ps.specular = (bits >> 30) & 1;
    ps.key.k0 = k.x;
    ps.key.k1 = k.y;
    return ps;
}

__device__ __forceinline__ void store_path(const Pool& P, int slot, const wf::PathState& ps) {
    P.ray_o[slot] = make_float4(ps.ray.o.x, ps.ray.o.y, ps.ray.o.z, ps.ray.tmin);
    P.ray_d[slot] = make_float4(ps.ray.d.x, ps.ray.d.y, ps.ray.d.z, ps.ray.tmax);
    P.thr[slot] = make_float4(ps.throughput.x, ps.throughput.y, ps.throughput.z, ps.prev_pdf);
    P.rad[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, __int_as_float(ps.depth | (ps.specular << 30)));
    P.key[slot] = make_uint2(ps.key.k0, ps.key.k1);
}

__device__ __forceinline__ void store_radiance(const Pool& P, int slot, const wf::PathState& ps) {
    P.rad[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, __int_as_float(ps.depth | (ps.specular << 30)));
}

// Grid-wide barrier over `nblocks` arrivals of co-resident CTAs (cooperative launch). Bounded: a
// wait longer than limit_ns, or an error raised elsewhere, makes every CTA leave with `false`.
__device__ bool grid_sync(Control* c, unsigned nblocks, int stage, unsigned long long* t_last,
                          unsigned long long limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = &c->bar_gen;
        const unsigned g = *gen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(&c->bar_count, 1u) == nblocks - 1) {
            c->bar_count = 0;
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (*gen == g) {
                if (*(volatile unsigned*)&c->err != 0u || global_ns() - t0 > limit_ns) {
                    atomicExch(&c->err, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile unsigned*)&c->err != 0u) ok = 0;
        if (blockIdx.x == 0 && stage >= 0) {
            const unsigned long long now = global_ns();
            c->stage_ns[stage] += now - *t_last;
            *t_last = now;
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Resumable closest-hit / any-hit traversal over a list of rays fetched dynamically.
// Extend: items[i] are slot ids. Shadow: the rays are shadow records 0..n-1 (items unused).
//
// Extension stragglers: the phase ends when its last ray does, and near the end a few long rays
// keep whole warps (and the grid barrier) waiting. Once `suspend_at` of the phase's n rays have
// finished, a warp that has nothing left to fetch parks its unfinished rays instead -- next node,
// pending leaf and best hit into the pool, slot state 2 -- and leaves; the slot skips this bounce's
// classify and shading, stays in the active list, and its ray resumes from exactly that state in
// the next iteration's extend phase. The traversal steps are the same, so the hit is the same.
template <bool SHADOW, bool MULTI>
__device__ void traverse_phase(const WfArgs& a, const uint32_t* items, unsigned n, unsigned* cursor,
                               unsigned long long* n_rays, unsigned* retired = nullptr,
                               unsigned suspend_at = 0xffffffffu) {
    const Pool& P = a.pool;
    // BVH of the lane's current ray: a batch reads its job's from the table at fetch time
    const float4* nodes = a.job0.s.nodes;
    const float4* prims = a.job0.s.prims;
    int n_nodes = a.job0.s.n_nodes, n_spheres = a.job0.s.n_spheres;
    const int lane = threadIdx.x & 31;
    int item = -1;  // list position, -1: none
    uint32_t id = 0;  // slot (extend) or shadow record (shadow) of the current ray
    int node = -1;
    int pend = 0;  // pending leaf (box_step / prim_step)
    bool spec = false;  // the ray may take box steps while it holds a pending leaf (box_step)
    wf::Vec3 o{0.f, 0.f, 0.f};
    TravRay ray;
    wf::HitRecord h;
    h.t = 0.f;
    h.prim = -1;
    h.u = h.v = 0.f;
    bool exhausted = false;
    for (;;) {
        // refill lanes without a ray
        const bool need = item < 0 && !exhausted;
        const unsigned nm = __ballot_sync(kFull, need);
        if (nm) {
            const int leader = __ffs(nm) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(cursor, (unsigned)__popc(nm));
            base = __shfl_sync(kFull, base, leader);
            if (need) {
                const unsigned i = base + __popc(nm & ((1u << lane) - 1u));
                if (i < n) {
                    item = (int)i;
                    id = SHADOW ? i : items[i];  // shadow records are numbered by queue position
                    // every ray starts at its path's origin with tmin = kRayEps (see TravRay)
                    const int slot = SHADOW ? __float_as_int(P.sh_c[id].w) : (int)id;
                    int nested = a.job0.s.boxes_nested;
                    if (MULTI) {
                        const DevScene& js = a.jobs[P.unit[slot].w].s;
                        nodes = js.nodes;
                        prims = js.prims;
                        n_nodes = js.n_nodes;
                        n_spheres = js.n_spheres;
                        nested = js.boxes_nested;
                    }
                    const float4 oo = P.ray_o[slot];
                    const float4 d = SHADOW ? P.sh_dir[id] : P.ray_d[id];
                    o = wf::Vec3{oo.x, oo.y, oo.z};
                    traversal_begin(n_nodes, wf::Vec3{d.x, d.y, d.z}, d.w, &ray, &node, &h);
                    pend = 0;
                    spec = a.speculate && (SHADOW || (nested && finite_inv(ray)));
                    if (!SHADOW && P.alive[slot] == 2u) {  // resume a suspended ray where it stopped
                        const int2 tv = P.trav[slot];
                        const float4 hv = P.hit[slot];
                        node = tv.x;
                        pend = tv.y;
                        h.t = hv.x;
                        h.prim = __float_as_int(hv.y);
                        h.u = hv.z;
                        h.v = hv.w;
                        P.alive[slot] = 1u;
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (__ballot_sync(kFull, item >= 0) == 0) return;
        // rounds of box steps or primitive steps while enough lanes traverse (or nothing is left
        // to fetch); see box_step / prim_step
        unsigned round = 0;
        for (;;) {
            const bool in_leaf = pend != 0;
            const bool at_box = can_box_step(node, pend, spec);
            const unsigned pm = __ballot_sync(kFull, in_leaf);
            const unsigned bm = __ballot_sync(kFull, at_box);
            const unsigned tm = pm | bm;
            if (tm == 0) break;
            if (__popc(tm) < a.min_active && __ballot_sync(kFull, !(in_leaf || at_box) && !exhausted) != 0) break;
            if (!SHADOW && (++round & 31u) == 0u && __ballot_sync(kFull, exhausted) != 0) {
                // nothing left to fetch: suspend the warp's rays once most of the phase is done
                unsigned done = 0;
                if (lane == 0) done = *(volatile unsigned*)retired;
                done = __shfl_sync(kFull, done, 0);
                if (done >= suspend_at) {
                    // every lane holding an item parks it, finished ones included: the saved best
                    // hit makes a finished ray retire with its result on resumption
                    const unsigned sm = __ballot_sync(kFull, item >= 0);
                    if (item >= 0) {
                        P.trav[id] = make_int2(node, pend);
                        P.hit[id] = make_float4(h.t, __int_as_float(h.prim), h.u, h.v);
                        P.alive[id] = 2u;
                        item = -1;
                        node = -1;
                        pend = 0;
                    }
                    if (lane == 0) atomicAdd(&a.pool.ctl->suspended, (unsigned)__popc(sm));
                    return;
                }
            }
            // a single-job launch reads its BVH from parameter space, keeping registers for the ray
            const int np = __popc(pm);
            if (np != 0 && (np >= a.leaf_batch || np >= __popc(bm))) {
                if (in_leaf) {
                    if (MULTI) prim_step(prims, n_spheres, o, ray, SHADOW, node, pend, h);
                    else prim_step(a.job0.s.prims, a.job0.s.n_spheres, o, ray, SHADOW, node, pend, h);
                }
            } else if (at_box) {
#pragma unroll
                for (int k = 0; k < kWfBoxSteps; ++k) {
                    if (k == 0 || can_box_step(node, pend, spec)) {
                        if (MULTI) box_step(nodes, n_nodes, o, ray, h.t, node, pend);
                        else box_step(a.job0.s.nodes, a.job0.s.n_nodes, o, ray, h.t, node, pend);
                    }
                }
            }
        }
        // retire finished rays
        const bool fin = item >= 0 && node < 0 && pend == 0;
        if (!SHADOW) {
            const unsigned fm = __ballot_sync(kFull, fin);
            if (fm && lane == __ffs(fm) - 1) atomicAdd(retired, (unsigned)__popc(fm));
        }
        if (fin) {
            ++*n_rays;
            if (SHADOW) {
                if (h.prim < 0) {  // unoccluded: L += contrib
                    const float4 c = P.sh_c[id];
                    const int slot = __float_as_int(c.w);
                    float4 l = P.rad[slot];
                    l.x += c.x;
                    l.y += c.y;
                    l.z += c.z;
                    P.rad[slot] = l;
                }
            } else {
                P.hit[id] = make_float4(h.t, __int_as_float(h.prim), h.u, h.v);
            }
            item = -1;
        }
    }
}

// MINB > 1 caps registers so that MINB CTAs fit an SM (the whole bounce loop is one kernel, so its
// register count is the largest of any phase's; the traversal phases want the warps more than the
// shading phases want the registers).
template <bool MULTI, int MINB>
__global__ void __launch_bounds__(kWfBlock, MINB) wavefront_persistent(const WfArgs a) {
    const Pool& P = a.pool;
    Control* c = P.ctl;
    const int lane = threadIdx.x & 31;
    const unsigned nblocks = gridDim.x + a.bar_extra;  // arrivals that complete a barrier
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gthreads = gridDim.x * blockDim.x;
    const unsigned total_units = MULTI ? a.hdr->total_units : a.job0.units;
    const int n_jobs = MULTI ? (int)a.hdr->n_jobs : 1;
    __shared__ uint32_t smem[33];
    __shared__ int s_tile;
    __shared__ uint32_t s_prefix;
    unsigned long long t_last = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) t_last = global_ns();
    unsigned long long n_ext = 0, n_sh = 0;
    unsigned n_invalid = 0;

    for (unsigned iter = 1;; ++iter) {
        const int cur = (iter - 1) & 1;
        const uint32_t* active = P.list[cur];
        uint32_t* next = P.list[cur ^ 1];
        const unsigned n_act = *(volatile unsigned*)&c->n_active;

        // ---------------- R: regenerate ended paths, compact the active list ----------------
        if (gtid == 0) {
            c->qcount[0] = c->qcount[1] = c->qcount[2] = c->qcount[3] = 0;
            c->fetch[0] = c->fetch[1] = 0;
            c->retired = 0;
        }
        const unsigned ntiles = (n_act + kWfBlock - 1) / kWfBlock;
        for (;;) {
            if (threadIdx.x == 0) s_tile = (int)atomicAdd(&c->ticket, 1u);
            __syncthreads();
            const int tile = s_tile;
            if (tile >= (int)ntiles) break;
            const unsigned i = (unsigned)tile * kWfBlock + threadIdx.x;
            const bool valid = i < n_act;
            const int slot = valid ? (int)active[i] : 0;
            bool has_path = false, need_unit = false;
            int4 u = make_int4(-1, 0, 0, 0);
            if (valid) {
                has_path = P.alive[slot] != 0u;
                if (!has_path) {
                    u = P.unit[slot];
                    if (u.x >= 0) {
                        const JobDesc& J = job_at<MULTI>(a, u.w);
                        const bool split = J.chunks > 1;
                        // commit the finished sample (film_add order, WVM/src/gpu/engine.cuh:25-32)
                        const float4 l = P.rad[slot];
                        if (split) {
                            float* dst = J.lbuf + sample_slot(u.x, u.y - J.first_sample, J.film.pixels);
                            dst[0] = l.x;
                            dst[1] = l.y;
                            dst[2] = l.z;
                        } else {
                            float4 ac = P.acc[slot];
                            float a2 = P.acc2[slot];
                            ac.x += l.x;
                            ac.y += l.y;
                            ac.z += l.z;
                            const float lu = wf::luminance(wf::Vec3{l.x, l.y, l.z});
                            ac.w += lu;
                            a2 += lu * lu;
                            P.acc[slot] = ac;
                            P.acc2[slot] = a2;
                        }
                        u.y += 1;
                        if (u.y < u.z) {
                            const int px = u.x % J.s.width, py = u.x / J.s.width;
                            store_path(P, slot, wf::init_path(J.s, px, py, (uint32_t)u.y, J.seed));
                            P.unit[slot] = u;
                            P.alive[slot] = 1u;
                            has_path = true;
                        } else {
                            if (!split) {
                                const float4 ac = P.acc[slot];
                                J.film.rgb[3 * u.x] = ac.x;
                                J.film.rgb[3 * u.x + 1] = ac.y;
                                J.film.rgb[3 * u.x + 2] = ac.z;
                                J.film.lum[u.x] = ac.w;
                                J.film.lum2[u.x] = P.acc2[slot];
                            }
                            u.x = -1;
                            P.unit[slot] = u;
                            need_unit = true;
                        }
                    } else {
                        need_unit = true;
                    }
                }
            }
            // fetch new units for slots that need one (one atomic per warp)
            const unsigned nm = __ballot_sync(kFull, need_unit);
            if (nm) {
                const int leader = __ffs(nm) - 1;
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(&c->unit_next, (unsigned)__popc(nm));
                base = __shfl_sync(kFull, base, leader);
                if (need_unit) {
                    const unsigned uid = base + __popc(nm & ((1u << lane) - 1u));
                    if (uid < total_units) {
                        // unit -> job, then pixel (local mod P) and chunk (local div P)
                        const int job = MULTI ? job_of_unit(a.jobs, n_jobs, uid) : 0;
                        const JobDesc& J = job_at<MULTI>(a, job);
                        const unsigned local = uid - J.unit_begin;
                        const int pixel = (int)(local % (unsigned)J.film.pixels);
                        const int ch = (int)(local / (unsigned)J.film.pixels);
                        const int first = J.first_sample + ch * J.chunk;
                        const int end = min(first + J.chunk, J.first_sample + J.sample_count);
                        P.unit[slot] = make_int4(pixel, first, end, job);
                        if (J.chunks == 1) {
                            P.acc[slot] = make_float4(J.film.rgb[3 * pixel], J.film.rgb[3 * pixel + 1],
                                                      J.film.rgb[3 * pixel + 2], J.film.lum[pixel]);
                            P.acc2[slot] = J.film.lum2[pixel];
                        }
                        store_path(P, slot, wf::init_path(J.s, pixel % J.s.width, pixel / J.s.width, (uint32_t)first, J.seed));
                        P.alive[slot] = 1u;
                        has_path = true;
                    }
                }
            }
            // stable compaction of the slots that still have a path
            const uint32_t flag = (valid && has_path) ? 1u : 0u;
            uint32_t agg;
            const uint32_t excl = block_exclusive_sum(flag, smem, &agg);
            if (threadIdx.x == 0) publish_status(P.status, tile, iter, tile == 0 ? kStatusPrefix : kStatusAggregate, agg);
            if (tile > 0 && threadIdx.x < 32) {
                const uint32_t pre = tile_lookback(P.status, tile, iter, &c->err, a.wait_ns);
                if (threadIdx.x == 0) {
                    publish_status(P.status, tile, iter, kStatusPrefix, pre + agg);
                    s_prefix = pre;
                }
            } else if (tile == 0 && threadIdx.x == 0) {
                s_prefix = 0;
            }
            __syncthreads();
            if (flag) next[s_prefix + excl] = (uint32_t)slot;
            if (tile == (int)ntiles - 1 && threadIdx.x == kWfBlock - 1) c->n_next = s_prefix + excl + flag;
            __syncthreads();
        }
        if (ntiles == 0 && gtid == 0) c->n_next = 0;
        if (!grid_sync(c, nblocks, 6, &t_last, a.wait_ns)) break;
        const unsigned n = *(volatile unsigned*)&c->n_next;
        if (gtid == 0) {
            c->n_active = n;
            c->ticket = 0;
            if (n > c->high_water[4]) c->high_water[4] = n;
        }
        if (n == 0) break;

        // ---------------- E: extension rays ----------------
        // stragglers may be suspended once 95% of a large phase's rays have finished
        traverse_phase<false, MULTI>(a, next, n, &c->fetch[0], &n_ext, &c->retired,
                                     a.suspend && n >= 4096 ? n - n / 20 : 0xffffffffu);
        if (!grid_sync(c, nblocks, 0, &t_last, a.wait_ns)) break;

        // ---------------- C: classify, push material queues ----------------
        for (unsigned base = (unsigned)blockIdx.x * kWfBlock; base < n; base += (unsigned)gthreads) {
            const unsigned i = base + threadIdx.x;
            const bool valid = i < n;
            const int slot = valid ? (int)next[i] : 0;
            int mat = -1;
            if (valid && P.alive[slot] != 2u) {  // a suspended ray has no hit yet
                const float4 hv = P.hit[slot];
                wf::HitRecord h;
                h.t = hv.x;
                h.prim = __float_as_int(hv.y);
                h.u = hv.z;
                h.v = hv.w;
                const JobDesc& J = job_at<MULTI>(a, MULTI ? P.unit[slot].w : 0);
                if (!hit_is_valid(J.s, h)) {
                    ++n_invalid;
                    h.prim = -1;  // treated as a miss
                }
                wf::PathState ps = load_path(P, slot);
                wf::Surface f;
                mat = wf::classify(J.s, ps, h, J.max_depth, &f);
                store_radiance(P, slot, ps);
                if (mat < 0) P.alive[slot] = 0u;
            }
            for (int q = 0; q < 3; ++q) {
                const bool mine = valid && mat == q;
                const uint32_t at = queue_push(P.queue[q], &c->qcount[q], a.qcap, (uint32_t)slot, mine, &c->overflow);
                if (mine && at == 0xFFFFFFFFu) P.alive[slot] = 0u;  // dropped on overflow: the path ends
            }
        }
        if (!grid_sync(c, nblocks, 1, &t_last, a.wait_ns)) break;

        // ---------------- S: shade the three material queues ----------------
        unsigned qn[3];
        for (int q = 0; q < 3; ++q) qn[q] = min(*(volatile unsigned*)&c->qcount[q], a.qcap);
        if (gtid == 0)
            for (int q = 0; q < 3; ++q)
                if (qn[q] > c->high_water[q]) c->high_water[q] = qn[q];
        bool ok = true;
        for (int q = 0; q < 3 && ok; ++q) {
            for (unsigned base = (unsigned)blockIdx.x * kWfBlock; base < qn[q]; base += (unsigned)gthreads) {
                const unsigned i = base + threadIdx.x;
                const bool valid = i < qn[q];
                bool push = false;
                int slot = 0;
                wf::Ray sh;
                wf::Vec3 contrib{0.f, 0.f, 0.f};
                if (valid) {
                    slot = (int)P.queue[q][i];
                    const DevScene& s = job_at<MULTI>(a, MULTI ? P.unit[slot].w : 0).s;
                    wf::PathState ps = load_path(P, slot);
                    // the surface classify saw: make_surface of the same ray and hit, so the same bits
                    const float4 hv = P.hit[slot];
                    wf::HitRecord h;
                    h.t = hv.x;
                    h.prim = __float_as_int(hv.y);
                    h.u = hv.z;
                    h.v = hv.w;
                    const wf::Surface f = wf::make_surface(s, ps.ray, h);
                    bool alive;
                    if (q == wf::kLambert) {
                        int has = 0;
                        alive = wf::shade_lambert(s, ps, f, &sh, &contrib, &has);
                        push = has != 0;
                    } else if (q == wf::kMetal) {
                        alive = wf::shade_metal(s, ps, f);
                    } else {
                        alive = wf::shade_dielectric(s, ps, f);
                    }
                    store_path(P, slot, ps);
                    P.alive[slot] = alive ? 1u : 0u;
                }
                if (q == wf::kLambert) {
                    const uint32_t at = queue_push(P.queue[3], &c->qcount[3], a.qcap, (uint32_t)slot, push, &c->overflow);
                    if (push && at != 0xFFFFFFFFu) {
                        P.sh_dir[at] = make_float4(sh.d.x, sh.d.y, sh.d.z, sh.tmax);
                        P.sh_c[at] = make_float4(contrib.x, contrib.y, contrib.z, __int_as_float(slot));
                    }
                }
            }
            if (a.split_shading && !grid_sync(c, nblocks, 2 + q, &t_last, a.wait_ns)) ok = false;
        }
        if (!ok) break;
        if (!a.split_shading && !grid_sync(c, nblocks, 2, &t_last, a.wait_ns)) break;

        // ---------------- H: shadow rays ----------------
        const unsigned nsh = min(*(volatile unsigned*)&c->qcount[3], a.qcap);
        if (gtid == 0 && nsh > c->high_water[3]) c->high_water[3] = nsh;
        traverse_phase<true, MULTI>(a, nullptr, nsh, &c->fetch[1], &n_sh);
        if (!grid_sync(c, nblocks, 5, &t_last, a.wait_ns)) break;
    }

    // ---- fold counters ----
    for (int off = 16; off > 0; off >>= 1) {
        n_ext += __shfl_down_sync(kFull, n_ext, off);
        n_sh += __shfl_down_sync(kFull, n_sh, off);
        n_invalid += __shfl_down_sync(kFull, n_invalid, off);
    }
    if (lane == 0) {
        if (n_ext) atomicAdd(&c->ext_rays, n_ext);
        if (n_sh) atomicAdd(&c->shadow_rays, n_sh);
        if (n_invalid) atomicAdd(&c->invalid, n_invalid);
    }
}

using WfKernel = void (*)(const WfArgs);

// The compiled register-cap variants: 0 (none), 6, 8 or 10 CTAs of kWfBlock threads per SM.
template <bool MULTI>
WfKernel wavefront_kernel(int occupancy) {
    switch (occupancy) {
        case 6: return wavefront_persistent<MULTI, 6>;
        case 8: return wavefront_persistent<MULTI, 8>;
        case 10: return wavefront_persistent<MULTI, 10>;
        default: return wavefront_persistent<MULTI, 1>;
    }
}

__global__ void wavefront_init(Pool P, int capacity) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        Control* c = P.ctl;
        c->n_active = (unsigned)capacity;
    }
    if (i < capacity) {
        P.list[0][i] = (uint32_t)i;
        P.alive[i] = 0u;
        P.unit[i] = make_int4(-1, 0, 0, 0);
    }
}

// Control block -> the renderer's counters (one thread; runs after the persistent kernel).
__global__ void wavefront_fold(const Control* c, DevCounters* out, int count_rays) {
    if (count_rays) {
        out->extension_rays += c->ext_rays;
        out->shadow_rays += c->shadow_rays;
    }
    out->invalid_hits += c->invalid;
    out->overflows += c->overflow;
    for (int i = 0; i < 5; ++i) out->high_water[i] = max(out->high_water[i], c->high_water[i]);
    if (c->err) out->error = kErrSpinTimeout;
}

template <class T>
T* carve(char*& p, size_t n) {
    T* r = reinterpret_cast<T*>(p);
    p += (n * sizeof(T) + 255) & ~(size_t)255;
    return r;
}

size_t pool_bytes(int cap, Pool* out, char* base) {
    char* p = base;
    Pool P;
    P.ray_o = carve<float4>(p, cap);
    P.ray_d = carve<float4>(p, cap);
    P.thr = carve<float4>(p, cap);
    P.rad = carve<float4>(p, cap);
    P.key = carve<uint2>(p, cap);
    P.unit = carve<int4>(p, cap);
    P.acc = nullptr;  // direct mode only: WavefrontEngine::reserve_direct
    P.acc2 = nullptr;
    P.hit = carve<float4>(p, cap);
    P.trav = carve<int2>(p, cap);
    P.alive = carve<uint32_t>(p, cap);
    P.list[0] = carve<uint32_t>(p, cap);
    P.list[1] = carve<uint32_t>(p, cap);
    for (int q = 0; q < 4; ++q) P.queue[q] = carve<uint32_t>(p, cap);
    P.sh_dir = carve<float4>(p, cap);
    P.sh_c = carve<float4>(p, cap);
    P.status = carve<unsigned long long>(p, (size_t)cap / kWfBlock + 2);
    P.ctl = carve<Control>(p, 1);
    if (out) *out = P;
    return (size_t)(p - base);
}

}  // namespace

struct WavefrontEngine::State {
    Pool pool{};
    float* lbuf = nullptr;
    size_t lbuf_floats = 0;
    void* acc = nullptr;  // direct-mode film sums per slot (float4 + float), allocated on first use
    WfKernel kernel = nullptr, kernel_multi = nullptr;  // the register-cap variant of cfg.occupancy
    int grid = 0;        // co-resident CTAs of the single-render kernel
    int grid_multi = 0;  // and of the batch kernel
    // L2 residency: an access-policy window over the pool arena on every launch (0 bytes: none)
    size_t window_bytes = 0;
    float hit_ratio = 0.f;
};

namespace {

// Persisting-L2 set-aside of this process's context (a context resource limit; it changes no device
// setting): raised to what the largest live L2-resident pool asks for, within the device's maximum,
// and set back to 0 when the last engine with a window is destroyed. A set-aside left in place cost
// every later kernel of the process L2 capacity: megakernel renders 2% slower, and a tuned 16M-path
// wavefront render 137 ms instead of 115 after the tuner had probed the resident pool.
std::mutex g_l2_mu;
size_t g_l2_persist = 0;
int g_l2_users = 0;

size_t reserve_persisting_l2(size_t want, int dev) {
    int max_persist = 0;
    cuda_check(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev), "persisting L2 size");
    want = std::min(want, (size_t)std::max(max_persist, 0));
    std::lock_guard<std::mutex> lock(g_l2_mu);
    if (want > g_l2_persist) {
        cuda_check(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want), "persisting L2 set-aside");
        g_l2_persist = want;
    }
    ++g_l2_users;
    return g_l2_persist;
}

// An engine with a window is gone: its lines become normal; the last one gives the set-aside back.
void release_persisting_l2() {
    std::lock_guard<std::mutex> lock(g_l2_mu);
    cudaCtxResetPersistingL2Cache();
    if (--g_l2_users <= 0) {
        g_l2_users = 0;
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
        g_l2_persist = 0;
    }
}

}  // namespace

size_t wavefront_slot_bytes() { return (pool_bytes(1 << 20, nullptr, nullptr) + (1 << 20) - 1) >> 20; }

size_t wavefront_l2_resident_paths(int device) {
    int max_persist = 0;
    cuda_check(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, device), "persisting L2 size");
    if (max_persist <= 0) return 0;
    // the largest multiple of the block whose whole arena fits the set-aside
    size_t slots = ((size_t)max_persist / wavefront_slot_bytes()) & ~(size_t)(kWfBlock - 1);
    while (slots > 0 && pool_bytes((int)slots, nullptr, nullptr) > (size_t)max_persist) slots -= kWfBlock;
    return slots;
}

WavefrontEngine::WavefrontEngine(int pixels, const WavefrontConfig& cfg) : pixels_(pixels), cfg_(cfg) {
    if (pixels <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "wavefront needs at least one pixel");
    int cap = cfg.paths_in_flight > 0 ? cfg.paths_in_flight : (1 << 24);
    if (cap > pixels * 64) cap = pixels * 64;  // never more slots than units can use
    if (cap < 32) cap = 32;
    capacity_ = cap;
    state_ = std::make_unique<State>();
    const size_t bytes = pool_bytes(cap, nullptr, nullptr);
    cuda_check(cudaMalloc(&arena_, bytes), "cudaMalloc wavefront pool");
    bytes_ = bytes;
    pool_bytes(cap, &state_->pool, static_cast<char*>(arena_));
    int dev = 0, sms = 0, occ = 0, coop = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "cooperative attribute");
    if (!coop) throw Error(WFB_ERR_UNSUPPORTED, "device does not support cooperative launches");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    if (cfg.occupancy != 0 && cfg.occupancy != 6 && cfg.occupancy != 8 && cfg.occupancy != 10)
        throw Error(WFB_ERR_INVALID_ARGUMENT, "wavefront occupancy target must be 0, 6, 8 or 10");
    state_->kernel = wavefront_kernel<false>(cfg.occupancy);
    state_->kernel_multi = wavefront_kernel<true>(cfg.occupancy);
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, state_->kernel, kWfBlock, 0), "occupancy");
    if (occ < 1) throw Error(WFB_ERR_UNSUPPORTED, "wavefront kernel does not fit on an SM");
    state_->grid = sms * occ;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, state_->kernel_multi, kWfBlock, 0), "occupancy");
    if (occ < 1) throw Error(WFB_ERR_UNSUPPORTED, "wavefront batch kernel does not fit on an SM");
    state_->grid_multi = sms * occ;
    // L2 residency: the pool (every field a bounce reads or writes) under a persisting window when
    // it fits the device's persisting set-aside (auto), or whenever asked (a partial window). Last in
    // the constructor: once the set-aside is counted, nothing can throw, so the destructor's release
    // always balances it.
    int max_persist = 0, max_window = 0;
    cuda_check(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev), "persisting L2 size");
    cuda_check(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev), "window size");
    const bool fits = bytes <= (size_t)max_persist;
    if (max_persist > 0 && max_window > 0 && (cfg.l2_persist > 0 || (cfg.l2_persist < 0 && fits))) {
        const size_t window = std::min(bytes, (size_t)max_window);
        const size_t carve = reserve_persisting_l2(window, dev);
        state_->window_bytes = window;
        state_->hit_ratio = (float)std::min(1.0, (double)carve / (double)window);
    }
}

WavefrontEngine::~WavefrontEngine() {
    if (state_ && state_->lbuf) cudaFree(state_->lbuf);
    if (state_ && state_->acc) cudaFree(state_->acc);
    if (state_ && state_->window_bytes) release_persisting_l2();
    if (arena_) cudaFree(arena_);
}

uint64_t WavefrontEngine::bytes() const {
    if (!state_) return bytes_;
    return bytes_ + state_->lbuf_floats * sizeof(float) + (state_->acc ? (size_t)capacity_ * 20 : 0);
}

size_t WavefrontEngine::l2_window_bytes() const { return state_ ? state_->window_bytes : 0; }

void WavefrontEngine::reserve_direct() {
    State& st = *state_;
    if (st.acc) return;
    const size_t acc_bytes = (size_t)capacity_ * sizeof(float4);
    cuda_check(cudaMalloc(&st.acc, acc_bytes + (size_t)capacity_ * sizeof(float)), "cudaMalloc direct-mode sums");
    st.pool.acc = static_cast<float4*>(st.acc);
    st.pool.acc2 = reinterpret_cast<float*>(static_cast<char*>(st.acc) + acc_bytes);
}

namespace {

// Control reset, pool init, the cooperative launch and the counter fold; returns kernels launched.
int launch_pool(WfKernel kernel, const WfArgs& args, int grid, int capacity, DevCounters* counters, bool count_rays,
                size_t window_bytes, float hit_ratio, cudaStream_t stream, KernelTimer* timer = nullptr) {
    const Pool& pool = args.pool;
    cuda_check(cudaMemsetAsync(pool.ctl, 0, sizeof(Control), stream), "memset control");
    cuda_check(cudaMemsetAsync(pool.status, 0, ((size_t)capacity / kWfBlock + 2) * sizeof(unsigned long long), stream),
               "memset status");
    wavefront_init<<<(capacity + 255) / 256, 256, 0, stream>>>(pool, capacity);
    cuda_check(cudaGetLastError(), "wavefront init launch");
    WfArgs a = args;
    a.wait_ns = device_wait_limit_ns();
    a.bar_extra = take_unsatisfiable_wait() ? 1u : 0u;
    // one cooperative launch; the pool arena (it starts at the path-state arrays) under a persisting
    // L2 window when the engine has one
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    int n_attr = 1;
    if (window_bytes > 0) {
        attr[1].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[1].val.accessPolicyWindow.base_ptr = static_cast<void*>(pool.ray_o);
        attr[1].val.accessPolicyWindow.num_bytes = window_bytes;
        attr[1].val.accessPolicyWindow.hitRatio = hit_ratio;
        attr[1].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[1].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        n_attr = 2;
    }
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(kWfBlock);
    lc.dynamicSmemBytes = 0;
    lc.stream = stream;
    lc.attrs = attr;
    lc.numAttrs = n_attr;
    if (timer) timer->begin(stream);
    cuda_check(cudaLaunchKernelEx(&lc, kernel, a), "wavefront cooperative launch");
    if (timer) timer->end(stream);
    wavefront_fold<<<1, 1, 0, stream>>>(pool.ctl, counters, count_rays ? 1 : 0);
    cuda_check(cudaGetLastError(), "wavefront fold launch");
    return 3;
}

}  // namespace

// One sample per unit while the per-sample buffer fits (as in the megakernel: consecutive slots get
// neighbouring pixels at the same sample, and a slot takes new work after every path); otherwise a
// pixel's samples are split only as far as needed to fill the pool.
int WavefrontEngine::chunks_for(int pixels, int sample_count) const {
    if (split_buffer_bytes(pixels, sample_count) <= kSplitBufferBytes) return sample_count;
    if (pixels < capacity_) return std::min(sample_count, (capacity_ + pixels - 1) / pixels);
    return 1;
}

void WavefrontEngine::reserve(int pixels, int sample_count) {
    State& st = *state_;
    if (pixels <= 0 || sample_count <= 0 || chunks_for(pixels, sample_count) <= 1) return;
    const size_t need = 3 * (size_t)pixels * (size_t)sample_count;
    if (need <= st.lbuf_floats) return;
    if (st.lbuf) cudaFree(st.lbuf);
    st.lbuf = nullptr;
    st.lbuf_floats = 0;
    cuda_check(cudaMalloc(&st.lbuf, need * sizeof(float)), "cudaMalloc wavefront sample buffer");
    st.lbuf_floats = need;
}

int WavefrontEngine::run(const DevScene& s, const DevFilm& film, DevCounters* counters, const PassParams& p,
                         wf::StageTimes* stages, cudaStream_t stream, KernelTimer* timer) {
    if (p.sample_count <= 0 || film.pixels <= 0) return 0;
    State& st = *state_;
    const int chunks = chunks_for(film.pixels, p.sample_count);
    WfArgs a{};
    a.job0 = make_job(s, film, nullptr, p.first_sample, p.sample_count, chunks, p.seed, p.max_depth);
    if (a.job0.chunks > 1) {
        reserve(film.pixels, p.sample_count);
        a.job0.lbuf = st.lbuf;
    } else {
        reserve_direct();
    }
    a.jobs = nullptr;
    a.hdr = nullptr;
    a.pool = st.pool;
    a.capacity = capacity_;
    a.qcap = (p.queue_capacity > 0 && p.queue_capacity < capacity_) ? (uint32_t)p.queue_capacity : (uint32_t)capacity_;
    a.min_active = cfg_.min_active > 0 ? cfg_.min_active : WavefrontConfig{}.min_active;
    a.leaf_batch = cfg_.leaf_batch > 0 ? cfg_.leaf_batch : 8;
    a.split_shading = p.stage_timing ? 1 : 0;
    a.suspend = cfg_.suspend_stragglers ? 1 : 0;
    a.speculate = cfg_.speculate ? 1 : 0;
    int launches = launch_pool(st.kernel, a, st.grid, capacity_, counters, p.count_rays, st.window_bytes, st.hit_ratio,
                                      stream, timer);
    if (a.job0.chunks > 1) {
        launch_film_commit(film, a.job0.lbuf, p.sample_count, stream);
        ++launches;
    }
    if (stages) {
        unsigned long long ns[kStages];
        cuda_check(cudaMemcpyAsync(ns, st.pool.ctl->stage_ns, sizeof(ns), cudaMemcpyDeviceToHost, stream), "stage times");
        cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        stages->extend += ns[0] * 1e-6;
        stages->classify += ns[1] * 1e-6;
        stages->shade_lambert += ns[2] * 1e-6;
        stages->shade_metal += ns[3] * 1e-6;
        stages->shade_dielectric += ns[4] * 1e-6;
        stages->shadow += ns[5] * 1e-6;
        stages->compact += ns[6] * 1e-6;
        stages->other += ns[7] * 1e-6;
    }
    return launches;
}

int WavefrontEngine::run_batch(const JobDesc* d_jobs, const BatchHeader* d_hdr, DevCounters* counters,
                               bool count_rays, cudaStream_t stream) {
    reserve_direct();  // a batch may hold direct-mode jobs
    WfArgs a{};
    a.jobs = d_jobs;
    a.hdr = d_hdr;
    a.pool = state_->pool;
    a.capacity = capacity_;
    a.qcap = (uint32_t)capacity_;
    a.min_active = cfg_.min_active > 0 ? cfg_.min_active : WavefrontConfig{}.min_active;
    a.leaf_batch = cfg_.leaf_batch > 0 ? cfg_.leaf_batch : 8;
    a.split_shading = 0;
    a.suspend = cfg_.suspend_stragglers ? 1 : 0;
    a.speculate = cfg_.speculate ? 1 : 0;
    return launch_pool(state_->kernel_multi, a, state_->grid_multi, capacity_, counters, count_rays, state_->window_bytes,
                             state_->hit_ratio, stream);
}

}  // namespace wfb
