// Device-side queue and scan primitives, written for sm_100a (no CUB, no Thrust):
//
//   queue_push       warp-aggregated reservation: one atomic per warp per push, drop-and-count past
//                    the capacity (semantics of WVM/src/gpu/queues.cuh:12-27).
//   block_scan       exclusive scan of one value per thread across a CTA (warp shuffles + smem).
//   tile_lookback    decoupled look-back over per-tile status words (Merrill & Garland, "Single-pass
//                    Parallel Prefix Scan with Decoupled Look-back", 2016), replacing the reference's
//                    three-kernel scan (WVM/src/gpu/queues.cu:69-140): one pass over the data.
//
// Tile status words are 64-bit: [63:34] epoch, [33:32] flag (1 aggregate, 2 inclusive prefix),
// [31:0] value. A status written by an earlier scan carries another epoch and reads as "not yet
// available", so the status array never has to be cleared between scans.
//
// Every spin is bounded: a wait that exceeds its limit (kDefaultWaitLimitNs of %globaltimer unless
// the host set another, device_wait_limit_ns) sets *err and returns, so a bug can never hang the
// GPU; callers report the error to the host.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace wfb {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr unsigned kStatusAggregate = 1u;
constexpr unsigned kStatusPrefix = 2u;
constexpr unsigned long long kDefaultWaitLimitNs = 2000000000ull;  // 2 s

#if defined(__CUDACC__)

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Lanes with pred reserve consecutive slots in `items` with ONE atomicAdd per warp; lanes past
// `capacity` are dropped and counted in *overflow. The whole warp must call it (full mask).
// Returns the slot, or 0xFFFFFFFF for lanes that did not push or were dropped.
__device__ __forceinline__ uint32_t queue_push(uint32_t* items, uint32_t* counter, uint32_t capacity,
                                               uint32_t value, bool pred, uint32_t* overflow) {
    const unsigned want = __ballot_sync(kFullMask, pred);
    if (want == 0) return 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(want) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(want));
    base = __shfl_sync(kFullMask, base, leader);
    if (!pred) return 0xFFFFFFFFu;
    const uint32_t slot = base + (uint32_t)__popc(want & ((1u << lane) - 1u));
    if (slot >= capacity) {
        atomicAdd(overflow, 1u);
        return 0xFFFFFFFFu;
    }
    items[slot] = value;
    return slot;
}

__device__ __forceinline__ uint32_t warp_inclusive_sum(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(kFullMask, v, off);
        if (lane >= off) v += o;
    }
    return v;
}

// Exclusive scan of `v` over the CTA; *total receives the CTA sum. `smem` holds >= 33 words.
// Every thread of the CTA must call it.
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* smem, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    const uint32_t inc = warp_inclusive_sum(v);
    __syncthreads();  // smem may still be read from a previous call
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < nwarps ? smem[lane] : 0u;
        const uint32_t wi = warp_inclusive_sum(w);
        if (lane < nwarps) smem[lane] = wi - w;  // exclusive prefix of warp totals
        if (lane == 31) smem[32] = wi;
    }
    __syncthreads();
    *total = smem[32];
    return smem[warp] + inc - v;
}

__device__ __forceinline__ unsigned long long pack_status(unsigned epoch, unsigned flag, uint32_t value) {
    return ((unsigned long long)(epoch & 0x3fffffffu) << 34) | ((unsigned long long)flag << 32) | value;
}

__device__ __forceinline__ void publish_status(unsigned long long* status, int tile, unsigned epoch,
                                               unsigned flag, uint32_t value) {
    // flag and value travel in one 64-bit word, so a single store publishes both atomically.
    atomicExch(status + tile, pack_status(epoch, flag, value));
}

// Exclusive prefix of tile `tile` (> 0) from its predecessors' status words. Called by ONE full
// warp. Returns the prefix; after waiting longer than limit_ns sets *err = 1 and returns 0.
__device__ __forceinline__ uint32_t tile_lookback(const unsigned long long* status, int tile, unsigned epoch,
                                                  unsigned* err, unsigned long long limit_ns) {
    const int lane = threadIdx.x & 31;
    const unsigned ep = epoch & 0x3fffffffu;
    uint32_t prefix = 0;
    int base = tile - 1;
    const unsigned long long t0 = global_ns();
    for (;;) {
        const int idx = base - lane;
        unsigned flag = kStatusPrefix;
        uint32_t value = 0;  // tiles before 0 read as an inclusive prefix of 0
        for (;;) {
            if (idx >= 0) {
                const unsigned long long w = *(volatile const unsigned long long*)(status + idx);
                flag = ((unsigned)(w >> 34) == ep) ? (unsigned)(w >> 32) & 3u : 0u;
                value = (uint32_t)w;
            }
            if (__ballot_sync(kFullMask, flag == 0u) == 0) break;
            // warp-uniform timeout decision (lane 0's clock), so all lanes leave together
            const int late = __shfl_sync(kFullMask, (int)(global_ns() - t0 > limit_ns), 0);
            if (late) {
                if (lane == 0) atomicExch(err, 1u);
                return 0;
            }
            __nanosleep(32);
        }
        const unsigned pmask = __ballot_sync(kFullMask, flag == kStatusPrefix);
        const int stop = pmask ? __ffs(pmask) - 1 : 31;  // lanes 0..stop are summed
        uint32_t part = lane <= stop ? value : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(kFullMask, part, off);
        prefix += part;
        if (pmask) return prefix;
        base -= 32;
    }
}

#endif  // __CUDACC__

}  // namespace wfb
