// Stand-alone queue primitives behind the C ABI (include/wfb200.h), replacing the reference's
// scan_workspace_create / scan_exclusive_u32 / compact_u32 / test_queue_push
// (WVM/src/gpu/queues.cuh:30-55, WVM/src/gpu/queues.cu:99-252) with single-pass kernels:
//   scan     one launch, one read and one write per element (decoupled look-back), in-place safe;
//   compact  one launch: flags -> tile scan -> stable scatter (no indicator array, no second pass).
// Tiles are claimed through an atomic ticket, so a tile only ever waits on tiles claimed before
// it by CTAs that are already running: the look-back always makes progress.
#include <atomic>
#include <cstring>
#include "engine.hpp"
#include "queues.cuh"
#include "queues.hpp"
#include "../../include/wfb200.h"

namespace wfb {
namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

// MODE 0: exclusive scan of in[] into out[] (in may equal out), *total = sum.
// MODE 1: stable compaction: out[k] = values[i] for the k-th i with flags[i] != 0, *total = count.
template <int MODE>
__global__ void __launch_bounds__(kScanBlock) scan_tiles(const uint32_t* in, const uint32_t* values, uint32_t* out,
                                                         int n, uint32_t* total, unsigned long long* status,
                                                         unsigned* ticket, unsigned epoch, unsigned* err,
                                                         unsigned long long wait_ns) {
    __shared__ uint32_t smem[33];
    __shared__ int s_tile;
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    const long long base = (long long)tile * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + k;
        uint32_t x = 0;
        if (i < n) x = MODE == 0 ? in[i] : (in[i] != 0u ? 1u : 0u);  // read before any write: in-place safe
        v[k] = x;
        local += x;
    }
    uint32_t aggregate;
    const uint32_t excl = block_exclusive_sum(local, smem, &aggregate);
    if (threadIdx.x == 0) {
        if (tile == 0) publish_status(status, 0, epoch, kStatusPrefix, aggregate);
        else publish_status(status, tile, epoch, kStatusAggregate, aggregate);
    }
    if (tile > 0 && threadIdx.x < 32) {
        const uint32_t p = tile_lookback(status, tile, epoch, err, wait_ns);
        if (threadIdx.x == 0) {
            publish_status(status, tile, epoch, kStatusPrefix, p + aggregate);
            s_prefix = p;
        }
    } else if (tile == 0 && threadIdx.x == 0) {
        s_prefix = 0;
    }
    __syncthreads();
    uint32_t run = s_prefix + excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + k;
        if (i < n) {
            if (MODE == 0) out[i] = run;
            else if (v[k]) out[run] = values[i];
        }
        run += v[k];
    }
    if (total && (long long)(tile + 1) * kScanTile >= n && threadIdx.x == kScanBlock - 1) *total = run;
}

__global__ void queue_push_test_kernel(const uint32_t* flags, int n, uint32_t* items, uint32_t capacity,
                                       uint32_t* counter, uint32_t* overflow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool pred = i < n && flags[i] != 0u;
    queue_push(items, counter, capacity, (uint32_t)i, pred, overflow);
}

int tiles_for(int n) { return (n + kScanTile - 1) / kScanTile; }

std::atomic<unsigned long long> g_wait_limit_ns{kDefaultWaitLimitNs};
std::atomic<bool> g_unsatisfiable_next{false};

// Tile tickets start at 0; a test that asked for an unsatisfiable wait starts them at 1, so no CTA
// claims tile 0 and every look-back waits for a prefix that nothing publishes.
void start_tickets(ScanWorkspace& ws, cudaStream_t stream) {
    if (take_unsatisfiable_wait()) {
        static const unsigned one = 1u;
        cuda_check(cudaMemcpyAsync(ws.ticket, &one, sizeof(unsigned), cudaMemcpyHostToDevice, stream), "set ticket");
        cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");  // `one` is read before returning
    } else {
        cuda_check(cudaMemsetAsync(ws.ticket, 0, sizeof(unsigned), stream), "memset ticket");
    }
}

}  // namespace

uint64_t device_wait_limit_ns() { return g_wait_limit_ns.load(); }

void set_device_wait_test(uint64_t limit_ns, bool unsatisfiable_next) {
    g_wait_limit_ns.store(limit_ns ? limit_ns : kDefaultWaitLimitNs);
    g_unsatisfiable_next.store(unsatisfiable_next);
}

bool take_unsatisfiable_wait() { return g_unsatisfiable_next.exchange(false); }

ScanWorkspace::~ScanWorkspace() {
    if (arena) cudaFree(arena);
}

std::unique_ptr<ScanWorkspace> scan_workspace_create(int capacity) {
    if (capacity <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "scan workspace capacity must be positive");
    auto ws = std::make_unique<ScanWorkspace>();
    const size_t tiles = (size_t)tiles_for(capacity) + 1;
    const size_t bytes = 256 + tiles * sizeof(unsigned long long);
    cuda_check(cudaMalloc(&ws->arena, bytes), "cudaMalloc scan workspace");
    cuda_check(cudaMemset(ws->arena, 0, bytes), "cudaMemset scan workspace");
    ws->ticket = static_cast<unsigned*>(ws->arena);
    ws->err = ws->ticket + 1;
    ws->status = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws->arena) + 256);
    ws->capacity = capacity;
    ws->bytes = bytes;
    return ws;
}

void scan_exclusive_u32(const uint32_t* in, uint32_t* out, int n, uint32_t* total, ScanWorkspace& ws,
                        cudaStream_t stream) {
    if (n < 0 || n > ws.capacity) throw Error(WFB_ERR_INVALID_ARGUMENT, "scan size exceeds the workspace capacity");
    if (n == 0) {
        if (total) cuda_check(cudaMemsetAsync(total, 0, sizeof(uint32_t), stream), "memset total");
        return;
    }
    start_tickets(ws, stream);
    const unsigned epoch = ++ws.epoch;
    scan_tiles<0><<<tiles_for(n), kScanBlock, 0, stream>>>(in, nullptr, out, n, total, ws.status, ws.ticket, epoch,
                                                           ws.err, device_wait_limit_ns());
    cuda_check(cudaGetLastError(), "scan launch");
}

void compact_u32(const uint32_t* values, const uint32_t* flags, uint32_t* out, uint32_t* count, int n,
                 ScanWorkspace& ws, cudaStream_t stream) {
    if (n < 0 || n > ws.capacity) throw Error(WFB_ERR_INVALID_ARGUMENT, "compaction size exceeds the workspace capacity");
    if (n == 0) {
        if (count) cuda_check(cudaMemsetAsync(count, 0, sizeof(uint32_t), stream), "memset count");
        return;
    }
    start_tickets(ws, stream);
    const unsigned epoch = ++ws.epoch;
    scan_tiles<1><<<tiles_for(n), kScanBlock, 0, stream>>>(flags, values, out, n, count, ws.status, ws.ticket, epoch,
                                                           ws.err, device_wait_limit_ns());
    cuda_check(cudaGetLastError(), "compact launch");
}

void test_queue_push(const uint32_t* flags, int n, uint32_t* items, uint32_t capacity, uint32_t* counter,
                     uint32_t* overflow, cudaStream_t stream) {
    if (n < 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "negative size");
    if (n == 0) return;
    queue_push_test_kernel<<<(n + 255) / 256, 256, 0, stream>>>(flags, n, items, capacity, counter, overflow);
    cuda_check(cudaGetLastError(), "queue push launch");
}

bool scan_workspace_failed(ScanWorkspace& ws, cudaStream_t stream) {
    unsigned e = 0;
    cuda_check(cudaMemcpyAsync(&e, ws.err, sizeof(e), cudaMemcpyDeviceToHost, stream), "read scan error flag");
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    return e != 0;
}

}  // namespace wfb
