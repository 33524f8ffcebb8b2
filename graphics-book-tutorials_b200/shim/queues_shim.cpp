// wf::gpu queue primitives over the C ABI: the reference's cudaError_t contract
// (WVM/src/gpu/queues.cu:99-252) on top of wfb_scan_* / wfb_compact_u32 / wfb_test_queue_push.
// Status mapping: WFB_ERR_INVALID_ARGUMENT -> cudaErrorInvalidValue (n < 0 or n > capacity, with
// nothing enqueued, as the reference), WFB_ERR_OUT_OF_MEMORY -> cudaErrorMemoryAllocation,
// anything else -> cudaErrorUnknown (the message stays in wfb_last_error()).
#include "wf_gpu_queues.hpp"
#include "../../include/wfb200.h"

namespace wf::gpu {
namespace {

cudaError_t to_cuda(int status) {
    switch (status) {
        case WFB_OK: return cudaSuccess;
        case WFB_ERR_INVALID_ARGUMENT: return cudaErrorInvalidValue;
        case WFB_ERR_OUT_OF_MEMORY: return cudaErrorMemoryAllocation;
        default: return cudaErrorUnknown;
    }
}

wfb_scan_workspace_t handle(const ScanWorkspace& ws) { return reinterpret_cast<wfb_scan_workspace_t>(ws.block_sums); }

}  // namespace

cudaError_t scan_workspace_create(ScanWorkspace* ws, int capacity) {
    if (ws == nullptr || capacity < 0) return cudaErrorInvalidValue;
    wfb_scan_workspace_t h = nullptr;
    const int st = wfb_scan_workspace_create(capacity, &h);
    if (st != WFB_OK) return to_cuda(st);
    ws->block_sums = reinterpret_cast<uint32_t*>(h);
    ws->capacity = capacity;
    return cudaSuccess;
}

void scan_workspace_destroy(ScanWorkspace* ws) {
    if (ws == nullptr) return;
    if (ws->block_sums != nullptr) wfb_scan_workspace_destroy(handle(*ws));
    ws->block_sums = nullptr;
    ws->capacity = 0;
}

cudaError_t scan_exclusive_u32(const uint32_t* d_in, uint32_t* d_out, int n, uint32_t* d_total, ScanWorkspace& ws,
                               cudaStream_t stream) {
    if (n < 0 || n > ws.capacity) return cudaErrorInvalidValue;
    return to_cuda(wfb_scan_exclusive_u32(d_in, d_out, n, d_total, handle(ws), stream));
}

cudaError_t compact_u32(const uint32_t* d_values, const uint32_t* d_flags, uint32_t* d_out, uint32_t* d_count,
                        uint32_t* d_scratch, int n, ScanWorkspace& ws, cudaStream_t stream) {
    if (n < 0 || n > ws.capacity) return cudaErrorInvalidValue;
    return to_cuda(wfb_compact_u32(d_values, d_flags, d_out, d_count, d_scratch, n, handle(ws), stream));
}

cudaError_t test_queue_push(const uint32_t* d_flags, int n, uint32_t* d_items, uint32_t capacity,
                            uint32_t* d_counter, uint32_t* d_overflow, cudaStream_t stream) {
    return to_cuda(wfb_test_queue_push(d_flags, n, d_items, capacity, d_counter, d_overflow, stream));
}

}  // namespace wf::gpu
