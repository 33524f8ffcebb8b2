// Host API of the reference's queue primitives (WVM/src/gpu/queues.cuh:29-55), declared with the
// same types and signatures so that callers built against the reference header link against
// libwf_gpu.so. The implementation (queues_shim.cpp) forwards to the engine's single-pass
// decoupled-look-back scan and compaction through the C ABI (include/wfb200.h).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace wf::gpu {

// Same layout as the reference struct. `block_sums` carries the engine's workspace handle (the
// single-pass scan keeps a look-back status array instead of block sums); callers only test it
// against nullptr and hand the struct back, as the reference's callers do.
struct ScanWorkspace {
    uint32_t* block_sums = nullptr;
    int capacity = 0;
};

cudaError_t scan_workspace_create(ScanWorkspace* ws, int capacity);
void scan_workspace_destroy(ScanWorkspace* ws);
cudaError_t scan_exclusive_u32(const uint32_t* d_in, uint32_t* d_out, int n, uint32_t* d_total, ScanWorkspace& ws,
                               cudaStream_t stream);
cudaError_t compact_u32(const uint32_t* d_values, const uint32_t* d_flags, uint32_t* d_out, uint32_t* d_count,
                        uint32_t* d_scratch, int n, ScanWorkspace& ws, cudaStream_t stream);
cudaError_t test_queue_push(const uint32_t* d_flags, int n, uint32_t* d_items, uint32_t capacity,
                            uint32_t* d_counter, uint32_t* d_overflow, cudaStream_t stream);

}  // namespace wf::gpu
