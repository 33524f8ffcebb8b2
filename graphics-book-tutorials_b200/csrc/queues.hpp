// Host side of the stand-alone queue primitives (queues.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <cuda_runtime.h>

namespace wfb {

// Look-back status words for up to `capacity` elements, plus the tile ticket and the error flag.
struct ScanWorkspace {
    void* arena = nullptr;
    unsigned* ticket = nullptr;
    unsigned* err = nullptr;
    unsigned long long* status = nullptr;
    unsigned epoch = 0;
    int capacity = 0;
    size_t bytes = 0;
    ~ScanWorkspace();
};

std::unique_ptr<ScanWorkspace> scan_workspace_create(int capacity);
// Stream-ordered, no host synchronisation. n > capacity throws Error(WFB_ERR_INVALID_ARGUMENT)
// before anything is enqueued.
void scan_exclusive_u32(const uint32_t* in, uint32_t* out, int n, uint32_t* total, ScanWorkspace& ws,
                        cudaStream_t stream);
void compact_u32(const uint32_t* values, const uint32_t* flags, uint32_t* out, uint32_t* count, int n,
                 ScanWorkspace& ws, cudaStream_t stream);
void test_queue_push(const uint32_t* flags, int n, uint32_t* items, uint32_t capacity, uint32_t* counter,
                     uint32_t* overflow, cudaStream_t stream);
// Synchronises `stream` and reports whether a look-back wait gave up since the workspace was made.
bool scan_workspace_failed(ScanWorkspace& ws, cudaStream_t stream);

}  // namespace wfb
