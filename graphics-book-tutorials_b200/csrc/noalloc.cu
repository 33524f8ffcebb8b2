// Render entry point that allocates no device memory (wfb_render_passes_noalloc, include/wfb200.h).
//
// Who needs it: callers that must not call cudaMalloc on their render path -- a host application
// that owns all device memory through its own pool and forbids plugins from allocating, or a
// real-time loop where an allocation (which can synchronise the device) would break its frame
// budget. They allocate the film themselves and hand its device pointers in.
//
// Scratch: the split-mode megakernel needs a work counter, ray counters and one radiance slot per
// (pixel, sample) of the call. Here they live in the file-scope array `g_noalloc_scratch`
// (kNoAllocScratchBytes, about 12 MB), which every GPU that loads this library holds until the
// process exits. The host-side symbol is only a stand-in and must never be passed to a kernel: the
// device address comes from cudaGetSymbolAddress, looked up on the first call in each CUDA context
// (per device, and again if that device's context was reset and created anew) and cached.
#include <mutex>
#include "engine.hpp"
#include "noalloc.hpp"
#include "../../include/wfb200.h"

namespace wfb {
namespace {

constexpr size_t kWorkOffset = 0;         // unsigned int work counter
constexpr size_t kCountersOffset = 256;   // DevCounters
constexpr size_t kSamplesOffset = 512;    // 3 floats per (pixel, sample) slot
constexpr size_t kNoAllocScratchBytes = kSamplesOffset + 3 * sizeof(float) * (size_t)WFB_NOALLOC_MAX_SAMPLES;
static_assert(sizeof(DevCounters) <= kSamplesOffset - kCountersOffset, "counters fit their slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// Per device: the unique id of the context the address was looked up in (0: none yet) and the address.
unsigned long long g_scratch_ctx[kMaxDevices] = {};
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Driver calls that identify the current context (cuCtxGetCurrent, cuCtxGetId: CUDA 12.0+), reached
// through the runtime's entry-point query so the library needs no link against libcuda.
using CtxGetCurrentFn = int (*)(void** ctx);
using CtxGetIdFn = int (*)(void* ctx, unsigned long long* id);
struct CtxQuery {
    CtxGetCurrentFn get_current = nullptr;
    CtxGetIdFn get_id = nullptr;
    CtxQuery() {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        cudaGetLastError();  // a failed query leaves no sticky error behind
    }
};

// Unique id of the calling thread's current context, 0 if the driver cannot say.
unsigned long long current_context_id() {
    static const CtxQuery q;
    if (!q.get_current || !q.get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (q.get_current(&ctx) != 0 || !ctx || q.get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array in the current device's context. Looked up with
// cudaGetSymbolAddress on the first call in each context; a context that was reset and created
// anew (cudaDeviceReset) has a new id, so the stale address is never reused. Where the driver
// cannot identify the context, the address is looked up on every call.
unsigned char* scratch_on_current_device(int dev) {
    if (dev < 0 || dev >= kMaxDevices) throw Error(WFB_ERR_UNSUPPORTED, "device index out of range for the no-alloc scratch table");
    // makes the device's primary context current on this thread (CUDA 12 initialises it here)
    cuda_check(cudaSetDevice(dev), "cudaSetDevice");
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_mu);
    if (ctx == 0 || g_scratch_ctx[dev] != ctx || !g_scratch_addr[dev]) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    return g_scratch_addr[dev];
}

}  // namespace

void render_passes_noalloc(const ResidentScene& scene, int first_sample, int count, uint32_t seed, int max_depth,
                           float* rgb_sum, float* lum_sum, float* lum2_sum, cudaStream_t stream) {
    int dev = -1;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (scene.device != dev)
        throw Error(WFB_ERR_INVALID_ARGUMENT, "scene is not resident on the current device");
    if (first_sample < 0 || count < 0 || max_depth < 0)
        throw Error(WFB_ERR_INVALID_ARGUMENT, "negative sample range or depth");
    if (!rgb_sum || !lum_sum || !lum2_sum) throw Error(WFB_ERR_INVALID_ARGUMENT, "null film pointer");
    const long long pixels = (long long)scene.dev.width * scene.dev.height;
    if (pixels * (long long)count > (long long)WFB_NOALLOC_MAX_SAMPLES)
        throw Error(WFB_ERR_INVALID_ARGUMENT,
                    "pixels * count exceeds WFB_NOALLOC_MAX_SAMPLES (1048576); render in passes of fewer samples");
    if (count == 0) return;
    unsigned char* base = scratch_on_current_device(dev);
    unsigned int* work = reinterpret_cast<unsigned int*>(base + kWorkOffset);
    DevCounters* counters = reinterpret_cast<DevCounters*>(base + kCountersOffset);
    float* samples = reinterpret_cast<float*>(base + kSamplesOffset);
    // The array keeps the previous call's contents: the counters start from zero on every call
    // (the work counter is zeroed by the launcher, the sample slots are all written before read).
    cuda_check(cudaMemsetAsync(counters, 0, sizeof(DevCounters), stream), "clear no-alloc counters");
    DevFilm film;
    film.rgb = rgb_sum;
    film.lum = lum_sum;
    film.lum2 = lum2_sum;
    film.pixels = (int)pixels;
    PassParams p;
    p.first_sample = first_sample;
    p.sample_count = count;
    p.seed = seed;
    p.max_depth = max_depth;
    MegakernelConfig cfg;
    const int chunks = megakernel_split_chunks((int)pixels, count, cfg);
    launch_megakernel(scene.dev, film, counters, work, samples, p, cfg, chunks, stream);
    // The scene's arena is freed (when its last owner lets go) only after this point of `stream`:
    // the caller may destroy the scene as soon as this call returns.
    cuda_check(cudaEventRecord(scene.last_use, stream), "record scene use");
}

}  // namespace wfb
