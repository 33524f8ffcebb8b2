// Render entry point that allocates no device memory (wfb_render_passes_noalloc, include/wfb200.h).
//
// Who needs it: callers that must not call cudaMalloc on their render path -- a host application
// that owns all device memory through its own pool and forbids plugins from allocating, a
// real-time loop where an allocation (which can synchronise the device) would break its frame
// budget, or work issued while a stream is being captured into a CUDA graph, where cudaMalloc is
// not allowed. They allocate the film themselves and hand its device pointers in.
//
// Scratch: the split-mode megakernel needs a work counter, ray counters and one radiance slot per
// (pixel, sample) of the call. Here they live in the file-scope array `g_noalloc_scratch`
// (kNoAllocScratchBytes, about 12 MB), which every GPU that loads this library holds until the
// process exits. Its device address is looked up once per device with cudaGetSymbolAddress (the
// host-side symbol is only a stand-in and must never be passed to a kernel).
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
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device; looked up on the first call per device.
unsigned char* scratch_on_current_device() {
    int dev = -1;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw Error(WFB_ERR_UNSUPPORTED, "device index out of range for the no-alloc scratch table");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
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
    unsigned char* base = scratch_on_current_device();
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
}

}  // namespace wfb
