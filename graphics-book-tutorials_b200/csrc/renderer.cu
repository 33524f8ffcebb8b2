// GPU renderer: one resident scene, one camera, one film (the wf::GpuRenderer contract,
// WVM/src/gpu/gpu_renderer.cu:100-377) on this engine's kernels.
#include <algorithm>
#include <cstring>
#include <vector>
#include "engine.hpp"
#include "wavefront.hpp"
#include "../../include/wfb200.h"

namespace wfb {

namespace {

// Film and sample buffers come from the device's stream-ordered pool, which keeps up to this many
// freed bytes for reuse: creating a renderer per frame (or per scene) then costs no device
// allocation after the first, where cudaMalloc of a 700 MB sample buffer takes milliseconds.
constexpr uint64_t kPoolKeepBytes = 8ull << 30;

void keep_pool_memory() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
    uint64_t keep = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) return;
    if (keep < kPoolKeepBytes) {
        keep = kPoolKeepBytes;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
}

// Reference download convention on the device (WVM/src/gpu/gpu_renderer.cu:306-337): mean rgb =
// sum * (1 / spp) in float; luminance variance = max(0, E[l^2] - E[l]^2) in double, narrowed to
// float. The same IEEE operations in the same order as the reference's host loops (this file is
// built without contraction), so the downloaded films are bit-identical; only the resolved film
// crosses PCIe.
__global__ void film_resolve(DevFilm film, int spp, float* __restrict__ rgb, float* __restrict__ lum_var) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= film.pixels) return;
    if (rgb) {
        const float inv = 1.0f / (float)spp;
        rgb[3 * p] = film.rgb[3 * p] * inv;
        rgb[3 * p + 1] = film.rgb[3 * p + 1] * inv;
        rgb[3 * p + 2] = film.rgb[3 * p + 2] * inv;
    }
    if (lum_var) {
        const double m = (double)film.lum[p] / (double)spp;
        const double m2 = (double)film.lum2[p] / (double)spp;
        const double var = m2 - m * m;
        lum_var[p] = (float)(0.0 < var ? var : 0.0);  // std::max(0.0, var)
    }
}

}  // namespace

struct Renderer::Wavefront {
    WavefrontConfig cfg;
    WavefrontEngine engine;
    Wavefront(int pixels, const WavefrontConfig& c) : cfg(c), engine(pixels, c) {}
};

Renderer::Renderer(std::shared_ptr<ResidentScene> scene, wf::GpuMode mode)
    : scene_(std::move(scene)), mode_(mode) {
    if (!scene_) throw Error(WFB_ERR_INVALID_ARGUMENT, "null scene");
    view_ = scene_->dev;
    width_ = view_.width;
    height_ = view_.height;
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaEventCreate(&ev0_), "cudaEventCreate");
    cuda_check(cudaEventCreate(&ev1_), "cudaEventCreate");
    keep_pool_memory();
    // Counters and the work counter share one block from the stream-ordered pool.
    const size_t cbytes = (sizeof(DevCounters) + 255) & ~(size_t)255;
    char* block = nullptr;
    cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&block), cbytes + 256, stream_), "allocate counters");
    counters_ = reinterpret_cast<DevCounters*>(block);
    work_ = reinterpret_cast<unsigned int*>(block + cbytes);
    alloc_film();
}

Renderer::~Renderer() {
    free_film();
    wf_.reset();
    if (counters_) cudaFreeAsync(counters_, stream_);  // work_ is part of the same block
    if (lbuf_) cudaFreeAsync(lbuf_, stream_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Renderer::alloc_film() {
    const size_t p = (size_t)width_ * height_;
    float* base = nullptr;
    cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&base), 5 * p * sizeof(float), stream_), "allocate film");
    film_.rgb = base;
    film_.lum = base + 3 * p;
    film_.lum2 = base + 4 * p;
    film_.pixels = (int)p;
    cuda_check(cudaMemsetAsync(base, 0, 5 * p * sizeof(float), stream_), "zero film");
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    if (mode_ == wf::GpuMode::Wavefront) wf_ = std::make_unique<Wavefront>((int)p, wf_cfg_);
}

void Renderer::free_film() {
    if (film_.rgb) cudaFreeAsync(film_.rgb, stream_);
    film_ = DevFilm{};
    wf_.reset();
}

void Renderer::set_camera(const wf::Camera& cam, int width, int height) {
    if (width <= 0 || height <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "resolution must be positive");
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    view_ = with_camera(scene_->dev, cam, width, height);
    if (width != width_ || height != height_) {
        free_film();
        width_ = width;
        height_ = height;
        alloc_film();
    } else {
        reset();
    }
}

void Renderer::reset() {
    cuda_check(cudaMemsetAsync(film_.rgb, 0, 5 * (size_t)pixels() * sizeof(float), stream_), "cudaMemset film");
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

void Renderer::run_passes(const PassParams& p, wf::RenderStats* stats) {
    if (p.sample_count < 0 || p.first_sample < 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "negative sample range");
    if (p.max_depth < 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "max_depth must be >= 0");
    cuda_check(cudaMemsetAsync(counters_, 0, sizeof(DevCounters), stream_), "zero counters");
    // Automatic splitting: a megakernel render whose per-sample buffer would pass the cap runs as
    // consecutive sub-passes of sample ranges; each pixel still gets its samples in ascending order,
    // so the film is the same. The sample buffer is sized for the largest sub-pass before the
    // timed region starts.
    int step = p.sample_count;
    if (mode_ == wf::GpuMode::Megakernel) {
        if (mk_cfg_.split_chunks == 0 && p.sample_count > 1 &&
            split_buffer_bytes(pixels(), p.sample_count) > kSplitBufferBytes)
            step = (int)std::max<uint64_t>(1, kSplitBufferBytes / split_buffer_bytes(pixels(), 1));
        const int first = std::min(step, p.sample_count);
        if (first > 0 && megakernel_split_chunks(pixels(), first, mk_cfg_) > 1) {
            const size_t need = 3 * (size_t)pixels() * (size_t)first;
            if (need > lbuf_floats_) {
                if (lbuf_) cudaFreeAsync(lbuf_, stream_);
                lbuf_ = nullptr;
                lbuf_floats_ = 0;
                cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&lbuf_), need * sizeof(float), stream_),
                           "allocate sample buffer");
                lbuf_floats_ = need;
            }
        }
    }
    if (mode_ == wf::GpuMode::Wavefront) wf_->engine.reserve(pixels(), p.sample_count);
    ktimer_.reset();
    cuda_check(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    if (mode_ == wf::GpuMode::Megakernel) {
        last_launches_ = 0;
        for (int done = 0; done < p.sample_count; done += step) {
            PassParams q = p;
            q.first_sample = p.first_sample + done;
            q.sample_count = std::min(step, p.sample_count - done);
            const int chunks = megakernel_split_chunks(pixels(), q.sample_count, mk_cfg_);
            if (chunks > 1 && 3 * (size_t)pixels() * (size_t)q.sample_count > lbuf_floats_)
                throw Error(WFB_ERR_INTERNAL, "sample buffer smaller than a sub-pass");
            last_launches_ +=
                launch_megakernel(view_, film_, counters_, work_, lbuf_, q, mk_cfg_, chunks, stream_, &ktimer_);
        }
    } else {
        last_launches_ =
            wf_->engine.run(view_, film_, counters_, p, stats ? &stats->stages : nullptr, stream_, &ktimer_);
    }
    cuda_check(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(ev1_), "render");
    DevCounters c{};
    cuda_check(cudaMemcpy(&c, counters_, sizeof(c), cudaMemcpyDeviceToHost), "download counters");
    if (c.error != kErrNone)
        throw Error(WFB_ERR_DEVICE_WAIT, "a bounded device-side wait gave up; the render is incomplete");
    last_kernel_ms_ = ktimer_.total_ms();
    last_node_visits_ = c.node_visits;
    last_prim_tests_ = c.prim_tests;
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0_, ev1_);
        stats->render_ms = ms;
        stats->extension_rays += c.extension_rays;
        stats->shadow_rays += c.shadow_rays;
        stats->invalid_hits += c.invalid_hits;
        stats->queue_overflows += c.overflows;
        for (int i = 0; i < 5; ++i)
            stats->queue_high_water[i] = std::max(stats->queue_high_water[i], (long long)c.high_water[i]);
        stats->peak_vram_bytes = device_bytes();
    }
}

void Renderer::download_sums(float* rgb_sum, float* lum_sum, float* lum2_sum) {
    const size_t p = (size_t)pixels();
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    if (rgb_sum) cuda_check(cudaMemcpy(rgb_sum, film_.rgb, 3 * p * sizeof(float), cudaMemcpyDeviceToHost), "download rgb");
    if (lum_sum) cuda_check(cudaMemcpy(lum_sum, film_.lum, p * sizeof(float), cudaMemcpyDeviceToHost), "download lum");
    if (lum2_sum) cuda_check(cudaMemcpy(lum2_sum, film_.lum2, p * sizeof(float), cudaMemcpyDeviceToHost), "download lum2");
}

void film_download(const DevFilm& film, int spp_done, float* rgb, float* lum_var, cudaStream_t stream) {
    if (spp_done <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "spp_done must be positive");
    if (!rgb && !lum_var) return;
    const cudaStream_t s = stream ? stream : cudaStreamPerThread;
    const size_t p = (size_t)film.pixels;
    float* out = nullptr;
    cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&out), 4 * p * sizeof(float), s), "allocate download");
    (void)cudaGetLastError();  // the check below is for this launch only, not an earlier unchecked call
    film_resolve<<<(unsigned)((p + 255) / 256), 256, 0, s>>>(film, spp_done, rgb ? out : nullptr,
                                                              lum_var ? out + 3 * p : nullptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && rgb) e = cudaMemcpyAsync(rgb, out, 3 * p * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && lum_var)
        e = cudaMemcpyAsync(lum_var, out + 3 * p, p * sizeof(float), cudaMemcpyDeviceToHost, s);
    const cudaError_t ef = cudaFreeAsync(out, s);
    const cudaError_t es = cudaStreamSynchronize(s);
    cuda_check(e, "download film");
    cuda_check(ef, "free download");
    cuda_check(es, "cudaStreamSynchronize");
}

void film_download_host(const DevFilm& film, int spp_done, float* rgb, float* lum_var, cudaStream_t stream,
                        PinnedStaging* staging) {
    if (spp_done <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "spp_done must be positive");
    const size_t p = (size_t)film.pixels;
    const bool contiguous = film.lum == film.rgb + 3 * p && film.lum2 == film.rgb + 4 * p;
    const float *h_rgb = nullptr, *h_lum = nullptr, *h_lum2 = nullptr;
    std::vector<float> lum, lum2;
    if (staging && contiguous) {
        // the whole film in one copy into reused pinned memory: full copy-engine bandwidth and no
        // page faults, where pageable destinations are staged by the driver a piece at a time
        const size_t bytes = 5 * p * sizeof(float);
        if (staging->bytes < bytes) {
            if (staging->ptr) cudaFreeHost(staging->ptr);
            staging->ptr = nullptr;
            staging->bytes = 0;
            cuda_check(cudaHostAlloc(&staging->ptr, bytes, cudaHostAllocDefault), "cudaHostAlloc download staging");
            staging->bytes = bytes;
        }
        cuda_check(cudaMemcpyAsync(staging->ptr, film.rgb, bytes, cudaMemcpyDeviceToHost, stream), "download film");
        const float* f = static_cast<const float*>(staging->ptr);
        h_rgb = f;
        h_lum = f + 3 * p;
        h_lum2 = f + 4 * p;
    } else {
        if (rgb) cuda_check(cudaMemcpyAsync(rgb, film.rgb, 3 * p * sizeof(float), cudaMemcpyDeviceToHost, stream), "download rgb");
        if (lum_var) {
            lum.resize(p);
            lum2.resize(p);
            cuda_check(cudaMemcpyAsync(lum.data(), film.lum, p * sizeof(float), cudaMemcpyDeviceToHost, stream), "download lum");
            cuda_check(cudaMemcpyAsync(lum2.data(), film.lum2, p * sizeof(float), cudaMemcpyDeviceToHost, stream),
                       "download lum2");
        }
        h_rgb = rgb;
        h_lum = lum.data();
        h_lum2 = lum2.data();
    }
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    // The reference's host loops (WVM/src/gpu/gpu_renderer.cu:319-336), as film_resolve does them.
    const float inv = 1.0f / (float)spp_done;
    if (rgb)
        for (size_t i = 0; i < 3 * p; ++i) rgb[i] = h_rgb[i] * inv;
    if (lum_var)
        for (size_t i = 0; i < p; ++i) {
            const double m = (double)h_lum[i] / (double)spp_done;
            const double m2 = (double)h_lum2[i] / (double)spp_done;
            lum_var[i] = (float)std::max(0.0, m2 - m * m);
        }
}

void Renderer::download(int spp_done, float* rgb, float* lum_var) { film_download(film_, spp_done, rgb, lum_var, stream_); }

void Renderer::download_mean(int spp_done, float* rgb) { download(spp_done, rgb, nullptr); }

void Renderer::configure(int block, int blocks_per_sm, int min_active, int split_chunks, int paths_in_flight,
                         int occupancy, int leaf_batch) {
    if (block > 0) mk_cfg_.block = block;
    if (blocks_per_sm >= 0) mk_cfg_.blocks_per_sm = blocks_per_sm;
    if (min_active > 0) mk_cfg_.min_active = min_active;
    if (split_chunks >= 0) mk_cfg_.split_chunks = split_chunks;
    if (occupancy >= 0) mk_cfg_.occupancy = occupancy;
    if (leaf_batch > 0) mk_cfg_.leaf_batch = leaf_batch;
    if (mode_ == wf::GpuMode::Wavefront && (paths_in_flight > 0 || min_active > 0 || leaf_batch > 0 || occupancy >= 0)) {
        if (paths_in_flight > 0) wf_cfg_.paths_in_flight = paths_in_flight;
        if (occupancy >= 0) wf_cfg_.occupancy = occupancy;
        if (min_active > 0) wf_cfg_.min_active = min_active;
        if (leaf_batch > 0) wf_cfg_.leaf_batch = leaf_batch;
        cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
        wf_.reset();
        wf_ = std::make_unique<Wavefront>(pixels(), wf_cfg_);
    }
}

void Renderer::set_l2_residency(int mode) {
    wf_cfg_.l2_persist = mode < 0 ? -1 : (mode > 0 ? 1 : 0);
    if (mode_ != wf::GpuMode::Wavefront) return;
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    wf_.reset();
    wf_ = std::make_unique<Wavefront>(pixels(), wf_cfg_);
}

void Renderer::set_speculation(bool on) {
    mk_cfg_.speculate = on;
    wf_cfg_.speculate = on;
    if (wf_) wf_->engine.set_speculate(on);
}

uint64_t Renderer::l2_window_bytes() const { return wf_ ? wf_->engine.l2_window_bytes() : 0; }

uint64_t Renderer::device_bytes() const {
    uint64_t b = scene_->bytes + 5ull * pixels() * sizeof(float) + sizeof(DevCounters);
    if (wf_) b += wf_->engine.bytes();
    return b;
}

}  // namespace wfb
