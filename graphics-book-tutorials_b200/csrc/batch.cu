// Batched rendering: many jobs of uneven size (scene, camera, resolution, spp, depth, seed) in one
// persistent launch of either arm: the megakernel (replayed through a CUDA graph captured once per
// launch shape) or the wavefront (paths of all jobs in one pool; each slot carries its job id).
//
// Every job renders exactly the bits it renders alone: pixel ids and RNG keys are job-local,
// and a pixel's samples are added in ascending order whatever the batch (see megakernel.cu).
// The reference has no counterpart (one scene, one camera, one job per GpuRenderer).
#include <algorithm>
#include <cstring>
#include <numeric>
#include "batch.hpp"
#include "../../include/wfb200.h"

namespace wfb {

// ---------------------------------------------------------------------------------------------
BatchLauncher::BatchLauncher(int max_jobs, const LaunchConfig& cfg) : max_jobs_(max_jobs), cfg_(cfg) {
    if (max_jobs <= 0 || max_jobs > 65535) throw Error(WFB_ERR_INVALID_ARGUMENT, "max_jobs must be in 1..65535");
    if (cfg_.mode == wf::GpuMode::Wavefront) {
        wf_ = std::make_unique<WavefrontEngine>(1 << 24, cfg_.wf);  // pool sized by paths_in_flight alone
        resident_lanes_ = wf_->capacity();
    } else {
        resident_lanes_ = megakernel_resident_threads(cfg_.mk);
    }
    const size_t table = sizeof(BatchHeader) + (size_t)max_jobs * sizeof(JobDesc);
    const size_t bytes = table + 256 + sizeof(DevCounters) + 256;
    cuda_check(cudaMalloc(&arena_, bytes), "cudaMalloc batch table");
    char* p = static_cast<char*>(arena_);
    d_hdr_ = reinterpret_cast<BatchHeader*>(p);
    d_jobs_ = reinterpret_cast<JobDesc*>(p + sizeof(BatchHeader));
    d_counters_ = reinterpret_cast<DevCounters*>(p + ((table + 255) & ~(size_t)255));
    d_work_ = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(d_counters_) + 256);
    cuda_check(cudaMallocHost(&h_pinned_, table), "cudaMallocHost batch staging");
    cuda_check(cudaEventCreateWithFlags(&staged_, cudaEventDisableTiming), "cudaEventCreate");
}

BatchLauncher::~BatchLauncher() {
    if (staged_) cudaEventDestroy(staged_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (h_pinned_) cudaFreeHost(h_pinned_);
    if (arena_) cudaFree(arena_);
}

int BatchLauncher::chunks_for(int pixels, int samples) const {
    // Megakernel: the single-render rule (one sample per unit while the job's buffer fits).
    if (!wf_) return megakernel_split_chunks(pixels, samples, cfg_.mk);
    // Wavefront: one sample per unit while the job's buffer fits, else split a job's samples only
    // when its pixels alone cannot fill the pool.
    if (samples <= 1) return 1;
    if (split_buffer_bytes(pixels, samples) <= kSplitBufferBytes) return samples;
    if (pixels >= resident_lanes_) return 1;
    const long long k = ((long long)resident_lanes_ + pixels - 1) / pixels;
    return (int)std::min<long long>(k, samples);
}

void BatchLauncher::launch(const std::vector<JobSpec>& jobs, const std::vector<JobBuffers>& bufs, bool count_rays,
                           cudaStream_t stream) {
    const int n = (int)jobs.size();
    if (n > max_jobs_) throw Error(WFB_ERR_INVALID_ARGUMENT, "more jobs than the batch holds");
    if (bufs.size() != jobs.size()) throw Error(WFB_ERR_INTERNAL, "job buffers do not match the jobs");
    // The staging buffer may still feed this launcher's previous table upload.
    cuda_check(cudaEventSynchronize(staged_), "wait for the previous table upload");
    std::vector<JobDesc> desc((size_t)n);
    for (int i = 0; i < n; ++i) {
        const JobSpec& j = jobs[i];
        if (!j.scene) throw Error(WFB_ERR_INVALID_ARGUMENT, "job without a scene");
        const DevScene view = with_camera(j.scene->dev, j.camera, j.width, j.height);
        desc[i] = make_job(view, bufs[i].film, bufs[i].lbuf, j.first_sample, j.sample_count, bufs[i].chunks, j.seed,
                           j.max_depth);
    }
    // Longest units first: they start early and the short ones fill the tail. Among equal unit
    // lengths, jobs of one scene run together (scenes in order of first appearance), so the L2
    // holds one scene's BVH at a time instead of every scene's at once.
    std::vector<int> order((size_t)n), group((size_t)n);
    for (int i = 0; i < n; ++i) {
        group[i] = i;
        for (int k = 0; k < i; ++k)
            if (desc[k].s.nodes == desc[i].s.nodes) {
                group[i] = group[k];
                break;
            }
    }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (desc[x].chunk != desc[y].chunk) return desc[x].chunk > desc[y].chunk;
        return group[x] < group[y];
    });
    BatchHeader* hdr = static_cast<BatchHeader*>(h_pinned_);
    JobDesc* table = reinterpret_cast<JobDesc*>(static_cast<char*>(h_pinned_) + sizeof(BatchHeader));
    unsigned long long units = 0;
    for (int k = 0; k < n; ++k) {
        JobDesc d = desc[order[k]];
        d.unit_begin = (unsigned)units;
        units += d.units;
        table[k] = d;
    }
    if (units >= 0xFFFFFFFFull) throw Error(WFB_ERR_UNSUPPORTED, "batch has more than 2^32 work units");
    std::memset(hdr, 0, sizeof(BatchHeader));
    hdr->n_jobs = (unsigned)n;
    hdr->total_units = (unsigned)units;
    cuda_check(cudaMemcpyAsync(d_hdr_, h_pinned_, sizeof(BatchHeader) + (size_t)n * sizeof(JobDesc),
                               cudaMemcpyHostToDevice, stream),
               "upload job table");
    cuda_check(cudaEventRecord(staged_, stream), "cudaEventRecord");
    cuda_check(cudaMemsetAsync(d_counters_, 0, sizeof(DevCounters), stream), "zero counters");
    if (wf_) {
        last_launches_ = wf_->run_batch(d_jobs_, d_hdr_, d_counters_, count_rays, stream);
        launch_film_commit_jobs(d_jobs_, d_hdr_, max_jobs_, stream);
        ++last_launches_;
        return;
    }
    last_launches_ = 2;  // persistent megakernel + film commits
    bool all_split = n > 0;
    for (int i = 0; i < n; ++i) all_split = all_split && desc[i].chunks > 1;
    if (!cfg_.use_graph) {
        launch_megakernel_batch(d_jobs_, d_hdr_, max_jobs_, d_counters_, d_work_, count_rays, cfg_.mk, all_split,
                                stream);
        return;
    }
    if (graph_exec_ && (count_rays_in_graph_ != count_rays || split_in_graph_ != all_split)) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (!graph_exec_) {
        cudaGraph_t graph = nullptr;
        cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            launch_megakernel_batch(d_jobs_, d_hdr_, max_jobs_, d_counters_, d_work_, count_rays, cfg_.mk, all_split,
                                    stream);
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        cuda_check(cudaStreamEndCapture(stream, &graph), "end capture");
        const cudaError_t e = cudaGraphInstantiate(&graph_exec_, graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "instantiate batch graph");
        count_rays_in_graph_ = count_rays;
        split_in_graph_ = all_split;
    }
    cuda_check(cudaGraphLaunch(graph_exec_, stream), "launch batch graph");
}

DevCounters BatchLauncher::counters(cudaStream_t stream) {
    DevCounters c{};
    cuda_check(cudaMemcpyAsync(&c, d_counters_, sizeof(c), cudaMemcpyDeviceToHost, stream), "download counters");
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    return c;
}

// ---------------------------------------------------------------------------------------------
BatchRenderer::BatchRenderer(int max_jobs, const LaunchConfig& cfg) : launcher_(max_jobs, cfg) {
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaEventCreate(&ev0_), "cudaEventCreate");
    cuda_check(cudaEventCreate(&ev1_), "cudaEventCreate");
}

BatchRenderer::~BatchRenderer() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (films_) cudaFree(films_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

int BatchRenderer::add(const JobSpec& job) {
    if ((int)jobs_.size() >= launcher_.max_jobs()) throw Error(WFB_ERR_INVALID_ARGUMENT, "batch is full");
    if (!job.scene) throw Error(WFB_ERR_INVALID_ARGUMENT, "job without a scene");
    if (job.width <= 0 || job.height <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "resolution must be positive");
    if (job.sample_count <= 0 || job.first_sample < 0 || job.max_depth < 0)
        throw Error(WFB_ERR_INVALID_ARGUMENT, "bad sample range or depth");
    jobs_.push_back(job);
    bufs_.clear();
    return (int)jobs_.size() - 1;
}

void BatchRenderer::clear() {
    jobs_.clear();
    bufs_.clear();
}

void BatchRenderer::alloc_buffers() {
    bufs_.assign(jobs_.size(), JobBuffers{});
    size_t total = 0;
    std::vector<size_t> film_off(jobs_.size()), lbuf_off(jobs_.size());
    for (size_t i = 0; i < jobs_.size(); ++i) {
        const size_t p = (size_t)jobs_[i].width * jobs_[i].height;
        bufs_[i].chunks = launcher_.chunks_for((int)p, jobs_[i].sample_count);
        film_off[i] = total;
        total += (5 * p * sizeof(float) + 255) & ~(size_t)255;
        lbuf_off[i] = total;
        if (bufs_[i].chunks > 1) total += (3 * p * (size_t)jobs_[i].sample_count * sizeof(float) + 255) & ~(size_t)255;
    }
    if (total > films_bytes_) {
        if (films_) cudaFree(films_);
        films_ = nullptr;
        films_bytes_ = 0;
        cuda_check(cudaMalloc(&films_, total), "cudaMalloc batch films");
        films_bytes_ = total;
    }
    char* base = static_cast<char*>(films_);
    for (size_t i = 0; i < jobs_.size(); ++i) {
        const size_t p = (size_t)jobs_[i].width * jobs_[i].height;
        float* f = reinterpret_cast<float*>(base + film_off[i]);
        bufs_[i].film = DevFilm{f, f + 3 * p, f + 4 * p, (int)p};
        bufs_[i].lbuf = bufs_[i].chunks > 1 ? reinterpret_cast<float*>(base + lbuf_off[i]) : nullptr;
    }
}

double BatchRenderer::run(bool count_rays, wf::RenderStats* stats) {
    if (jobs_.empty()) return 0.0;
    alloc_buffers();
    for (const JobBuffers& b : bufs_)
        cuda_check(cudaMemsetAsync(b.film.rgb, 0, 5 * (size_t)b.film.pixels * sizeof(float), stream_), "zero film");
    cuda_check(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    launcher_.launch(jobs_, bufs_, count_rays, stream_);
    cuda_check(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(ev1_), "batch render");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    const DevCounters c = launcher_.counters(stream_);
    if (stats) {
        stats->render_ms = ms;
        stats->extension_rays += c.extension_rays;
        stats->shadow_rays += c.shadow_rays;
        stats->invalid_hits += c.invalid_hits;
        uint64_t bytes = films_bytes_;
        stats->peak_vram_bytes = bytes;
    }
    return ms;
}

void BatchRenderer::download_sums(int id, float* rgb, float* lum, float* lum2) {
    if (id < 0 || id >= (int)bufs_.size()) throw Error(WFB_ERR_INVALID_ARGUMENT, "no such job (or batch not run)");
    const DevFilm& f = bufs_[id].film;
    const size_t p = (size_t)f.pixels;
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    if (rgb) cuda_check(cudaMemcpy(rgb, f.rgb, 3 * p * sizeof(float), cudaMemcpyDeviceToHost), "download rgb");
    if (lum) cuda_check(cudaMemcpy(lum, f.lum, p * sizeof(float), cudaMemcpyDeviceToHost), "download lum");
    if (lum2) cuda_check(cudaMemcpy(lum2, f.lum2, p * sizeof(float), cudaMemcpyDeviceToHost), "download lum2");
}

void BatchRenderer::download(int id, int spp_done, float* rgb, float* lum_var) {
    if (id < 0 || id >= (int)bufs_.size()) throw Error(WFB_ERR_INVALID_ARGUMENT, "no such job (or batch not run)");
    film_download(bufs_[id].film, spp_done, rgb, lum_var, stream_);
}

}  // namespace wfb
