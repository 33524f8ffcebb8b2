// Batched rendering: many render jobs of uneven size in ONE persistent launch (batch.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <vector>
#include <cuda_runtime.h>
#include "engine.hpp"
#include "wavefront.hpp"

namespace wfb {

struct JobSpec {
    std::shared_ptr<ResidentScene> scene;
    wf::Camera camera;
    int width = 0, height = 0;
    int first_sample = 0;
    int sample_count = 0;
    uint32_t seed = 1234;
    int max_depth = 8;
};

// Per-job device film (and split-mode sample buffer) handed to a batch launch.
struct JobBuffers {
    DevFilm film{};
    float* lbuf = nullptr;
    int chunks = 1;
};

// Launch machinery shared by the batch API and the server: device job table, counters, and the
// arm -- the persistent megakernel (one CUDA graph per launch shape, replayed for every batch) or
// the persistent wavefront over a pool of paths_in_flight slots.
class BatchLauncher {
public:
    BatchLauncher(int max_jobs, const LaunchConfig& cfg);
    ~BatchLauncher();
    BatchLauncher(const BatchLauncher&) = delete;
    BatchLauncher& operator=(const BatchLauncher&) = delete;

    int max_jobs() const { return max_jobs_; }
    const LaunchConfig& config() const { return cfg_; }
    int resident_lanes() const { return resident_lanes_; }  // megakernel lanes or wavefront slots
    // Work units per pixel for a job of `pixels` pixels and `samples` samples.
    int chunks_for(int pixels, int samples) const;
    // Kernels launched by the last launch().
    int last_launches() const { return last_launches_; }
    // Enqueues one launch over `jobs` (their films must hold the sums to add to); jobs are
    // reordered longest-unit-first on the device table only. Returns after enqueueing; it waits
    // only for this launcher's previous table upload (not for earlier launches), so a caller with
    // two launchers can prepare one launch while the other runs.
    void launch(const std::vector<JobSpec>& jobs, const std::vector<JobBuffers>& bufs, bool count_rays,
                cudaStream_t stream);
    // Counters of the last launch (synchronises the stream).
    DevCounters counters(cudaStream_t stream);
    bool graph_used() const { return graph_exec_ != nullptr; }

private:
    int max_jobs_;
    LaunchConfig cfg_;
    int resident_lanes_;  // megakernel lanes or wavefront slots working at once
    int last_launches_ = 0;
    std::unique_ptr<WavefrontEngine> wf_;
    void* arena_ = nullptr;  // header + job table + counters + work counter
    BatchHeader* d_hdr_ = nullptr;
    JobDesc* d_jobs_ = nullptr;
    DevCounters* d_counters_ = nullptr;
    unsigned* d_work_ = nullptr;
    void* h_pinned_ = nullptr;  // staging for header + table
    cudaEvent_t staged_ = nullptr;  // recorded after the last table upload: the staging is free again
    cudaGraphExec_t graph_exec_ = nullptr;
    bool count_rays_in_graph_ = false;
    bool split_in_graph_ = false;  // the captured graph runs the all-split kernel variant
};

// Synchronous batch API (wfb_batch_*): owns the films of its jobs.
class BatchRenderer {
public:
    BatchRenderer(int max_jobs, const LaunchConfig& cfg);
    ~BatchRenderer();
    int add(const JobSpec& job);  // returns the job id
    void clear();
    int size() const { return (int)jobs_.size(); }
    // Zeroes every film, renders all jobs in one launch, waits. Returns device milliseconds.
    double run(bool count_rays, wf::RenderStats* stats);
    void download_sums(int id, float* rgb, float* lum, float* lum2);
    void download(int id, int spp_done, float* rgb, float* lum_var);
    const JobSpec& job(int id) const { return jobs_.at(id); }
    BatchLauncher& launcher() { return launcher_; }

private:
    void alloc_buffers();
    BatchLauncher launcher_;
    std::vector<JobSpec> jobs_;
    std::vector<JobBuffers> bufs_;
    void* films_ = nullptr;
    size_t films_bytes_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
};


}  // namespace wfb
