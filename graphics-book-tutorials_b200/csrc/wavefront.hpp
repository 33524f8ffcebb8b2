// Persistent-threads wavefront engine (wavefront.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <cuda_runtime.h>
#include "engine.hpp"

namespace wfb {

class WavefrontEngine {
public:
    explicit WavefrontEngine(int pixels, const WavefrontConfig& cfg = WavefrontConfig{});
    ~WavefrontEngine();
    WavefrontEngine(const WavefrontEngine&) = delete;
    WavefrontEngine& operator=(const WavefrontEngine&) = delete;

    // Adds samples [p.first_sample, p.first_sample + p.sample_count) of every pixel to `film`;
    // returns the number of kernels launched.
    int run(const DevScene& s, const DevFilm& film, DevCounters* counters, const PassParams& p,
             wf::StageTimes* stages, cudaStream_t stream, KernelTimer* timer = nullptr);
    // Sizes the per-sample buffer that run() needs for this many pixels and samples (run() calls
    // it too; a caller that times run() calls it first, outside the timed region).
    void reserve(int pixels, int sample_count);
    // Batch: every job of a device job table (units numbered across jobs, as for the batch
    // megakernel) in one cooperative launch; the caller commits split-mode films afterwards
    // (launch_film_commit_jobs). Returns the number of kernels launched.
    int run_batch(const JobDesc* d_jobs, const BatchHeader* d_hdr, DevCounters* counters, bool count_rays,
                  cudaStream_t stream);
    uint64_t bytes() const;
    int capacity() const { return capacity_; }
    // Bytes of the pool under a persisting L2 access-policy window on every launch (0: none).
    size_t l2_window_bytes() const;
    // Speculative traversal on or off for the following launches (box_step; same films either way).
    void set_speculate(bool on) { cfg_.speculate = on; }

private:
    struct State;
    std::unique_ptr<State> state_;
    void* arena_ = nullptr;
    uint64_t bytes_ = 0;
    int capacity_ = 0;
    int pixels_ = 0;
    WavefrontConfig cfg_;
    int chunks_for(int pixels, int sample_count) const;
    void reserve_direct();  // direct-mode film sums per slot
};

// Pool bytes per path slot, and the largest pool (a multiple of the block) that fits the
// device's persisting L2 set-aside.
size_t wavefront_slot_bytes();
size_t wavefront_l2_resident_paths(int device);

}  // namespace wfb
