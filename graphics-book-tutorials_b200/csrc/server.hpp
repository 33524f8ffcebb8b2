// Render server: continuous batching of render jobs on one GPU (server.cpp).
#pragma once
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "batch.hpp"
#include "schedule.hpp"

namespace wfb {

struct ServerConfig {
    uint64_t budget_bytes = 40ull << 30;  // device bytes of admitted jobs (films + sample buffers)
    int max_jobs = 256;                   // jobs per launch
    double launch_target_ms = 20.0;       // slice size aims at launches of about this length
    int fixed_slice = 0;                  // > 0: samples per job per launch (0: adaptive)
    bool one_job_per_launch = false;      // plain mode: FIFO, whole job, one launch per job
    int schedule = kScheduleExpress;      // how a launch's budget is shared (schedule.hpp)
    LaunchConfig launch;  // arm and knobs of every launch
};

// Work units per pixel of a served job unless configured: served jobs advance in slices of a few
// samples per launch, and at lambda = 10 jobs/s on the 64-job mix 4 units per pixel gave the lowest
// p50/p95/p99 on a B200 (one-sample units: p95 3.5x higher; whole-pixel units: p95 1.4x higher).
constexpr int kServerSplitChunks = 4;

enum JobState : int { kQueued = 0, kActive = 1, kDone = 2, kCancelled = 3, kFailed = 4 };

struct ServerStats {
    uint64_t submitted = 0, completed = 0, cancelled = 0, failed = 0, launches = 0;
    uint64_t samples_done = 0;
    double busy_ms = 0.0;  // device time of all launches
    double wall_s = 0.0;   // since the first submission
    double p50_ms = 0.0, p95_ms = 0.0, p99_ms = 0.0, mean_ms = 0.0, max_ms = 0.0;
    uint64_t bytes_in_use = 0, peak_bytes = 0;
    int queued = 0, active = 0;
};

class Server {
public:
    explicit Server(const ServerConfig& cfg);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    uint64_t submit(const JobSpec& job);  // thread-safe; the arrival time is now
    int state(uint64_t ticket);
    // Waits for completion; false on timeout (timeout_ms < 0: forever).
    bool wait(uint64_t ticket, int timeout_ms);
    // Copies the finished film (GPU-arm download convention) and releases the job.
    void result(uint64_t ticket, float* rgb, float* lum_var, double* latency_ms);
    bool cancel(uint64_t ticket);
    ServerStats stats();
    void reset_stats();
    void shutdown();

private:
    struct Job;
    void worker();
    uint64_t job_bytes(const Job& j) const;
    bool admit_locked();
    void release_idle_locked(bool worker = true);
    void downloader();
    void allocator();
    std::vector<int> plan_launch(const std::vector<Job*>& act);

    ServerConfig cfg_;
    std::unique_ptr<BatchLauncher> launchers_[2];  // alternate launches: one renders, one is prepared
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};  // start / end of each launcher's launch
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::map<uint64_t, std::unique_ptr<Job>> jobs_;
    std::deque<uint64_t> queue_;
    std::vector<uint64_t> active_;
    uint64_t next_ticket_ = 1;
    int max_active_ = 256;  // admitted jobs at once
    bool stop_ = false;
    std::thread thread_;
    std::thread dl_thread_;               // copies finished films to the host
    std::thread alloc_thread_;            // allocates admitted jobs' films (allocator())
    std::condition_variable cv_alloc_;
    std::deque<uint64_t> allocating_;     // admitted jobs waiting for their memory, in order
    bool alloc_blocked_ = false;          // an allocation failed: admit again once memory returns
    std::condition_variable cv_dl_;
    std::deque<uint64_t> dl_queue_;
    std::vector<void*> to_free_;          // device memory released off the worker, freed by it
    uint64_t bytes_in_use_ = 0, peak_bytes_ = 0;
    // Rendering rate (Msamples/s) per job class -- scene content and depth limit: the mix's classes
    // differ several-fold (a 36-triangle box at depth 4 against 164k triangles at depth 8), so one
    // rate for all would size launches for the last class that ran. Unseen classes start at the
    // slowest known class rate (msps_default_ before any). Refined by launches that filled half their
    // budget.
    std::map<uint64_t, double> class_msps_;
    double msps_default_ = 500.0;
    double class_rate(uint64_t key) const;
    std::vector<double> latencies_ms_;
    ServerStats st_;
    double t_first_ = -1.0;
    int device_ = 0;
};

double now_seconds();

}  // namespace wfb
