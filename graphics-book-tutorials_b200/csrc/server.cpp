// Render server: a request loop that admits jobs of uneven size as they arrive and renders them
// with continuous batching on one GPU.
//
//  * Admission: a queued job is admitted when the device bytes of all admitted jobs (film sums +
//    split-mode sample buffer) stay within the budget and the launch has room.
//  * Iteration-level scheduling: every launch advances admitted jobs by slices of their samples;
//    a job that arrives while a launch runs joins the next launch, so new requests overlap on the
//    device with the ones in progress. The launch's sample budget comes from the measured
//    throughput so a launch takes about launch_target_ms, which bounds how long a new arrival
//    waits before its first samples run; plan_launch shares it out (express lane for small jobs,
//    large jobs in arrival order; or equal slices).
//  * Bit-exactness: slices add samples [done, done + k) to the job's film sums, which is the
//    progressive API's contract (WVM/include/wf/renderer.hpp:54-60): the finished film equals the
//    job rendered alone in one call.
//  * Device memory comes from the stream-ordered pool (cudaMallocAsync / cudaFreeAsync), so
//    admitting and retiring jobs never blocks the device.
//  * Plain mode (one_job_per_launch) renders queued jobs one at a time, FIFO, one launch each:
//    the sequential baseline at the same arrival stream.
//  * Two launches are in flight: the worker prepares and enqueues the next launch (and copies
//    finished films) while the GPU renders the current one.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include "server.hpp"
#include "../../include/wfb200.h"

namespace wfb {

double now_seconds() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Server::Job {
    JobSpec spec;
    uint64_t rate_key = 0;  // class of its rendering rate (scene content, depth limit)
    int state = kQueued;
    int done = 0;      // samples added to the film so far (launches finished)
    int issued = 0;    // samples enqueued (launches finished or in flight)
    int inflight = 0;  // launches in flight that render some of this job
    bool downloading = false;  // all samples rendered; the download thread is copying the film
    double t_arrival = 0.0, t_done = 0.0;
    JobBuffers buf;
    void* mem = nullptr;
    uint64_t bytes = 0;
    std::vector<float> rgb, lum_var;
    std::string error;
};

Server::Server(const ServerConfig& cfg) : cfg_(cfg) {
    // Plain mode launches one job at a time but admits two, so that it too keeps one launch in
    // flight while the previous one is retired.
    max_active_ = cfg_.one_job_per_launch ? 2 : cfg_.max_jobs;
    if (cfg_.one_job_per_launch) cfg_.max_jobs = 1;
    for (auto& l : launchers_) l = std::make_unique<BatchLauncher>(cfg_.max_jobs, cfg_.launch);
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : ev_) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    device_ = dev;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = cfg_.budget_bytes;  // retain freed blocks in the pool between jobs
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    thread_ = std::thread([this] { worker(); });
    dl_thread_ = std::thread([this] { downloader(); });
    alloc_thread_ = std::thread([this] { allocator(); });
}

Server::~Server() { shutdown(); }

void Server::shutdown() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        if (stop_ && !thread_.joinable()) return;
        stop_ = true;
    }
    cv_work_.notify_all();
    cv_dl_.notify_all();
    cv_alloc_.notify_all();
    if (thread_.joinable()) thread_.join();
    if (dl_thread_.joinable()) dl_thread_.join();
    if (alloc_thread_.joinable()) alloc_thread_.join();
    std::lock_guard<std::mutex> lock(mu_);
    for (auto& kv : jobs_)
        if (kv.second->mem) {
            cudaFreeAsync(kv.second->mem, stream_);
            kv.second->mem = nullptr;
        }
    for (void* m : to_free_) cudaFreeAsync(m, stream_);
    to_free_.clear();
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
        stream_ = nullptr;
    }
    for (auto& e : ev_) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    for (auto& l : launchers_) l.reset();
    cv_done_.notify_all();
}

uint64_t Server::job_bytes(const Job& j) const {
    const uint64_t p = (uint64_t)j.spec.width * j.spec.height;
    const int chunks = launchers_[0]->chunks_for((int)p, j.spec.sample_count);
    uint64_t b = 5 * p * sizeof(float);
    if (chunks > 1) b += 3 * p * (uint64_t)j.spec.sample_count * sizeof(float);
    return b;
}

uint64_t Server::submit(const JobSpec& job) {
    if (!job.scene) throw Error(WFB_ERR_INVALID_ARGUMENT, "job without a scene");
    if (job.width <= 0 || job.height <= 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "resolution must be positive");
    if (job.sample_count <= 0 || job.max_depth < 0) throw Error(WFB_ERR_INVALID_ARGUMENT, "bad spp or depth");
    auto j = std::make_unique<Job>();
    j->spec = job;
    j->rate_key = mix_key(job.scene->content_key, &job.max_depth, sizeof(job.max_depth));
    j->spec.first_sample = 0;
    j->t_arrival = now_seconds();
    uint64_t ticket;
    {
        std::lock_guard<std::mutex> lock(mu_);
        if (stop_) throw Error(WFB_ERR_INVALID_ARGUMENT, "server is shut down");
        j->bytes = job_bytes(*j);
        if (j->bytes > cfg_.budget_bytes) throw Error(WFB_ERR_OUT_OF_MEMORY, "job exceeds the server's memory budget");
        ticket = next_ticket_++;
        if (t_first_ < 0) t_first_ = j->t_arrival;
        jobs_[ticket] = std::move(j);
        queue_.push_back(ticket);
        st_.submitted++;
    }
    cv_work_.notify_one();
    return ticket;
}

int Server::state(uint64_t ticket) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) throw Error(WFB_ERR_INVALID_ARGUMENT, "unknown ticket");
    return it->second->state;
}

bool Server::wait(uint64_t ticket, int timeout_ms) {
    std::unique_lock<std::mutex> lock(mu_);
    auto finished = [&] {
        auto it = jobs_.find(ticket);
        return it == jobs_.end() || it->second->state >= kDone || stop_;
    };
    if (timeout_ms < 0) {
        cv_done_.wait(lock, finished);
        return true;
    }
    return cv_done_.wait_for(lock, std::chrono::milliseconds(timeout_ms), finished);
}

void Server::result(uint64_t ticket, float* rgb, float* lum_var, double* latency_ms) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) throw Error(WFB_ERR_INVALID_ARGUMENT, "unknown ticket");
    Job& j = *it->second;
    if (j.state == kFailed) {
        const std::string msg = j.error;
        jobs_.erase(it);
        throw Error(WFB_ERR_CUDA, "job failed: " + msg);
    }
    if (j.state != kDone) throw Error(WFB_ERR_INVALID_ARGUMENT, "job is not finished");
    if (rgb) std::memcpy(rgb, j.rgb.data(), j.rgb.size() * sizeof(float));
    if (lum_var) std::memcpy(lum_var, j.lum_var.data(), j.lum_var.size() * sizeof(float));
    if (latency_ms) *latency_ms = 1e3 * (j.t_done - j.t_arrival);
    jobs_.erase(it);
}

bool Server::cancel(uint64_t ticket) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end() || it->second->state >= kDone) return false;
    Job& j = *it->second;
    if (j.state == kQueued) queue_.erase(std::remove(queue_.begin(), queue_.end(), ticket), queue_.end());
    j.state = kCancelled;  // an active job is dropped at the next launch boundary
    st_.cancelled++;
    cv_done_.notify_all();
    return true;
}

static double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = (size_t)std::ceil(pos);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

ServerStats Server::stats() {
    std::lock_guard<std::mutex> lock(mu_);
    ServerStats s = st_;
    s.p50_ms = percentile(latencies_ms_, 0.50);
    s.p95_ms = percentile(latencies_ms_, 0.95);
    s.p99_ms = percentile(latencies_ms_, 0.99);
    s.max_ms = latencies_ms_.empty() ? 0.0 : *std::max_element(latencies_ms_.begin(), latencies_ms_.end());
    double sum = 0.0;
    for (double v : latencies_ms_) sum += v;
    s.mean_ms = latencies_ms_.empty() ? 0.0 : sum / latencies_ms_.size();
    s.wall_s = t_first_ < 0 ? 0.0 : now_seconds() - t_first_;
    s.bytes_in_use = bytes_in_use_;
    s.peak_bytes = peak_bytes_;
    s.queued = (int)(queue_.size() + allocating_.size());
    s.active = (int)active_.size();
    return s;
}

void Server::reset_stats() {
    std::lock_guard<std::mutex> lock(mu_);
    latencies_ms_.clear();
    const uint64_t submitted = st_.submitted - st_.completed - st_.cancelled - st_.failed;
    st_ = ServerStats{};
    st_.submitted = submitted;
    t_first_ = -1.0;
    peak_bytes_ = bytes_in_use_;
}

// Moves queued jobs to the allocator while the budget and the launch's capacity allow (FIFO, no
// overtaking): their bytes are reserved here, the memory itself comes from allocator().
bool Server::admit_locked() {
    bool any = false;
    while (!alloc_blocked_ && !queue_.empty() && (int)(active_.size() + allocating_.size()) < max_active_) {
        Job& j = *jobs_[queue_.front()];
        if (bytes_in_use_ + j.bytes > cfg_.budget_bytes) break;
        bytes_in_use_ += j.bytes;
        peak_bytes_ = std::max(peak_bytes_, bytes_in_use_);
        allocating_.push_back(queue_.front());
        queue_.pop_front();
        any = true;
    }
    if (any) cv_alloc_.notify_one();
    return any;
}

// Allocates and zeroes the films of admitted jobs, in admission order, on its own stream and
// without the server lock: growing the stream-ordered pool while persistent launches run took up to
// 0.8 s for 1.6 GB on a B200, and done under the lock (as admission once did) it stalled the worker
// and every submit meanwhile. A job becomes active once its memory is ready. The thread first grows
// the pool to the budget (at most 80% of the free memory), which it then keeps (release threshold).
void Server::allocator() {
    cudaSetDevice(device_);
    cudaStream_t s = nullptr;
    const cudaError_t se = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (se == cudaSuccess) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const uint64_t warm = std::min<uint64_t>(cfg_.budget_bytes, (uint64_t)(0.8 * (double)free_b));
            void* p = nullptr;
            if (warm > 0 && cudaMallocAsync(&p, warm, s) == cudaSuccess) cudaFreeAsync(p, s);
            cudaStreamSynchronize(s);
        }
        cudaGetLastError();  // a pool that cannot grow that far is not an error here
    }
    for (;;) {
        uint64_t ticket;
        Job* j;
        {
            std::unique_lock<std::mutex> lock(mu_);
            cv_alloc_.wait(lock, [&] { return stop_ || !allocating_.empty(); });
            if (stop_) break;
            ticket = allocating_.front();
            j = jobs_[ticket].get();
        }
        const uint64_t p = (uint64_t)j->spec.width * j->spec.height;
        void* mem = nullptr;
        cudaError_t e = se;
        if (e == cudaSuccess) e = cudaMallocAsync(&mem, j->bytes, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(mem, 0, 5 * p * sizeof(float), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) cudaGetLastError();
        {
            std::lock_guard<std::mutex> lock(mu_);
            allocating_.pop_front();
            if (e != cudaSuccess) {
                // no room now (or a failed allocation): back to the head of the queue until a job
                // releases memory
                if (mem) to_free_.push_back(mem);
                bytes_in_use_ -= j->bytes;
                if (j->state == kCancelled) {
                    jobs_.erase(ticket);
                } else {
                    queue_.push_front(ticket);
                    alloc_blocked_ = true;
                }
            } else if (j->state == kCancelled) {
                to_free_.push_back(mem);
                bytes_in_use_ -= j->bytes;
                jobs_.erase(ticket);
            } else {
                j->mem = mem;
                j->buf.chunks = launchers_[0]->chunks_for((int)p, j->spec.sample_count);
                float* f = static_cast<float*>(mem);
                j->buf.film = DevFilm{f, f + 3 * p, f + 4 * p, (int)p};
                j->buf.lbuf = j->buf.chunks > 1 ? f + 5 * p : nullptr;
                j->state = kActive;
                active_.push_back(ticket);
            }
        }
        cv_work_.notify_one();
    }
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
}

double Server::class_rate(uint64_t key) const {
    auto it = class_msps_.find(key);
    if (it != class_msps_.end()) return it->second;
    // an unseen class starts at the slowest known rate: its first launch can only come out
    // shorter than planned, never several times longer
    double r = msps_default_;
    for (const auto& kv : class_msps_) r = std::min(r, kv.second);
    return r;
}

// Samples of each admitted job (in admission order) for the next launch; 0 leaves a job out. The
// budget is the launch's target length; a job's cost per sample is its pixels at its class's rate.
std::vector<int> Server::plan_launch(const std::vector<Job*>& act) {
    std::vector<int> k(act.size(), 0);
    for (size_t i = 0; i < act.size(); ++i) {
        const int rem = act[i]->spec.sample_count - act[i]->issued;
        if (cfg_.one_job_per_launch) k[i] = rem;
        else if (cfg_.fixed_slice > 0) k[i] = std::min(cfg_.fixed_slice, rem);
    }
    if (cfg_.one_job_per_launch || cfg_.fixed_slice > 0) return k;
    std::vector<SliceJob> jobs(act.size());
    for (size_t i = 0; i < act.size(); ++i) {
        const double pixels = (double)act[i]->spec.width * act[i]->spec.height;
        jobs[i] = SliceJob{pixels / (class_rate(act[i]->rate_key) * 1e3), act[i]->spec.sample_count - act[i]->issued};
    }
    return plan_slices(jobs, cfg_.launch_target_ms, cfg_.schedule);
}

// Two launches in flight: while the GPU renders launch N, the worker retires launch N-1's
// finished jobs (film copies overlap launch N) and enqueues launch N+1 on the other launcher, so
// the device does not idle through host bookkeeping. Slices are planned from `issued` samples;
// launches on the one stream run in order, so a job's slices still add in ascending sample order.
void Server::worker() {
    cudaSetDevice(device_);  // the device the server was created on
    struct Flight {
        std::vector<Job*> jobs;
        std::vector<uint64_t> tickets;
        std::vector<int> counts;  // samples of each job in this launch
        std::vector<double> pred_ms;  // predicted device time of each job's slice
        uint64_t samples = 0;
        int slot = 0;
        std::string err;
    };
    std::deque<Flight> flights;
    int next_slot = 0;
    for (;;) {
        Flight f;
        {
            std::unique_lock<std::mutex> lock(mu_);
            release_idle_locked();
            admit_locked();
            auto issuable = [&] {
                for (uint64_t t : active_) {
                    const Job& j = *jobs_[t];
                    if (j.state == kActive && j.issued < j.spec.sample_count) return true;
                }
                return false;
            };
            while (!stop_ && flights.empty() && !issuable()) {
                cv_work_.wait(lock);
                release_idle_locked();
                admit_locked();
            }
            if (stop_) break;
            if (flights.size() < 2)
                for (uint64_t t : active_) {
                    Job* j = jobs_[t].get();
                    if (j->state == kActive && j->issued < j->spec.sample_count) {
                        f.tickets.push_back(t);
                        f.jobs.push_back(j);
                        if (cfg_.one_job_per_launch) break;  // the oldest admitted job, whole
                    }
                }
        }
        if (!f.jobs.empty()) {
            // ---- enqueue one launch: each planned job advances by its slice ----
            const std::vector<int> plan = plan_launch(f.jobs);
            std::vector<Job*> jobs;
            std::vector<uint64_t> tickets;
            std::vector<JobSpec> specs;
            std::vector<JobBuffers> bufs;
            for (size_t i = 0; i < f.jobs.size(); ++i) {
                if (plan[i] <= 0) continue;
                Job* j = f.jobs[i];
                JobSpec sp = j->spec;
                sp.first_sample = j->issued;
                sp.sample_count = plan[i];
                f.samples += (uint64_t)sp.width * sp.height * sp.sample_count;
                f.counts.push_back(sp.sample_count);
                f.pred_ms.push_back((double)sp.width * sp.height * sp.sample_count / (class_rate(j->rate_key) * 1e3));
                JobBuffers b = j->buf;
                b.chunks = std::min(b.chunks, sp.sample_count);
                if (b.chunks > 1 && b.lbuf != nullptr) {
                    // at least two work units per resident lane: a small image's slice is cut into
                    // more, shorter units instead of a few long ones that leave the launch a tail
                    const long long px = (long long)sp.width * sp.height;
                    const long long want = (2ll * launchers_[0]->resident_lanes() + px - 1) / px;
                    b.chunks = (int)std::min<long long>(sp.sample_count, std::max<long long>(b.chunks, want));
                }
                if (b.chunks > 1 && b.lbuf == nullptr) b.chunks = 1;
                jobs.push_back(j);
                tickets.push_back(f.tickets[i]);
                specs.push_back(sp);
                bufs.push_back(b);
            }
            f.jobs = std::move(jobs);
            f.tickets = std::move(tickets);
            f.slot = next_slot;
            next_slot ^= 1;
            try {
                cuda_check(cudaEventRecord(ev_[2 * f.slot], stream_), "cudaEventRecord");
                launchers_[f.slot]->launch(specs, bufs, false, stream_);
                cuda_check(cudaEventRecord(ev_[2 * f.slot + 1], stream_), "cudaEventRecord");
            } catch (const std::exception& e) {
                f.err = e.what();
            }
            {
                std::lock_guard<std::mutex> lock(mu_);
                for (size_t i = 0; i < f.jobs.size(); ++i) {
                    f.jobs[i]->issued += f.counts[i];
                    f.jobs[i]->inflight++;
                }
            }
            flights.push_back(std::move(f));
            if (flights.size() < 2) continue;  // fill the pipeline before waiting
        }
        if (flights.empty()) continue;
        // ---- retire the oldest launch ----
        Flight done = std::move(flights.front());
        flights.pop_front();
        float ms = 0.f;
        if (done.err.empty()) {
            const cudaError_t e = cudaEventSynchronize(ev_[2 * done.slot + 1]);
            if (e != cudaSuccess) done.err = cudaGetErrorString(e);
            else cudaEventElapsedTime(&ms, ev_[2 * done.slot], ev_[2 * done.slot + 1]);
        }
        // Only launches that filled most of their budget refine the rate: a launch carrying a few
        // small jobs is dominated by its ramp-up and tail, and its low rate would shrink every
        // following slice (large jobs would then crawl through many short launches).
        // Refine the rates: each class in the launch moves toward the ratio of predicted to measured
        // time, by half of it (at most 2x either way) to the power of its share of the prediction: a
        // class converges over a few launches, and no single launch (a cold start, a tail) can move
        // a rate far.
        double pred = 0.0;
        for (double v : done.pred_ms) pred += v;
        if (done.err.empty() && ms > 0.f && pred >= 0.5 * cfg_.launch_target_ms) {
            const double ratio = std::clamp(pred / (double)ms, 0.5, 2.0);
            std::map<uint64_t, double> share;
            for (size_t i = 0; i < done.jobs.size(); ++i) share[done.jobs[i]->rate_key] += done.pred_ms[i] / pred;
            std::map<uint64_t, double> next;
            for (const auto& [key, w] : share) next[key] = class_rate(key) * std::pow(ratio, 0.5 * w);
            for (const auto& [key, r] : next) class_msps_[key] = r;
        }
        // Jobs this launch finished go to the download thread: no later launch touches their films,
        // so the copies overlap the launch in flight and the worker goes on enqueueing.
        bool handed = false;
        {
            std::lock_guard<std::mutex> lock(mu_);
            st_.launches++;
            st_.busy_ms += ms;
            st_.samples_done += done.samples;
            for (size_t i = 0; i < done.jobs.size(); ++i) {
                Job* j = done.jobs[i];
                j->inflight--;
                j->done += done.counts[i];
                if (j->state != kActive) continue;  // cancelled meanwhile: released when idle
                if (!done.err.empty()) {
                    j->state = kFailed;
                    j->error = done.err;
                    st_.failed++;
                } else if (j->done >= j->spec.sample_count) {
                    j->downloading = true;
                    dl_queue_.push_back(done.tickets[i]);
                    handed = true;
                }
            }
            release_idle_locked();
        }
        if (handed) cv_dl_.notify_one();
        cv_done_.notify_all();
    }
    // stopping: let launches in flight finish before their memory is released
    cudaStreamSynchronize(stream_);
}

// Copies the films of finished jobs to the host (GPU-arm download convention) and completes them.
// The film is final: its job's last launch has finished and no later launch renders it.
void Server::downloader() {
    cudaSetDevice(device_);
    cudaStream_t dl_stream = nullptr;  // this thread's copies: ordered after nothing but themselves
    const cudaError_t se = cudaStreamCreateWithFlags(&dl_stream, cudaStreamNonBlocking);
    // Pinned staging for the films, sized up front for a 1920x1080 film (grown if a larger one comes):
    // pinning host memory while launches run is one more driver call that can wait.
    PinnedStaging staging;
    if (cudaHostAlloc(&staging.ptr, 5ull * 1920 * 1080 * sizeof(float), cudaHostAllocDefault) == cudaSuccess)
        staging.bytes = 5ull * 1920 * 1080 * sizeof(float);
    else
        staging.ptr = nullptr, cudaGetLastError();
    for (;;) {
        uint64_t ticket;
        Job* j;
        {
            std::unique_lock<std::mutex> lock(mu_);
            cv_dl_.wait(lock, [&] { return stop_ || !dl_queue_.empty(); });
            if (dl_queue_.empty()) break;  // stopping with nothing left to copy
            ticket = dl_queue_.front();
            dl_queue_.pop_front();
            j = jobs_[ticket].get();
        }
        const size_t p = (size_t)j->spec.width * j->spec.height;
        std::string err;
        try {
            j->rgb.resize(3 * p);
            j->lum_var.resize(p);
            cuda_check(se, "cudaStreamCreate download");
            film_download_host(j->buf.film, j->spec.sample_count, j->rgb.data(), j->lum_var.data(), dl_stream,
                               &staging);
        } catch (const std::exception& e) {
            err = e.what();
        }
        {
            std::lock_guard<std::mutex> lock(mu_);
            j->downloading = false;
            if (j->state == kActive) {
                if (err.empty()) {
                    j->state = kDone;
                    j->t_done = now_seconds();
                    st_.completed++;
                    latencies_ms_.push_back(1e3 * (j->t_done - j->t_arrival));
                } else {
                    j->state = kFailed;
                    j->error = err;
                    st_.failed++;
                }
            }
            release_idle_locked(false);  // the worker frees the film's memory (stream_ is its own)
        }
        cv_done_.notify_all();
        cv_work_.notify_one();  // memory came back: more jobs may be admitted
    }
    if (dl_stream) cudaStreamDestroy(dl_stream);
    if (staging.ptr) cudaFreeHost(staging.ptr);
}

// Releases jobs that left the active set (done, failed or cancelled) once no launch in flight
// renders them; cancelled jobs are forgotten, finished ones wait for result(). Their device memory
// is freed on stream_ by the worker, the only thread that enqueues work there (it may be capturing
// a graph on it); other threads leave it in to_free_ for the worker's next call.
void Server::release_idle_locked(bool worker) {
    for (auto it = active_.begin(); it != active_.end();) {
        Job& j = *jobs_[*it];
        if (j.state == kActive || j.inflight > 0 || j.downloading) {
            ++it;
            continue;
        }
        if (j.mem) to_free_.push_back(j.mem);
        j.mem = nullptr;
        bytes_in_use_ -= j.bytes;
        alloc_blocked_ = false;  // memory came back: a job that found no room may try again
        if (j.state == kCancelled) jobs_.erase(*it);
        it = active_.erase(it);
    }
    if (!worker) return;
    for (void* m : to_free_) cudaFreeAsync(m, stream_);
    to_free_.clear();
}

}  // namespace wfb
