// Render server: a request loop that admits jobs of uneven size as they arrive and renders them
// with continuous batching on one GPU.
//
//  * Admission: a queued job is admitted when the device bytes of all admitted jobs (film sums +
//    split-mode sample buffer) stay within the budget and the launch has room.
//  * Iteration-level scheduling: every launch advances every admitted job by a slice of its
//    samples; a job that arrives while a launch runs joins the next launch, so new requests
//    overlap on the device with the ones in progress. The slice is chosen from the measured
//    throughput so a launch takes about launch_target_ms, which bounds how long a new arrival
//    waits before its first samples run.
//  * Bit-exactness: slices add samples [done, done + k) to the job's film sums, which is the
//    progressive API's contract (WVM/include/wf/renderer.hpp:54-60): the finished film equals the
//    job rendered alone in one call.
//  * Device memory comes from the stream-ordered pool (cudaMallocAsync / cudaFreeAsync), so
//    admitting and retiring jobs never blocks the device.
//  * Plain mode (one_job_per_launch) renders queued jobs one at a time, FIFO, one launch each:
//    the sequential baseline at the same arrival stream.
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
    int state = kQueued;
    int done = 0;  // samples added to the film so far
    double t_arrival = 0.0, t_done = 0.0;
    JobBuffers buf;
    void* mem = nullptr;
    uint64_t bytes = 0;
    std::vector<float> rgb, lum_var;
    std::string error;
};

Server::Server(const ServerConfig& cfg) : cfg_(cfg) {
    if (cfg_.one_job_per_launch) cfg_.max_jobs = 1;
    launcher_ = std::make_unique<BatchLauncher>(cfg_.max_jobs, cfg_.launch);
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaEventCreate(&ev0_), "cudaEventCreate");
    cuda_check(cudaEventCreate(&ev1_), "cudaEventCreate");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    device_ = dev;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = cfg_.budget_bytes;  // retain freed blocks in the pool between jobs
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    thread_ = std::thread([this] { worker(); });
}

Server::~Server() { shutdown(); }

void Server::shutdown() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        if (stop_ && !thread_.joinable()) return;
        stop_ = true;
    }
    cv_work_.notify_all();
    if (thread_.joinable()) thread_.join();
    std::lock_guard<std::mutex> lock(mu_);
    for (auto& kv : jobs_)
        if (kv.second->mem) {
            cudaFreeAsync(kv.second->mem, stream_);
            kv.second->mem = nullptr;
        }
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
        stream_ = nullptr;
    }
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    ev0_ = ev1_ = nullptr;
    launcher_.reset();
    cv_done_.notify_all();
}

uint64_t Server::job_bytes(const Job& j) const {
    const uint64_t p = (uint64_t)j.spec.width * j.spec.height;
    const int chunks = launcher_->chunks_for((int)p, j.spec.sample_count);
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
    s.queued = (int)queue_.size();
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

// Moves queued jobs to the active set while budget and launch capacity allow (FIFO, no overtaking).
bool Server::admit_locked() {
    bool any = false;
    while (!queue_.empty() && (int)active_.size() < cfg_.max_jobs) {
        Job& j = *jobs_[queue_.front()];
        if (bytes_in_use_ + j.bytes > cfg_.budget_bytes) break;
        const uint64_t p = (uint64_t)j.spec.width * j.spec.height;
        j.buf.chunks = launcher_->chunks_for((int)p, j.spec.sample_count);
        if (cudaMallocAsync(&j.mem, j.bytes, stream_) != cudaSuccess) {
            cudaGetLastError();
            break;  // try again after a job retires
        }
        float* f = static_cast<float*>(j.mem);
        j.buf.film = DevFilm{f, f + 3 * p, f + 4 * p, (int)p};
        j.buf.lbuf = j.buf.chunks > 1 ? f + 5 * p : nullptr;
        cudaMemsetAsync(f, 0, 5 * p * sizeof(float), stream_);
        bytes_in_use_ += j.bytes;
        peak_bytes_ = std::max(peak_bytes_, bytes_in_use_);
        j.state = kActive;
        active_.push_back(queue_.front());
        queue_.pop_front();
        any = true;
    }
    return any;
}

// Samples per job for the next launch: the largest k whose total stays within the launch budget.
int Server::choose_slice(const std::vector<Job*>& act) {
    if (cfg_.one_job_per_launch) return 1 << 30;
    if (cfg_.fixed_slice > 0) return cfg_.fixed_slice;
    const double budget = msps_estimate_ * 1e3 * cfg_.launch_target_ms;  // samples
    auto total = [&](int k) {
        double s = 0.0;
        for (const Job* j : act)
            s += (double)j->spec.width * j->spec.height * std::min(k, j->spec.sample_count - j->done);
        return s;
    };
    int lo = 1, hi = 1;
    for (const Job* j : act) hi = std::max(hi, j->spec.sample_count - j->done);
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (total(mid) <= budget) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

void Server::worker() {
    cudaSetDevice(device_);  // the device the server was created on
    for (;;) {
        std::vector<Job*> act;
        std::vector<uint64_t> tickets;
        {
            std::unique_lock<std::mutex> lock(mu_);
            // drop cancelled active jobs
            for (auto it = active_.begin(); it != active_.end();) {
                Job& j = *jobs_[*it];
                if (j.state == kCancelled) {
                    if (j.mem) cudaFreeAsync(j.mem, stream_);
                    j.mem = nullptr;
                    bytes_in_use_ -= j.bytes;
                    jobs_.erase(*it);
                    it = active_.erase(it);
                } else {
                    ++it;
                }
            }
            admit_locked();
            while (active_.empty() && !stop_) {
                cv_work_.wait(lock);
                admit_locked();
            }
            if (stop_) return;
            for (uint64_t t : active_) {
                tickets.push_back(t);
                act.push_back(jobs_[t].get());
            }
        }
        // ---- one launch: every active job advances by a slice ----
        const int k = choose_slice(act);
        std::vector<JobSpec> specs;
        std::vector<JobBuffers> bufs;
        uint64_t samples = 0;
        for (Job* j : act) {
            JobSpec s = j->spec;
            s.first_sample = j->done;
            s.sample_count = std::min(k, j->spec.sample_count - j->done);
            samples += (uint64_t)s.width * s.height * s.sample_count;
            JobBuffers b = j->buf;
            b.chunks = std::min(b.chunks, s.sample_count);
            if (b.chunks > 1 && b.lbuf == nullptr) b.chunks = 1;
            specs.push_back(s);
            bufs.push_back(b);
        }
        std::string err;
        float ms = 0.f;
        try {
            cuda_check(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
            launcher_->launch(specs, bufs, false, stream_);
            cuda_check(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
            cuda_check(cudaEventSynchronize(ev1_), "server launch");
            cudaEventElapsedTime(&ms, ev0_, ev1_);
        } catch (const std::exception& e) {
            err = e.what();
        }
        if (err.empty() && ms > 0.f && samples > 0) {
            const double rate = (double)samples / (ms * 1e3);  // Msamples/s
            msps_estimate_ = 0.7 * msps_estimate_ + 0.3 * rate;
        }
        // ---- retire finished jobs: download outside the lock, then update states under it ----
        std::vector<char> over(act.size(), 0);
        for (size_t i = 0; i < act.size(); ++i) {
            Job* j = act[i];
            if (!err.empty()) {
                over[i] = 1;
                continue;
            }
            j->done += specs[i].sample_count;
            if (j->done < j->spec.sample_count) continue;
            over[i] = 1;
            const size_t p = (size_t)j->spec.width * j->spec.height;
            j->rgb.resize(3 * p);
            j->lum_var.resize(p);
            try {
                film_download(j->buf.film, j->spec.sample_count, j->rgb.data(), j->lum_var.data(), stream_);
            } catch (const std::exception& e) {
                if (err.empty()) err = e.what();
            }
        }
        {
            std::lock_guard<std::mutex> lock(mu_);
            st_.launches++;
            st_.busy_ms += ms;
            st_.samples_done += samples;
            const double t = now_seconds();
            for (size_t i = 0; i < act.size(); ++i) {
                if (!over[i]) continue;
                Job* j = act[i];
                if (j->mem) cudaFreeAsync(j->mem, stream_);
                j->mem = nullptr;
                bytes_in_use_ -= j->bytes;
                active_.erase(std::remove(active_.begin(), active_.end(), tickets[i]), active_.end());
                if (j->state == kCancelled) {
                    jobs_.erase(tickets[i]);  // nobody waits for a cancelled job's film
                } else if (!err.empty()) {
                    j->state = kFailed;
                    j->error = err;
                    st_.failed++;
                } else {
                    j->state = kDone;
                    j->t_done = t;
                    st_.completed++;
                    latencies_ms_.push_back(1e3 * (t - j->t_arrival));
                }
            }
        }
        cv_done_.notify_all();
    }
}

}  // namespace wfb
