// How one launch of the render server shares its sample budget among admitted jobs (pure host
// logic, no CUDA; server.cpp calls it, tests/schedule_check.cpp checks it on the CPU).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

namespace wfb {

// Continuous-batching schedules (wfb_server_config::schedule):
//   express: jobs whose remaining work fits a quarter of the budget ride in the next launch whole
//            (an express lane: they never wait behind a large job); large jobs share the rest in
//            arrival order -- the oldest takes all it can, the next ones what is left -- so a large
//            job is not slowed by the large jobs that arrived after it. The oldest large job always
//            gets at least a quarter of the budget, so a stream of small jobs cannot starve it.
//   shared:  every admitted job advances by the same number of samples per launch (processor
//            sharing): small jobs finish early, but each large job is slowed by all the others.
constexpr int kScheduleExpress = 0;
constexpr int kScheduleShared = 1;

struct SliceJob {
    double cost;    // predicted cost of one sample of every pixel of the job (e.g. ms)
    int remaining;  // samples per pixel not yet issued (> 0)
};

// Samples per pixel of each job (in admission order) for the next launch; 0 leaves a job out.
// `budget` is the launch's cost budget, in the unit of SliceJob::cost. At least one job advances.
inline std::vector<int> plan_slices(const std::vector<SliceJob>& jobs, double budget, int schedule) {
    std::vector<int> k(jobs.size(), 0);
    if (jobs.empty()) return k;
    if (schedule == kScheduleShared) {
        // the largest common slice whose total stays within the budget (at least one sample)
        auto total = [&](int s) {
            double t = 0.0;
            for (const SliceJob& j : jobs) t += j.cost * std::min(s, j.remaining);
            return t;
        };
        int lo = 1, hi = 1;
        for (const SliceJob& j : jobs) hi = std::max(hi, j.remaining);
        while (lo < hi) {
            const int mid = lo + (hi - lo + 1) / 2;
            if (total(mid) <= budget) lo = mid;
            else hi = mid - 1;
        }
        for (size_t i = 0; i < jobs.size(); ++i) k[i] = std::min(lo, jobs[i].remaining);
        return k;
    }
    // express: small jobs whole (arrival order, while the budget lasts), then large jobs FIFO
    const double small = 0.25 * budget;
    double left = budget;
    bool any = false;
    for (size_t i = 0; i < jobs.size(); ++i) {
        const double work = jobs[i].cost * jobs[i].remaining;
        if (work <= small && (work <= left || !any)) {
            k[i] = jobs[i].remaining;
            left -= work;
            any = true;
        }
    }
    bool oldest_large = true;
    for (size_t i = 0; i < jobs.size(); ++i) {
        if (k[i] > 0 || jobs[i].cost * jobs[i].remaining <= small) continue;
        const double share = oldest_large ? std::max(left, small) : left;
        int s = (int)std::min<double>(jobs[i].remaining, std::floor(share / jobs[i].cost));
        if (s < 1 && (oldest_large || !any)) s = 1;  // the oldest large job always advances
        if (s < 1) break;                             // later large jobs wait their turn
        k[i] = s;
        left -= jobs[i].cost * s;
        any = true;
        oldest_large = false;
    }
    return k;
}

}  // namespace wfb
