// CPU checks of the render server's launch planning (csrc/schedule.hpp): prints "ok <cases>" or
// the first failed check and exits non-zero.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include "schedule.hpp"

using wfb::SliceJob;

static int g_cases = 0;
#define CHECK(c)                                                            \
    do {                                                                    \
        ++g_cases;                                                          \
        if (!(c)) {                                                         \
            std::printf("FAILED line %d: %s\n", __LINE__, #c);              \
            std::exit(1);                                                   \
        }                                                                   \
    } while (0)

static double work(const std::vector<SliceJob>& j, const std::vector<int>& k) {
    double s = 0;
    for (size_t i = 0; i < j.size(); ++i) s += j[i].cost * k[i];
    return s;
}

int main() {
    const double B = 20e6;  // a 20 ms launch at 1000 Msamples/s
    // express: a small job rides whole beside a large one, which takes the rest of the budget
    {
        std::vector<SliceJob> j = {{2073600, 64}, {65536, 4}};
        auto k = wfb::plan_slices(j, B, wfb::kScheduleExpress);
        CHECK(k[1] == 4);
        CHECK(k[0] == (int)((B - 65536.0 * 4) / 2073600));
        CHECK(work(j, k) <= B);
    }
    // express: large jobs in arrival order -- the oldest takes all it can, the next gets the rest
    {
        std::vector<SliceJob> j = {{921600, 64}, {921600, 64}};
        auto k = wfb::plan_slices(j, B, wfb::kScheduleExpress);
        CHECK(k[0] == (int)(B / 921600));
        CHECK(k[1] == 0);
        j[0].remaining = 3;  // the oldest is nearly done: the next one takes what is left
        k = wfb::plan_slices(j, B, wfb::kScheduleExpress);
        CHECK(k[0] == 3 && k[1] == (int)((B - 3 * 921600.0) / 921600));
    }
    // express: a flood of small jobs cannot starve the oldest large job (a quarter of the budget)
    {
        std::vector<SliceJob> j = {{2073600, 64}};
        for (int i = 0; i < 400; ++i) j.push_back({65536, 16});
        auto k = wfb::plan_slices(j, B, wfb::kScheduleExpress);
        CHECK(k[0] >= (int)(0.25 * B / 2073600));
        CHECK(k[0] >= 1);
        int small = 0;
        for (size_t i = 1; i < j.size(); ++i) small += k[i] > 0;
        CHECK(small > 0 && small < 400);
        CHECK(work(j, k) <= 1.25 * B + 1);
    }
    // a job larger than the whole budget still advances by one sample
    {
        std::vector<SliceJob> j = {{1e9, 8}};
        for (int s : {wfb::kScheduleExpress, wfb::kScheduleShared}) {
            auto k = wfb::plan_slices(j, B, s);
            CHECK(k[0] == 1);
        }
    }
    // shared: one common slice, the largest whose total fits
    {
        std::vector<SliceJob> j = {{2073600, 64}, {921600, 64}, {65536, 1}};
        auto k = wfb::plan_slices(j, B, wfb::kScheduleShared);
        CHECK(k[2] == 1 && k[0] == k[1] && k[0] >= 1);
        CHECK(work(j, k) <= B);
        std::vector<int> k1 = k;
        for (auto& x : k1) ++x;
        k1[2] = 1;
        CHECK(work(j, k1) > B);
    }
    // random mixes: bounds, progress and no over-issue for both schedules
    std::mt19937 rng(1234);
    const double px[] = {65536, 230400, 921600, 2073600};
    const int spp[] = {1, 4, 16, 64};
    for (int t = 0; t < 20000; ++t) {
        std::vector<SliceJob> j(1 + rng() % 40);
        for (auto& x : j) x = SliceJob{px[rng() % 4], 1 + (int)(rng() % spp[rng() % 4])};
        const double b = 1e6 * (1 + rng() % 60);
        for (int s : {wfb::kScheduleExpress, wfb::kScheduleShared}) {
            auto k = wfb::plan_slices(j, b, s);
            int advancing = 0;
            for (size_t i = 0; i < j.size(); ++i) {
                CHECK(k[i] >= 0 && k[i] <= j[i].remaining);
                advancing += k[i] > 0;
            }
            CHECK(advancing >= 1);
            // express: over budget only by the starvation guard (a quarter) and one sample of the
            // oldest large job; shared: every job advances at least one sample
            double biggest = 0, all = 0;
            for (const auto& x : j) {
                biggest = std::max(biggest, x.cost);
                all += x.cost;
            }
            if (s == wfb::kScheduleExpress) CHECK(work(j, k) <= 1.25 * b + biggest + 1);
            else CHECK(work(j, k) <= std::max(b, all) + 1);
        }
    }
    std::printf("ok %d\n", g_cases);
    return 0;
}
