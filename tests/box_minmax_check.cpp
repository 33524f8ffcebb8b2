// Checks that wf::hit_box_minmax (the GPU traversal's box test) returns wf::hit_box's result on
// adversarial inputs: every slab quantity drawn from signed zeros, infinities, NaN, denormals,
// FLT_MAX and ordinary values, exhaustively per axis and by random mixing across axes.
// Built and run by tests/test_box_minmax.py; prints the number of cases and exits 1 on a mismatch.
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include "wf/bvh.hpp"
#include "wf/path_core.hpp"

namespace {

float bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

const float kSpecial[] = {-INFINITY, -FLT_MAX, -3.5f, -1.0f, -bits(1), -0.0f, 0.0f, bits(1), 1e-30f,
                          1.0f,      2.5f,     FLT_MAX, INFINITY, NAN, 1e30f, -1e-30f};
constexpr int kN = sizeof(kSpecial) / sizeof(kSpecial[0]);

long long g_cases = 0, g_bad = 0;

void check(wf::Vec3 lo, wf::Vec3 hi, wf::Vec3 o, wf::Vec3 inv, float tmin, float tmax) {
    ++g_cases;
    const bool want = wf::hit_box(lo, hi, o, inv, tmin, tmax);
    const bool got = wf::hit_box_minmax(lo, hi, o, inv, tmin, tmax);
    if (want != got && g_bad++ < 10)
        std::printf("mismatch: lo %g %g %g hi %g %g %g o %g %g %g inv %g %g %g tmin %g tmax %g want %d got %d\n", lo.x,
                    lo.y, lo.z, hi.x, hi.y, hi.z, o.x, o.y, o.z, inv.x, inv.y, inv.z, tmin, tmax, want, got);
}

}  // namespace

int main() {
    const float tmins[] = {wf::kRayEps, 0.0f, -0.0f, 1.0f};
    const float tmaxs[] = {wf::kInf, INFINITY, NAN, 0.0f, -0.0f, 1.0f, 2.5f, -1.0f, wf::kRayEps};
    // Exhaustive on x with y/z either neutral (the ray inside a wide slab) or special themselves.
    const wf::Vec3 wide_lo{-4.0f, -4.0f, -4.0f}, wide_hi{4.0f, 4.0f, 4.0f};
    for (float lx : kSpecial)
        for (float hx : kSpecial)
            for (float ox : kSpecial)
                for (float ix : kSpecial)
                    for (float tmin : tmins)
                        for (float tmax : tmaxs) {
                            check({lx, wide_lo.y, wide_lo.z}, {hx, wide_hi.y, wide_hi.z}, {ox, 0.5f, -0.5f},
                                  {ix, 0.75f, -2.0f}, tmin, tmax);
                            check({wide_lo.x, lx, wide_lo.z}, {wide_hi.x, wide_hi.y, hx}, {0.25f, ox, ox},
                                  {1.5f, ix, ix}, tmin, tmax);
                        }
    // Random mixing: each of the twelve components special (half the time) or a random bit pattern.
    std::mt19937_64 rng(20240613);
    auto pick = [&]() -> float {
        const uint64_t r = rng();
        if (r & 1) return kSpecial[(r >> 1) % kN];
        if (r & 2) return (float)((int64_t)(r >> 40) % 9 - 4) * 0.5f;  // small grid values: exact ties
        return bits((uint32_t)(r >> 32));
    };
    for (int i = 0; i < 6000000; ++i) {
        const wf::Vec3 lo{pick(), pick(), pick()}, hi{pick(), pick(), pick()}, o{pick(), pick(), pick()};
        const wf::Vec3 inv{pick(), pick(), pick()};
        check(lo, hi, o, inv, tmins[rng() % 4], (rng() & 1) ? tmaxs[rng() % 9] : pick());
    }
    std::printf("cases %lld mismatches %lld\n", g_cases, g_bad);
    return g_bad == 0 ? 0 : 1;
}
