// Render results and image comparison (host). API surface of WVM/include/wf/film.hpp:11-33.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "wf/math.hpp"

namespace wf {

struct RenderResult {
    int width = 0, height = 0, spp = 0;
    std::vector<float> rgb;      // 3*w*h mean radiance
    std::vector<float> lum_var;  // w*h per-pixel variance of per-sample luminance
};

// exposure, Reinhard x/(1+x), sRGB transfer, 8-bit.
std::vector<uint8_t> tonemap_to_srgb8(const std::vector<float>& rgb, float exposure = 1.0f);
// Pixels with any non-finite channel.
int count_nonfinite(const std::vector<float>& rgb);

struct ImageDiff {
    double max_abs_rel = 0.0;      // max |a-b| / max(|a|,|b|,1e-6) over finite channels
    double mean_rel = 0.0;         // |mean lum(a) - mean lum(b)| / max(mean lum(a), 1e-12)
    double frac_within_3se = 0.0;  // pixels with |lum a - lum b| <= 3 sqrt(se_a^2 + se_b^2)
    int nonfinite = 0;             // non-finite channels over both images
};
// se = sqrt(lum_var / spp); throws std::invalid_argument on a size mismatch.
ImageDiff compare_results(const RenderResult& a, const RenderResult& b);

}  // namespace wf
