// Tone mapping and image comparison on the host (API: WVM/include/wf/film.hpp:16-33).
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include "wf/film.hpp"

namespace wf {

std::vector<uint8_t> tonemap_to_srgb8(const std::vector<float>& rgb, float exposure) {
    std::vector<uint8_t> out(rgb.size());
    for (size_t i = 0; i < rgb.size(); ++i) {
        const double y = (double)rgb[i] * (double)exposure;
        double r = y / (1.0 + y);  // Reinhard
        if (!(r > 0.0)) r = 0.0;   // negatives and NaN to black
        if (r > 1.0) r = 1.0;
        const double s = r <= 0.0031308 ? 12.92 * r : 1.055 * std::pow(r, 1.0 / 2.4) - 0.055;  // sRGB transfer
        out[i] = (uint8_t)std::clamp(std::lround(255.0 * s), 0L, 255L);
    }
    return out;
}

int count_nonfinite(const std::vector<float>& rgb) {
    int n = 0;
    for (size_t p = 0; p + 2 < rgb.size(); p += 3)
        n += !(std::isfinite(rgb[p]) && std::isfinite(rgb[p + 1]) && std::isfinite(rgb[p + 2]));
    return n;
}

ImageDiff compare_results(const RenderResult& a, const RenderResult& b) {
    if (a.width != b.width || a.height != b.height)
        throw std::invalid_argument("compare_results: images of different dimensions");
    const size_t n = (size_t)a.width * (size_t)a.height;
    if (a.rgb.size() < 3 * n || b.rgb.size() < 3 * n || a.lum_var.size() < n || b.lum_var.size() < n)
        throw std::invalid_argument("compare_results: buffers smaller than width x height");
    ImageDiff d;
    double sum_a = 0.0, sum_b = 0.0;
    size_t within = 0;
    for (size_t p = 0; p < n; ++p) {
        const Vec3 ca{a.rgb[3 * p], a.rgb[3 * p + 1], a.rgb[3 * p + 2]};
        const Vec3 cb{b.rgb[3 * p], b.rgb[3 * p + 1], b.rgb[3 * p + 2]};
        for (int k = 0; k < 3; ++k) {
            const float x = a.rgb[3 * p + k], y = b.rgb[3 * p + k];
            d.nonfinite += !std::isfinite(x);
            d.nonfinite += !std::isfinite(y);
            if (std::isfinite(x) && std::isfinite(y)) {
                const double den = std::max({(double)std::fabs(x), (double)std::fabs(y), 1e-6});
                d.max_abs_rel = std::max(d.max_abs_rel, std::fabs((double)x - (double)y) / den);
            }
        }
        const double la = luminance(ca), lb = luminance(cb);
        sum_a += la;
        sum_b += lb;
        const double sea2 = (double)a.lum_var[p] / (double)a.spp, seb2 = (double)b.lum_var[p] / (double)b.spp;
        if (std::isfinite(la) && std::isfinite(lb) && std::fabs(la - lb) <= 3.0 * std::sqrt(sea2 + seb2)) ++within;
    }
    if (n > 0) {
        const double ma = sum_a / (double)n, mb = sum_b / (double)n;
        d.mean_rel = std::fabs(ma - mb) / std::max(ma, 1e-12);
        d.frac_within_3se = (double)within / (double)n;
    }
    return d;
}

}  // namespace wf
