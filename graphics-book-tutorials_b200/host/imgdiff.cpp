// `imgdiff A.pfm B.pfm [--tol T]`: the reference's image comparison tool (command line, output and
// exit codes of WVM/tools/imgdiff.cpp) on this engine's PFM reader.
//
// Over the pixel components where both images are finite it reports
//   max_abs_rel = max |a - b| / max(|a|, |b|)   (components with max(|a|, |b|) <= 1e-20 skipped)
//   mean_rel    = |sum a - sum b| / sum a        (0 when sum a <= 1e-12)
// printed with 17 significant digits. A non-finite component must equal its counterpart exactly
// (so a NaN never matches). Exit 0 when max_abs_rel <= T (default 1e-5), 1 when it is larger,
// 2 on a usage error, unreadable or mismatched images, or a non-finite mismatch.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>
#include "wf/image_io.hpp"

namespace {

struct Diff {
    double max_abs_rel = 0.0, mean_rel = 0.0;
    bool nonfinite_mismatch = false;
};

Diff compare(const std::vector<float>& x, const std::vector<float>& y) {
    Diff d;
    double sum_x = 0.0, sum_y = 0.0;
    for (size_t i = 0; i < x.size(); ++i) {
        const float a = x[i], b = y[i];
        if (!std::isfinite(a) || !std::isfinite(b)) {
            if (!(a == b)) {
                d.nonfinite_mismatch = true;
                return d;
            }
            continue;
        }
        sum_x += a;
        sum_y += b;
        const double scale = std::max(std::fabs((double)a), std::fabs((double)b));
        if (scale > 1e-20) d.max_abs_rel = std::max(d.max_abs_rel, std::fabs((double)a - (double)b) / scale);
    }
    if (sum_x > 1e-12) d.mean_rel = std::fabs(sum_x - sum_y) / sum_x;
    return d;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc < 3) {
            std::cerr << "Usage: imgdiff <img1> <img2> [--tol <tolerance>]\n";
            return 2;
        }
        double tol = 1e-5;
        for (int i = 3; i < argc; ++i) {
            const std::string arg = argv[i];
            if (arg == "--tol" && i + 1 < argc) {
                tol = std::stod(argv[++i]);
            } else {
                std::cerr << "Unknown option: " << arg << "\n";
                return 2;
            }
        }
        int w1 = 0, h1 = 0, w2 = 0, h2 = 0;
        const std::vector<float> x = wf::read_pfm(argv[1], &w1, &h1);
        const std::vector<float> y = wf::read_pfm(argv[2], &w2, &h2);
        if (w1 != w2 || h1 != h2) {
            std::cerr << "Image dimensions mismatch\n";
            return 2;
        }
        if (x.size() != y.size()) {
            std::cerr << "Image size mismatch\n";
            return 2;
        }
        const Diff d = compare(x, y);
        if (d.nonfinite_mismatch) {
            std::cerr << "Non-finite pixel mismatch\n";
            return 2;
        }
        std::printf("max_abs_rel=%.17g\n", d.max_abs_rel);
        std::printf("mean_rel=%.17g\n", d.mean_rel);
        return d.max_abs_rel <= tol ? 0 : 1;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 2;
    }
}
