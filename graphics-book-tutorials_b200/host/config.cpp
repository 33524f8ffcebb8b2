// `render` flag parser (contract: WVM/include/wf/config.hpp:30-34, WVM/src/config.cpp:62-175).
#include <cerrno>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <string>
#include "wf/config.hpp"

namespace wf {
namespace {

// Whole-token decimal integer in [lo, hi]; false for empty, partial or out-of-range text.
bool to_long(const char* s, long long lo, long long hi, long long* out) {
    if (s == nullptr || *s == '\0') return false;
    errno = 0;
    char* end = nullptr;
    const long long v = std::strtoll(s, &end, 10);
    if (errno != 0 || end == s || *end != '\0' || v < lo || v > hi) return false;
    *out = v;
    return true;
}

int int_flag(const std::string& flag, const char* value, int lo, int hi, const char* range) {
    long long v = 0;
    if (!to_long(value, INT_MIN, INT_MAX, &v)) throw ConfigError(flag + ": expected an integer, got '" + value + "'");
    if (v < lo || v > hi) throw ConfigError(flag + ": " + value + " is outside " + range);
    return (int)v;
}

}  // namespace

std::string usage() {
    return "Usage: render [--scene NAME|FILE.obj] [--width W] [--height H] [--spp N] [--seed S]\n"
           "              [--max-depth D] [--mode cpu|megakernel|wavefront] [--report PATH]\n"
           "              [--out PREFIX] [--threads N] [--reps N] [--warmup N]\n"
           "Defaults: --scene cornell --width 1280 --height 720 --spp 64 --seed 1234 --max-depth 8\n"
           "          --mode wavefront --threads 0 (all cores) --reps 1 --warmup 0; no report, no images.\n"
           "--report writes report.json (schema 1); --out writes PREFIX.png and PREFIX.pfm.\n";
}

std::string mode_name(Mode m) {
    switch (m) {
        case Mode::Cpu: return "cpu";
        case Mode::Megakernel: return "megakernel";
        case Mode::Wavefront: return "wavefront";
    }
    return "unknown";
}

Config parse_args(int argc, const char* const* argv) {
    if (argc < 2 || argv[1] == nullptr || std::strcmp(argv[1], "render") != 0)
        throw ConfigError("the first argument must be \"render\"");
    Config c;
    for (int i = 2; i < argc; ++i) {
        const std::string flag = argv[i];
        const bool known = flag == "--scene" || flag == "--width" || flag == "--height" || flag == "--spp" ||
                           flag == "--seed" || flag == "--max-depth" || flag == "--mode" || flag == "--report" ||
                           flag == "--out" || flag == "--threads" || flag == "--reps" || flag == "--warmup";
        if (!known) throw ConfigError(flag + ": unknown flag");
        if (i + 1 >= argc) throw ConfigError(flag + ": missing value");
        const char* v = argv[++i];
        if (flag == "--scene") {
            c.scene = v;
        } else if (flag == "--width") {
            c.width = int_flag(flag, v, 1, 8192, "1..8192");
        } else if (flag == "--height") {
            c.height = int_flag(flag, v, 1, 8192, "1..8192");
        } else if (flag == "--spp") {
            c.spp = int_flag(flag, v, 1, INT_MAX, "1 or more");
        } else if (flag == "--seed") {
            long long s = 0;
            if (!to_long(v, 0, UINT_MAX, &s)) throw ConfigError(flag + ": expected an unsigned integer, got '" + v + "'");
            c.seed = (unsigned)s;
        } else if (flag == "--max-depth") {
            c.max_depth = int_flag(flag, v, 1, 64, "1..64");
        } else if (flag == "--mode") {
            const std::string m = v;
            if (m == "cpu") c.mode = Mode::Cpu;
            else if (m == "megakernel") c.mode = Mode::Megakernel;
            else if (m == "wavefront") c.mode = Mode::Wavefront;
            else throw ConfigError(flag + ": unknown mode '" + m + "' (cpu, megakernel or wavefront)");
        } else if (flag == "--report") {
            c.report_path = v;
        } else if (flag == "--out") {
            c.out_prefix = v;
        } else if (flag == "--threads") {
            c.threads = int_flag(flag, v, INT_MIN, INT_MAX, "int");
        } else if (flag == "--reps") {
            c.reps = int_flag(flag, v, 1, INT_MAX, "1 or more");
        } else {  // --warmup
            c.warmup = int_flag(flag, v, 0, INT_MAX, "0 or more");
        }
    }
    return c;
}

}  // namespace wf
