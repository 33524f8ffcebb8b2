// `render` command-line configuration. Same types and functions as the reference's
// WVM/include/wf/config.hpp:8-37, so its CLI tests link against this host library.
#pragma once
#include <stdexcept>
#include <string>

namespace wf {

enum class Mode { Cpu, Megakernel, Wavefront };

struct Config {
    std::string scene = "cornell";  // procedural scene name, or a path ending in .obj
    int width = 1280, height = 720;
    int spp = 64;
    unsigned seed = 1234;
    int max_depth = 8;
    Mode mode = Mode::Wavefront;
    std::string report_path;  // --report PATH; empty: no report
    std::string out_prefix;   // --out PREFIX: PREFIX.png and PREFIX.pfm
    int threads = 0;          // CPU arm threads (0: all)
    int reps = 1;             // timed repetitions
    int warmup = 0;           // untimed renders first
};

struct ConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// argv[1] must be "render"; then any of --scene --width --height --spp --seed --max-depth --mode
// --report --out --threads --reps --warmup, each followed by its value, in any order (the last
// occurrence wins). Throws ConfigError naming the flag for an unknown flag, a missing or
// non-numeric value, width/height outside 1..8192, spp < 1, max-depth outside 1..64, reps < 1,
// warmup < 0 or an unknown mode.
Config parse_args(int argc, const char* const* argv);
std::string usage();
std::string mode_name(Mode m);  // "cpu", "megakernel", "wavefront"

}  // namespace wf
