// report.json, schema version 1: writer, validator and the percentile helper. Same types and
// functions as the reference's WVM/include/wf/report.hpp:9-54 (the schema is an interface the
// reference's scripts read, so it is kept key for key).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace wf {

constexpr int kReportSchemaVersion = 1;

struct DeviceInfo {
    std::string name = "cpu";
    std::string driver_version;
    std::string cuda_runtime_version;
    std::string cuda_driver_version;
    std::string compute_capability;
    uint64_t total_memory_bytes = 0;
};

struct Report {
    std::string git_revision;  // empty: written as null
    std::string scene_name;
    uint64_t scene_hash = 0;
    int width = 0, height = 0, spp = 0, max_depth = 0;
    unsigned seed = 0;
    std::string mode;  // cpu | megakernel | wavefront
    DeviceInfo device;
    std::vector<double> run_ms;
    double samples_per_second = 0.0;
    double rays_per_second = 0.0;  // 0: written as null
    uint64_t peak_vram_bytes = 0;
    long long queue_high_water[5] = {0, 0, 0, 0, 0};  // lambert, metal, dielectric, shadow, active
    std::string image_png, image_pfm;
    uint64_t pfm_hash = 0;
    long long nonfinite_pixels = 0, queue_overflows = 0, invalid_hits = 0;
};

// Linear interpolation between order statistics; p in [0, 1]. Throws on empty input.
double percentile(std::vector<double> v, double p);

// Keys: schema_version, git_revision, scene{name,hash}, config{width,height,spp,seed,max_depth,mode},
// device{name,driver_version,cuda_runtime_version,cuda_driver_version,compute_capability,
// total_memory_bytes}, timings_ms{runs[],min,median,p10,p90,max},
// throughput{samples_per_second,rays_per_second}, peak_vram_bytes,
// queue_high_water{lambert,metal,dielectric,shadow,active}, outputs{png,pfm,pfm_hash},
// validity{nonfinite_pixels,queue_overflows,invalid_hits}; hashes as 16 lowercase hex digits.
std::string report_to_json(const Report& r);

// "" when `json_text` is one JSON object of that schema (every key present with its type; null
// only for git_revision and rays_per_second; schema_version 1; runs non-empty; min <= median <=
// max; hashes 16 hex digits), else the first problem found.
std::string validate_report_json(const std::string& json_text);

}  // namespace wf
