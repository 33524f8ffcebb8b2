// report.json v1 writer and validator (schema: WVM/include/wf/report.hpp:41-54).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include "wf/image_io.hpp"
#include "wf/json.hpp"
#include "wf/report.hpp"

namespace wf {

double percentile(std::vector<double> v, double p) {
    if (v.empty()) throw std::invalid_argument("percentile of an empty sample");
    std::sort(v.begin(), v.end());
    const double q = std::min(1.0, std::max(0.0, p)) * (double)(v.size() - 1);
    const size_t i = (size_t)std::floor(q);
    if (i + 1 >= v.size()) return v.back();
    const double f = q - (double)i;
    return v[i] + (v[i + 1] - v[i]) * f;
}

namespace {

std::string num(double x) {
    if (!std::isfinite(x)) return "null";
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", x);
    return buf;
}
std::string num(long long x) { return std::to_string(x); }
std::string num(uint64_t x) { return std::to_string(x); }
std::string str(const std::string& s) { return "\"" + json_escape(s) + "\""; }

// Writes `{"k": v, ...}` from key/value-text pairs.
std::string object(std::initializer_list<std::pair<const char*, std::string>> kv, int indent) {
    const std::string pad((size_t)indent + 2, ' '), end_pad((size_t)indent, ' ');
    std::string o = "{\n";
    size_t n = 0;
    for (const auto& [k, v] : kv) {
        o += pad + "\"" + k + "\": " + v;
        o += ++n < kv.size() ? ",\n" : "\n";
    }
    return o + end_pad + "}";
}

}  // namespace

std::string report_to_json(const Report& r) {
    std::string runs = "[";
    for (size_t i = 0; i < r.run_ms.size(); ++i) runs += (i ? ", " : "") + num(r.run_ms[i]);
    runs += "]";
    const bool have = !r.run_ms.empty();
    const double mn = have ? *std::min_element(r.run_ms.begin(), r.run_ms.end()) : 0.0;
    const double mx = have ? *std::max_element(r.run_ms.begin(), r.run_ms.end()) : 0.0;
    const double md = have ? percentile(r.run_ms, 0.5) : 0.0;
    const double p10 = have ? percentile(r.run_ms, 0.1) : 0.0;
    const double p90 = have ? percentile(r.run_ms, 0.9) : 0.0;
    const auto& q = r.queue_high_water;
    return object(
               {{"schema_version", num((long long)kReportSchemaVersion)},
                {"git_revision", r.git_revision.empty() ? "null" : str(r.git_revision)},
                {"scene", object({{"name", str(r.scene_name)}, {"hash", str(hex64(r.scene_hash))}}, 2)},
                {"config", object({{"width", num((long long)r.width)},
                                   {"height", num((long long)r.height)},
                                   {"spp", num((long long)r.spp)},
                                   {"seed", num((long long)r.seed)},
                                   {"max_depth", num((long long)r.max_depth)},
                                   {"mode", str(r.mode)}},
                                  2)},
                {"device", object({{"name", str(r.device.name)},
                                   {"driver_version", str(r.device.driver_version)},
                                   {"cuda_runtime_version", str(r.device.cuda_runtime_version)},
                                   {"cuda_driver_version", str(r.device.cuda_driver_version)},
                                   {"compute_capability", str(r.device.compute_capability)},
                                   {"total_memory_bytes", num(r.device.total_memory_bytes)}},
                                  2)},
                {"timings_ms", object({{"runs", runs},
                                       {"min", num(mn)},
                                       {"median", num(md)},
                                       {"p10", num(p10)},
                                       {"p90", num(p90)},
                                       {"max", num(mx)}},
                                      2)},
                {"throughput", object({{"samples_per_second", num(r.samples_per_second)},
                                       {"rays_per_second", r.rays_per_second > 0.0 ? num(r.rays_per_second) : "null"}},
                                      2)},
                {"peak_vram_bytes", num(r.peak_vram_bytes)},
                {"queue_high_water", object({{"lambert", num(q[0])},
                                             {"metal", num(q[1])},
                                             {"dielectric", num(q[2])},
                                             {"shadow", num(q[3])},
                                             {"active", num(q[4])}},
                                            2)},
                {"outputs", object({{"png", str(r.image_png)},
                                    {"pfm", str(r.image_pfm)},
                                    {"pfm_hash", str(hex64(r.pfm_hash))}},
                                   2)},
                {"validity", object({{"nonfinite_pixels", num(r.nonfinite_pixels)},
                                     {"queue_overflows", num(r.queue_overflows)},
                                     {"invalid_hits", num(r.invalid_hits)}},
                                    2)}},
               0) +
           "\n";
}

namespace {

enum class Kind { Number, String, HexString, NumberOrNull, StringOrNull, NumberArray, Object };

struct Field {
    const char* key;
    Kind kind;
};

bool is_hex16(const std::string& s) {
    if (s.size() != 16) return false;
    for (const char c : s)
        if (!((c >= '0' && c <= '9') || (c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F'))) return false;
    return true;
}

// "" when `v` has kind `k`, else the problem.
std::string check(const Json& v, Kind k, const std::string& where) {
    switch (k) {
        case Kind::Number:
            return v.type == Json::Number ? "" : where + " must be a number";
        case Kind::String:
            return v.type == Json::String ? "" : where + " must be a string";
        case Kind::HexString:
            if (v.type != Json::String) return where + " must be a string";
            return is_hex16(v.str) ? "" : where + " must be 16 hex digits";
        case Kind::NumberOrNull:
            return v.type == Json::Number || v.type == Json::Null ? "" : where + " must be a number or null";
        case Kind::StringOrNull:
            return v.type == Json::String || v.type == Json::Null ? "" : where + " must be a string or null";
        case Kind::NumberArray:
            if (v.type != Json::Array) return where + " must be an array";
            for (const Json& e : v.arr)
                if (e.type != Json::Number) return where + " must hold numbers only";
            return "";
        case Kind::Object:
            return v.type == Json::Object ? "" : where + " must be an object";
    }
    return where + ": unknown kind";
}

std::string check_fields(const Json& obj, const std::string& prefix, std::initializer_list<Field> fields) {
    for (const Field& f : fields) {
        const std::string where = prefix.empty() ? f.key : prefix + "." + f.key;
        if (!obj.has(f.key)) return "missing key " + where;
        const std::string p = check(obj.at(f.key), f.kind, where);
        if (!p.empty()) return p;
    }
    return "";
}

}  // namespace

std::string validate_report_json(const std::string& json_text) {
    Json j;
    try {
        j = json_parse(json_text);
    } catch (const std::exception& e) {
        return std::string("not valid JSON: ") + e.what();
    }
    if (j.type != Json::Object) return "the document is not a JSON object";
    std::string p = check_fields(j, "", {{"schema_version", Kind::Number}, {"git_revision", Kind::StringOrNull},
                                         {"scene", Kind::Object}, {"config", Kind::Object}, {"device", Kind::Object},
                                         {"timings_ms", Kind::Object}, {"throughput", Kind::Object},
                                         {"peak_vram_bytes", Kind::Number}, {"queue_high_water", Kind::Object},
                                         {"outputs", Kind::Object}, {"validity", Kind::Object}});
    if (!p.empty()) return p;
    if (j.at("schema_version").num != (double)kReportSchemaVersion)
        return "schema_version must be " + std::to_string(kReportSchemaVersion);
    if (!(p = check_fields(j.at("scene"), "scene", {{"name", Kind::String}, {"hash", Kind::HexString}})).empty())
        return p;
    if (!(p = check_fields(j.at("config"), "config",
                           {{"width", Kind::Number}, {"height", Kind::Number}, {"spp", Kind::Number},
                            {"seed", Kind::Number}, {"max_depth", Kind::Number}, {"mode", Kind::String}}))
             .empty())
        return p;
    if (!(p = check_fields(j.at("device"), "device",
                           {{"name", Kind::String}, {"driver_version", Kind::String},
                            {"cuda_runtime_version", Kind::String}, {"cuda_driver_version", Kind::String},
                            {"compute_capability", Kind::String}, {"total_memory_bytes", Kind::Number}}))
             .empty())
        return p;
    const Json& t = j.at("timings_ms");
    if (!(p = check_fields(t, "timings_ms",
                           {{"runs", Kind::NumberArray}, {"min", Kind::Number}, {"median", Kind::Number},
                            {"p10", Kind::Number}, {"p90", Kind::Number}, {"max", Kind::Number}}))
             .empty())
        return p;
    if (t.at("runs").arr.empty()) return "timings_ms.runs must not be empty";
    if (t.at("min").num > t.at("median").num) return "timings_ms.min exceeds timings_ms.median";
    if (t.at("median").num > t.at("max").num) return "timings_ms.median exceeds timings_ms.max";
    if (!(p = check_fields(j.at("throughput"), "throughput",
                           {{"samples_per_second", Kind::Number}, {"rays_per_second", Kind::NumberOrNull}}))
             .empty())
        return p;
    if (!(p = check_fields(j.at("queue_high_water"), "queue_high_water",
                           {{"lambert", Kind::Number}, {"metal", Kind::Number}, {"dielectric", Kind::Number},
                            {"shadow", Kind::Number}, {"active", Kind::Number}}))
             .empty())
        return p;
    if (!(p = check_fields(j.at("outputs"), "outputs",
                           {{"png", Kind::String}, {"pfm", Kind::String}, {"pfm_hash", Kind::HexString}}))
             .empty())
        return p;
    if (!(p = check_fields(j.at("validity"), "validity",
                           {{"nonfinite_pixels", Kind::Number}, {"queue_overflows", Kind::Number},
                            {"invalid_hits", Kind::Number}}))
             .empty())
        return p;
    return "";
}

}  // namespace wf
