// Minimal JSON value with a strict parser (RFC 8259) and a string escaper: the API of the
// reference's WVM/include/wf/json.hpp:9-30, used by the report validator and its tests.
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace wf {

struct Json {
    enum Type { Null, Bool, Number, String, Array, Object } type = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    bool has(const std::string& k) const { return type == Object && obj.count(k) > 0; }
    const Json& at(const std::string& k) const { return obj.at(k); }
};

// Parses one JSON document; std::runtime_error (with the byte offset) on any malformed input,
// trailing garbage included. \uXXXX escapes decode to UTF-8.
Json json_parse(const std::string& text);
// The body of a JSON string literal for `s` (no surrounding quotes).
std::string json_escape(const std::string& s);

}  // namespace wf
