// Wavefront OBJ loader (contract: WVM/src/obj_loader.cpp:49-186, tests WVM/tests/test_obj.cpp):
// `v x y z` and `f a b c ...` (1-based absolute indices, "i", "i/t", "i/t/n", "i//n"), fan
// triangulation, one grey Lambertian material, a camera looking down -z at the mesh from 1.5
// bounding-box diagonals, then finalize_scene. Other statements are ignored. Errors are
// std::runtime_error naming the file and, for a bad line, its 1-based number.
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "wf/scene.hpp"

namespace wf {
namespace {

// The file is read whole and parsed in place: a line is [p, end), tokens are runs of characters
// other than ' ', '\t' and '\r', and a '#' ends the line. Numbers are converted with strtof / strtol
// straight from the buffer (the buffer is NUL-terminated, and a token is always followed by a
// character that neither function consumes), so large meshes parse without a string per field.
bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

struct Token {
    const char* b = nullptr;
    const char* e = nullptr;
    bool is(const char* lit) const {
        const size_t n = std::strlen(lit);
        return (size_t)(e - b) == n && std::memcmp(b, lit, n) == 0;
    }
    std::string str() const { return std::string(b, e); }
};

// Splits [p, end) into at most `cap` tokens; returns the number of tokens found (which can be larger
// than `cap`: the rest are counted, not stored).
size_t tokenize(const char* p, const char* end, Token* out, size_t cap) {
    size_t n = 0;
    while (p < end) {
        while (p < end && is_space(*p)) ++p;
        const char* b = p;
        while (p < end && !is_space(*p)) ++p;
        if (p > b) {
            if (n < cap) out[n] = Token{b, p};
            ++n;
        }
    }
    return n;
}

bool whole_float(const Token& t, float* out) {
    if (t.b == t.e) return false;
    char* end = nullptr;
    errno = 0;
    const float v = std::strtof(t.b, &end);
    if (end != t.e) return false;
    *out = v;
    return true;
}

// The vertex index of a face token: the part before the first '/', a whole base-10 integer.
bool face_index(const Token& t, long* out) {
    const char* stop = static_cast<const char*>(std::memchr(t.b, '/', (size_t)(t.e - t.b)));
    if (!stop) stop = t.e;
    if (stop == t.b) return false;
    char* end = nullptr;
    errno = 0;
    const long v = std::strtol(t.b, &end, 10);
    if (end != stop || errno != 0) return false;
    *out = v;
    return true;
}

}  // namespace

Scene load_obj(const std::string& path, int width, int height) {
    std::string text;
    {
        std::ifstream in(path, std::ios::binary);
        if (!in) throw std::runtime_error("load_obj: cannot open " + path);
        in.seekg(0, std::ios::end);
        const std::streamoff size = in.tellg();
        in.seekg(0, std::ios::beg);
        if (size > 0) {
            text.resize((size_t)size);
            in.read(&text[0], size);
            text.resize((size_t)in.gcount());
        }
    }
    Scene s;
    s.name = path;
    s.width = width;
    s.height = height;
    auto fail = [&](int line, const std::string& what) {
        throw std::runtime_error(path + " line " + std::to_string(line) + ": " + what);
    };
    std::vector<Token> tok(64);
    std::vector<int> idx;
    const char* p = text.c_str();
    const char* const text_end = p + text.size();
    int n = 0;
    while (p < text_end) {  // lines as std::getline yields them: no empty line after a final '\n'
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(text_end - p)));
        const char* line_end = nl ? nl : text_end;
        const char* next = nl ? nl + 1 : text_end;
        ++n;
        const char* hash = static_cast<const char*>(std::memchr(p, '#', (size_t)(line_end - p)));
        if (hash) line_end = hash;
        size_t nt = tokenize(p, line_end, tok.data(), tok.size());
        if (nt > tok.size()) {  // a face with very many corners
            tok.resize(nt);
            nt = tokenize(p, line_end, tok.data(), tok.size());
        }
        p = next;
        if (nt == 0) continue;
        if (tok[0].is("v")) {
            if (nt != 4) fail(n, "a vertex needs exactly 3 coordinates");
            Vec3 v;
            if (!whole_float(tok[1], &v.x) || !whole_float(tok[2], &v.y) || !whole_float(tok[3], &v.z))
                fail(n, "malformed vertex coordinate");
            s.vertices.push_back(v);
        } else if (tok[0].is("f")) {
            if (nt < 4) fail(n, "a face needs at least 3 indices");
            idx.clear();
            for (size_t k = 1; k < nt; ++k) {
                long v = 0;
                if (!face_index(tok[k], &v)) fail(n, "malformed face index '" + tok[k].str() + "'");
                if (v < 1 || v > (long)s.vertices.size())
                    fail(n, "face index " + std::to_string(v) + " outside 1.." + std::to_string(s.vertices.size()));
                idx.push_back((int)v - 1);
            }
            for (size_t k = 1; k + 1 < idx.size(); ++k)
                s.triangles.push_back(Triangle{idx[0], idx[k], idx[k + 1], 0});
        }
    }
    if (s.triangles.empty()) throw std::runtime_error(path + ": no faces");

    Material grey{};
    grey.type = kLambert;
    grey.ior = 1.5f;
    grey.albedo = Vec3{0.7f, 0.7f, 0.7f};
    s.materials.push_back(grey);

    Vec3 lo = s.vertices[0], hi = s.vertices[0];
    for (const Vec3& v : s.vertices) {
        lo = vmin(lo, v);
        hi = vmax(hi, v);
    }
    const Vec3 centre = (lo + hi) * 0.5f;
    const float diag = length(hi - lo);
    s.camera.position = centre + Vec3{0.0f, 0.0f, diag * 1.5f};
    s.camera.look_at = centre;
    s.camera.up = Vec3{0.0f, 1.0f, 0.0f};
    s.camera.vfov_deg = 45.0f;
    finalize_scene(s);
    return s;
}

}  // namespace wf
