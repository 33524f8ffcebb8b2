// Wavefront OBJ loader (contract: WVM/src/obj_loader.cpp:49-186, tests WVM/tests/test_obj.cpp):
// `v x y z` and `f a b c ...` (1-based absolute indices, "i", "i/t", "i/t/n", "i//n"), fan
// triangulation, one grey Lambertian material, a camera looking down -z at the mesh from 1.5
// bounding-box diagonals, then finalize_scene. Other statements are ignored. Errors are
// std::runtime_error naming the file and, for a bad line, its 1-based number.
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <thread>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "wf/scene.hpp"

namespace wf {
namespace {

// The file is read whole and parsed in place (in chunks of whole lines on several threads for large
// files): a line is [p, end), tokens are runs of characters
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

// A run of whole lines parsed on its own: vertices and fan triangles in file order, or the first
// error (its 1-based line number and message). `first_line` and `vertex_base` are the number of
// lines and of `v` statements before the run, so indices and messages are those of a serial parse.
struct Chunk {
    const char* b = nullptr;
    const char* e = nullptr;
    int first_line = 0, lines = 0;
    size_t vertex_base = 0, v_lines = 0;
    std::vector<Vec3> vertices;
    std::vector<Triangle> triangles;
    int error_line = 0;
    std::string error;
};

// Calls fn(line_begin, line_end_before_comment) for every line of [p, end), as std::getline would
// split them (no empty line after a final '\n'); stops early when fn returns false.
template <class F>
void for_lines(const char* p, const char* end, F&& fn) {
    while (p < end) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        const char* line_end = nl ? nl : end;
        const char* next = nl ? nl + 1 : end;
        const char* hash = static_cast<const char*>(std::memchr(p, '#', (size_t)(line_end - p)));
        if (!fn(p, hash ? hash : line_end)) return;
        p = next;
    }
}

void parse_chunk(Chunk& c) {
    std::vector<Token> tok(64);
    std::vector<int> idx;
    int n = c.first_line;
    auto fail = [&](const std::string& what) {
        c.error_line = n;
        c.error = what;
        return false;
    };
    for_lines(c.b, c.e, [&](const char* p, const char* line_end) {
        ++n;
        size_t nt = tokenize(p, line_end, tok.data(), tok.size());
        if (nt > tok.size()) {  // a face with very many corners
            tok.resize(nt);
            nt = tokenize(p, line_end, tok.data(), tok.size());
        }
        if (nt == 0) return true;
        if (tok[0].is("v")) {
            if (nt != 4) return fail("a vertex needs exactly 3 coordinates");
            Vec3 v;
            if (!whole_float(tok[1], &v.x) || !whole_float(tok[2], &v.y) || !whole_float(tok[3], &v.z))
                return fail("malformed vertex coordinate");
            c.vertices.push_back(v);
        } else if (tok[0].is("f")) {
            if (nt < 4) return fail("a face needs at least 3 indices");
            const long seen = (long)(c.vertex_base + c.vertices.size());
            idx.clear();
            for (size_t k = 1; k < nt; ++k) {
                long v = 0;
                if (!face_index(tok[k], &v)) return fail("malformed face index '" + tok[k].str() + "'");
                if (v < 1 || v > seen) return fail("face index " + std::to_string(v) + " outside 1.." + std::to_string(seen));
                idx.push_back((int)v - 1);
            }
            for (size_t k = 1; k + 1 < idx.size(); ++k) c.triangles.push_back(Triangle{idx[0], idx[k], idx[k + 1], 0});
        }
        return true;
    });
}

// Lines and `v` statements of a chunk (the offsets of the chunks after it).
void count_chunk(Chunk& c) {
    for_lines(c.b, c.e, [&](const char* p, const char* line_end) {
        ++c.lines;
        while (p < line_end && is_space(*p)) ++p;
        if (p < line_end && *p == 'v' && (p + 1 == line_end || is_space(p[1]))) ++c.v_lines;
        return true;
    });
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
    // Large files are cut at line boundaries into one chunk per core: a counting pass gives each
    // chunk its line and vertex offsets, then the chunks parse side by side.
    const char* const text_begin = text.c_str();
    const char* const text_end = text_begin + text.size();
    constexpr size_t kChunkMin = 4u << 20;
    const size_t cores = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t n_chunks = std::max<size_t>(1, std::min(cores, text.size() / kChunkMin));
    std::vector<Chunk> chunks(n_chunks);
    const char* p = text_begin;
    for (size_t k = 0; k < n_chunks; ++k) {
        const char* e = k + 1 == n_chunks ? text_end : text_begin + text.size() * (k + 1) / n_chunks;
        if (e < p) e = p;
        if (e < text_end) {  // extend to the end of the line
            const char* nl = static_cast<const char*>(std::memchr(e, '\n', (size_t)(text_end - e)));
            e = nl ? nl + 1 : text_end;
        }
        chunks[k].b = p;
        chunks[k].e = e;
        p = e;
    }
    auto run_all = [&](void (*fn)(Chunk&)) {
        if (n_chunks == 1) {
            fn(chunks[0]);
            return;
        }
        std::vector<std::thread> threads;
        for (size_t k = 1; k < n_chunks; ++k) threads.emplace_back([&, k] { fn(chunks[k]); });
        fn(chunks[0]);
        for (auto& t : threads) t.join();
    };
    if (n_chunks > 1) {
        run_all(count_chunk);
        for (size_t k = 1; k < n_chunks; ++k) {
            chunks[k].first_line = chunks[k - 1].first_line + chunks[k - 1].lines;
            chunks[k].vertex_base = chunks[k - 1].vertex_base + chunks[k - 1].v_lines;
        }
    }
    run_all(parse_chunk);
    size_t nv = 0, ntri = 0;
    for (const Chunk& c : chunks) {
        if (!c.error.empty()) throw std::runtime_error(path + " line " + std::to_string(c.error_line) + ": " + c.error);
        nv += c.vertices.size();
        ntri += c.triangles.size();
    }
    s.vertices.reserve(nv);
    s.triangles.reserve(ntri);
    for (const Chunk& c : chunks) {
        s.vertices.insert(s.vertices.end(), c.vertices.begin(), c.vertices.end());
        s.triangles.insert(s.triangles.end(), c.triangles.begin(), c.triangles.end());
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
