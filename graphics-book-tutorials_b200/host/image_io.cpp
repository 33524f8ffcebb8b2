// PNG (stored deflate) and PFM files, FNV-1a 64 (API: WVM/include/wf/image_io.hpp).
// Files are written to "<path>.tmp" and renamed into place, so a failed write leaves no file.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include "wf/image_io.hpp"

namespace wf {
namespace {

uint32_t crc32_update(uint32_t crc, const uint8_t* p, size_t n) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        init = true;
    }
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return crc;
}

void put_be32(std::vector<uint8_t>& o, uint32_t v) {
    o.push_back((uint8_t)(v >> 24));
    o.push_back((uint8_t)(v >> 16));
    o.push_back((uint8_t)(v >> 8));
    o.push_back((uint8_t)v);
}

void chunk(std::vector<uint8_t>& out, const char type[4], const std::vector<uint8_t>& data) {
    put_be32(out, (uint32_t)data.size());
    const size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    const uint32_t crc = crc32_update(0xFFFFFFFFu, out.data() + start, out.size() - start) ^ 0xFFFFFFFFu;
    put_be32(out, crc);
}

// Writes `bytes` to `path` through a temporary file renamed into place.
void write_file(const std::string& path, const char* what, const void* bytes, size_t n) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) throw std::runtime_error(std::string(what) + ": cannot open " + path + " for writing");
        f.write(static_cast<const char*>(bytes), (std::streamsize)n);
        f.flush();
        if (!f) {
            f.close();
            std::remove(tmp.c_str());
            throw std::runtime_error(std::string(what) + ": write to " + path + " failed");
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw std::runtime_error(std::string(what) + ": cannot move the file into " + path);
    }
}

}  // namespace

void write_png(const std::string& path, int width, int height, const std::vector<uint8_t>& rgb8) {
    if (width <= 0 || height <= 0) throw std::runtime_error("write_png: width and height must be positive");
    const size_t row = 3 * (size_t)width;
    if (rgb8.size() != row * (size_t)height)
        throw std::runtime_error("write_png: pixel buffer holds " + std::to_string(rgb8.size()) + " bytes, expected " +
                                 std::to_string(row * (size_t)height));
    // raw scanlines, each prefixed with filter type 0
    std::vector<uint8_t> raw;
    raw.reserve((row + 1) * (size_t)height);
    for (int y = 0; y < height; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgb8.begin() + (ptrdiff_t)(row * (size_t)y), rgb8.begin() + (ptrdiff_t)(row * (size_t)(y + 1)));
    }
    // zlib: CMF/FLG (deflate, 32K window, no dictionary, check bits), stored blocks, Adler-32
    std::vector<uint8_t> z = {0x78, 0x01};
    size_t pos = 0;
    do {
        const size_t len = std::min<size_t>(65535, raw.size() - pos);
        const bool last = pos + len == raw.size();
        z.push_back(last ? 1 : 0);  // BFINAL, BTYPE = 00
        z.push_back((uint8_t)(len & 0xFF));
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)(~len & 0xFF));
        z.push_back((uint8_t)((~len >> 8) & 0xFF));
        z.insert(z.end(), raw.begin() + (ptrdiff_t)pos, raw.begin() + (ptrdiff_t)(pos + len));
        pos += len;
    } while (pos < raw.size());
    uint32_t a = 1, b = 0;
    for (const uint8_t v : raw) {
        a = (a + v) % 65521u;
        b = (b + a) % 65521u;
    }
    put_be32(z, (b << 16) | a);

    std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit, truecolour, deflate, filter 0, no interlace
    chunk(out, "IHDR", ihdr);
    chunk(out, "IDAT", z);
    chunk(out, "IEND", {});
    write_file(path, "write_png", out.data(), out.size());
}

void write_pfm(const std::string& path, int width, int height, const std::vector<float>& rgb) {
    if (width <= 0 || height <= 0) throw std::runtime_error("write_pfm: width and height must be positive");
    const size_t row = 3 * (size_t)width;
    if (rgb.size() != row * (size_t)height) throw std::runtime_error("write_pfm: pixel buffer size mismatch");
    const std::string header = "PF\n" + std::to_string(width) + " " + std::to_string(height) + "\n-1.0\n";
    std::vector<uint8_t> out(header.begin(), header.end());
    out.reserve(header.size() + rgb.size() * 4);
    for (int y = height - 1; y >= 0; --y) {  // bottom row first
        const uint8_t* p = reinterpret_cast<const uint8_t*>(rgb.data() + row * (size_t)y);
        out.insert(out.end(), p, p + row * 4);  // little-endian host
    }
    write_file(path, "write_pfm", out.data(), out.size());
}

std::vector<float> read_pfm(const std::string& path, int* width, int* height) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("read_pfm: cannot open " + path);
    std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    // header: three whitespace-separated tokens after the magic, then exactly one whitespace byte
    size_t i = 0;
    auto token = [&](const char* what) {
        while (i < data.size() && std::isspace((unsigned char)data[i])) ++i;
        const size_t s = i;
        while (i < data.size() && !std::isspace((unsigned char)data[i])) ++i;
        if (s == i) throw std::runtime_error(std::string("read_pfm: truncated header (") + what + ") in " + path);
        return data.substr(s, i - s);
    };
    if (data.size() < 2 || data[0] != 'P' || data[1] != 'F') throw std::runtime_error("read_pfm: " + path + " is not a colour PFM");
    i = 2;
    if (i >= data.size() || !std::isspace((unsigned char)data[i])) throw std::runtime_error("read_pfm: bad magic in " + path);
    int w = 0, h = 0;
    float scale = 0.0f;
    try {
        size_t used = 0;
        const std::string ws = token("width"), hs = token("height"), ss = token("scale");
        w = std::stoi(ws, &used);
        if (used != ws.size()) throw std::invalid_argument(ws);
        h = std::stoi(hs, &used);
        if (used != hs.size()) throw std::invalid_argument(hs);
        scale = std::stof(ss, &used);
        if (used != ss.size()) throw std::invalid_argument(ss);
    } catch (const std::logic_error&) {
        throw std::runtime_error("read_pfm: malformed header in " + path);
    }
    if (w <= 0 || h <= 0 || scale == 0.0f) throw std::runtime_error("read_pfm: bad dimensions or scale in " + path);
    if (i >= data.size()) throw std::runtime_error("read_pfm: truncated file " + path);
    ++i;  // the single whitespace byte after the scale
    const size_t row = 3 * (size_t)w;
    const size_t need = row * (size_t)h * 4;
    if (data.size() - i < need) throw std::runtime_error("read_pfm: truncated pixel data in " + path);
    const bool big = scale > 0.0f;
    std::vector<float> out(row * (size_t)h);
    for (int y = 0; y < h; ++y) {
        const size_t src_row = (size_t)(h - 1 - y);  // file rows are bottom to top
        for (size_t k = 0; k < row; ++k) {
            const uint8_t* p = reinterpret_cast<const uint8_t*>(data.data() + i + 4 * (src_row * row + k));
            const uint32_t u = big ? ((uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3])
                                   : ((uint32_t)p[3] << 24 | (uint32_t)p[2] << 16 | (uint32_t)p[1] << 8 | p[0]);
            float v;
            std::memcpy(&v, &u, 4);
            out[(size_t)y * row + k] = v;
        }
    }
    *width = w;
    *height = h;
    return out;
}

uint64_t fnv1a64(const void* data, size_t bytes) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < bytes; ++i) {
        h ^= p[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

std::string hex64(uint64_t v) {
    char buf[17];
    std::snprintf(buf, sizeof buf, "%016llx", (unsigned long long)v);
    return buf;
}

}  // namespace wf
