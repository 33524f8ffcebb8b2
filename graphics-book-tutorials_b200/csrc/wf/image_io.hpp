// Image files and hashing: the API of the reference's WVM/include/wf/image_io.hpp:9-27.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace wf {

// 8-bit RGB PNG (colour type 2, no interlace, filter None per row) whose zlib stream holds only
// stored deflate blocks (at most 65,535 bytes each); CRC-32 and Adler-32 computed here. Throws
// std::runtime_error on a size mismatch or a write failure, leaving no file behind.
void write_png(const std::string& path, int width, int height, const std::vector<uint8_t>& rgb8);
// Little-endian PFM: "PF\n<w> <h>\n-1.0\n", rows bottom to top.
void write_pfm(const std::string& path, int width, int height, const std::vector<float>& rgb);
// Reads a colour PFM of either endianness (scale sign); rows returned top to bottom. Throws
// std::runtime_error on a missing, truncated or non-PFM file.
std::vector<float> read_pfm(const std::string& path, int* width, int* height);
uint64_t fnv1a64(const void* data, size_t bytes);
std::string hex64(uint64_t v);  // 16 lowercase hex digits

}  // namespace wf
