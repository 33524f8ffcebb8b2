// Counter-based random numbers: every draw is a pure function of
// (seed, pixel, sample, depth, dimension), so any execution order -- one thread per path, a
// wavefront stage, a batch of jobs -- consumes identical numbers for the same path.
//
// Reference: WVM/include/wf/rng.hpp:8-42. The hash is the "lowbias32" integer finaliser
// (Chris Wellons, hash-prospector); the key derivation and the counter layout below must stay
// bit-identical to the reference because the images are compared bit for bit.
#pragma once
#include "wf/math.hpp"

namespace wf {

WF_HD uint32_t hash_u32(uint32_t x) {
    x = (x ^ (x >> 16)) * 0x7feb352dU;
    x = (x ^ (x >> 15)) * 0x846ca68bU;
    return x ^ (x >> 16);
}

struct PathKey {
    uint32_t k0, k1;
};

// Two independent hash chains of (seed, pixel, sample). `pixel` is the job-local linear pixel
// index py * width + px.
WF_HD PathKey make_path_key(uint32_t seed, uint32_t pixel, uint32_t sample) {
    const uint32_t sa = hash_u32(seed ^ 0x9e3779b9U);
    const uint32_t sb = hash_u32(seed + 0x85ebca6bU);
    PathKey key;
    key.k0 = hash_u32(hash_u32(sa + pixel * 0xc2b2ae35U) ^ (sample * 0x27d4eb2fU + 0x165667b1U));
    key.k1 = hash_u32(hash_u32(sb ^ (pixel * 0x9e3779b1U)) + (sample * 0x85ebca77U + 0xc2b2ae3dU));
    return key;
}

// Dimension slots within one depth (16 slots per depth).
enum RngDim : uint32_t {
    kDimPixelX = 0,
    kDimPixelY = 1,
    kDimLightPick = 2,
    kDimLightU = 3,
    kDimLightV = 4,
    kDimBsdfU = 5,
    kDimBsdfV = 6,
    kDimRoulette = 7,
    kDimDielectric = 8,
    kDimCount = 16
};

// Uniform float in [0, 1) with 24 bits: the top 24 bits of the hash times 2^-24.
WF_HD float rng(PathKey key, uint32_t depth, uint32_t dim) {
    const uint32_t counter = depth * kDimCount + dim;
    const uint32_t h = hash_u32(key.k0 ^ hash_u32(counter * 0x9e3779b9U + key.k1));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

}  // namespace wf
