// Small vector algebra shared by host code and sm_100a kernels.
//
// API surface of the reference header WVM/include/wf/math.hpp (names, struct layouts and the
// exact floating-point operation order). Every function here is evaluated without fused
// multiply-add (host: -ffp-contract=off, device: --fmad=false) so that a host-side
// precomputation (triangle edges, normals, areas) and the device estimator round identically.
// Division of a vector by a scalar is a reciprocal followed by three multiplies, as in the
// reference (WVM/include/wf/math.hpp:29); it is NOT three IEEE divides.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define WF_HD __host__ __device__ __forceinline__
#else
#define WF_HD inline
#endif

namespace wf {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInf = 3.402823466e+38f;  // FLT_MAX: "no upper bound" for a ray

struct Vec3 {
    float x, y, z;
};

WF_HD Vec3 make_vec3(float x, float y, float z) { return Vec3{x, y, z}; }

WF_HD Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
WF_HD Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
WF_HD Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
WF_HD Vec3 operator*(Vec3 a, Vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
WF_HD Vec3 operator*(Vec3 a, float k) { return {a.x * k, a.y * k, a.z * k}; }
WF_HD Vec3 operator*(float k, Vec3 a) { return {a.x * k, a.y * k, a.z * k}; }
// Reciprocal then multiply (reference rounding, see file comment).
WF_HD Vec3 operator/(Vec3 a, float k) {
    const float inv = 1.0f / k;
    return {a.x * inv, a.y * inv, a.z * inv};
}
WF_HD Vec3& operator+=(Vec3& a, Vec3 b) {
    a.x += b.x; a.y += b.y; a.z += b.z;
    return a;
}
WF_HD Vec3& operator*=(Vec3& a, Vec3 b) {
    a.x *= b.x; a.y *= b.y; a.z *= b.z;
    return a;
}
WF_HD Vec3& operator*=(Vec3& a, float k) {
    a.x *= k; a.y *= k; a.z *= k;
    return a;
}

// (x*x' + y*y') + z*z', left to right.
WF_HD float dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
WF_HD Vec3 cross(Vec3 a, Vec3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
WF_HD float length2(Vec3 a) { return dot(a, a); }
WF_HD float length(Vec3 a) { return sqrtf(dot(a, a)); }
WF_HD Vec3 normalize(Vec3 a) {
    const float len = length(a);
    if (len > 0.0f) return a / len;
    return a;
}
// Compare-and-select minimum / maximum: a NaN operand in the first slot is dropped exactly the
// way the reference's ternaries drop it (fminf/fmaxf would differ for NaN inputs).
WF_HD float fminf3(float a, float b) { return a < b ? a : b; }
WF_HD float fmaxf3(float a, float b) { return a > b ? a : b; }
WF_HD float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
WF_HD float max_component(Vec3 a) { return fmaxf3(a.x, fmaxf3(a.y, a.z)); }
WF_HD Vec3 vmin(Vec3 a, Vec3 b) { return {fminf3(a.x, b.x), fminf3(a.y, b.y), fminf3(a.z, b.z)}; }
WF_HD Vec3 vmax(Vec3 a, Vec3 b) { return {fmaxf3(a.x, b.x), fmaxf3(a.y, b.y), fmaxf3(a.z, b.z)}; }
WF_HD Vec3 reflect(Vec3 d, Vec3 n) { return d - n * (2.0f * dot(d, n)); }
// Rec. 709 luma weights.
WF_HD float luminance(Vec3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
// v - v is 0 for every finite v and NaN for NaN and +-inf; needs no fast-math-sensitive builtin.
WF_HD bool is_finite1(float v) { return v - v == 0.0f; }
WF_HD bool is_finite3(Vec3 a) { return is_finite1(a.x) && is_finite1(a.y) && is_finite1(a.z); }

// Orthonormal basis (t, b) around the unit normal n: the branch-on-sign construction of
// Duff et al. 2017 ("Building an Orthonormal Basis, Revisited"), same operand order as
// WVM/include/wf/math.hpp:54-60.
WF_HD void make_basis(Vec3 n, Vec3* t, Vec3* b) {
    const float sgn = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (sgn + n.z);
    const float c = n.x * n.y * a;
    *t = Vec3{1.0f + sgn * n.x * n.x * a, sgn * c, -sgn * n.x};
    *b = Vec3{c, sgn + n.y * n.y * a, -n.y};
}

// 32-byte ray: origin, tmin, direction, tmax (reference layout, WVM/include/wf/math.hpp:62-67).
struct Ray {
    Vec3 o;
    float tmin;
    Vec3 d;
    float tmax;
};

}  // namespace wf
