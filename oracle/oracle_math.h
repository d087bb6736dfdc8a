// TEST INFRASTRUCTURE ONLY -- CPU oracle of the Psycles path-trace
// integrator.  Nothing in the product links, loads or calls this code; only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as
// the checker.
//
// Scalar float math shared by the oracle.  Every operation is written out so
// that the order of IEEE-754 single-precision operations is explicit; the
// oracle is compiled with -ffp-contract=off so a*b+c is never fused unless
// std::fma is written.  Luisa builtins that the reference calls but whose
// implementation is not in the reference tree (normalize, length, lerp) are
// fixed here as: normalize(v) = v / sqrt(dot(v, v)), length(v) =
// sqrt(dot(v, v)), dot = ((x*x' + y*y') + z*z').
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace oracle {

struct float2 {
    float x{}, y{};
};
struct float3 {
    float x{}, y{}, z{};
};
struct float4 {
    float x{}, y{}, z{}, w{};
};

inline float2 f2(float x, float y) { return {x, y}; }
inline float3 f3(float x, float y, float z) { return {x, y, z}; }
inline float3 f3(float v) { return {v, v, v}; }

inline float3 operator+(float3 a, float3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float3 operator-(float3 a, float3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float3 operator-(float3 a) { return {-a.x, -a.y, -a.z}; }
inline float3 operator*(float3 a, float3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline float3 operator*(float3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float3 operator*(float s, float3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float3 operator/(float3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float3 operator/(float3 a, float3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline float3 &operator+=(float3 &a, float3 b) { a = a + b; return a; }
inline float3 &operator*=(float3 &a, float3 b) { a = a * b; return a; }
inline float3 &operator*=(float3 &a, float s) { a = a * s; return a; }
inline float3 &operator/=(float3 &a, float s) { a = a / s; return a; }
inline float2 operator*(float2 a, float s) { return {a.x * s, a.y * s}; }

inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float3 cross(float3 a, float3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(float3 v) { return std::sqrt(dot(v, v)); }
inline float length_squared(float3 v) { return dot(v, v); }
inline float3 normalize(float3 v) { return v / std::sqrt(dot(v, v)); }
inline float minf(float a, float b) { return a < b ? a : b; }
inline float maxf(float a, float b) { return a > b ? a : b; }
inline float clampf(float v, float lo, float hi) { return minf(maxf(v, lo), hi); }
inline float3 max3(float3 a, float3 b) { return {maxf(a.x, b.x), maxf(a.y, b.y), maxf(a.z, b.z)}; }
inline float3 clamp3(float3 v, float lo, float hi) {
    return {clampf(v.x, lo, hi), clampf(v.y, lo, hi), clampf(v.z, lo, hi)};
}
inline float lerp(float a, float b, float t) { return a + t * (b - a); }
inline bool any_nonzero(float3 v) { return v.x != 0.0f || v.y != 0.0f || v.z != 0.0f; }
inline bool any_nan(float3 v) { return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z); }
inline float max_component(float3 v) { return maxf(v.x, maxf(v.y, v.z)); }
inline float max_abs_component(float3 v) {
    return maxf(std::fabs(v.x), maxf(std::fabs(v.y), std::fabs(v.z)));
}
inline uint32_t float_bits(float v) { uint32_t u; std::memcpy(&u, &v, 4); return u; }
inline float bits_float(uint32_t u) { float v; std::memcpy(&v, &u, 4); return v; }

// Column-major 4x4 matrix, the psycles::Mat4f / luisa::float4x4 layout.
struct mat4 {
    float3 c0, c1, c2, c3;  // xyz of each column (the w row is 0,0,0,1)
};

inline mat4 mat4_from_column_major(const float *e) {
    return {{e[0], e[1], e[2]}, {e[4], e[5], e[6]}, {e[8], e[9], e[10]}, {e[12], e[13], e[14]}};
}

// cycles_transform::point / direction: the explicit FMA tree of
// src/luisa/cycles_transform.cpp:7-24.
inline float3 transform_affine(const mat4 &m, float3 v, bool translate) {
    const float tx = translate ? m.c3.x : 0.0f;
    const float ty = translate ? m.c3.y : 0.0f;
    const float tz = translate ? m.c3.z : 0.0f;
    return {std::fma(v.x, m.c0.x, std::fma(v.y, m.c1.x, std::fma(v.z, m.c2.x, tx))),
            std::fma(v.x, m.c0.y, std::fma(v.y, m.c1.y, std::fma(v.z, m.c2.y, ty))),
            std::fma(v.x, m.c0.z, std::fma(v.y, m.c1.z, std::fma(v.z, m.c2.z, tz)))};
}
inline float3 transform_point(const mat4 &m, float3 v) { return transform_affine(m, v, true); }
inline float3 transform_direction(const mat4 &m, float3 v) { return transform_affine(m, v, false); }

// Inverse of an affine column-major transform, computed in double precision
// with the adjugate and rounded once to float.  The same recipe produces the
// world-to-object matrices of the product, so both traverse with identical
// object-space rays.
inline mat4 affine_inverse(const mat4 &m) {
    const double a00 = m.c0.x, a10 = m.c0.y, a20 = m.c0.z;
    const double a01 = m.c1.x, a11 = m.c1.y, a21 = m.c1.z;
    const double a02 = m.c2.x, a12 = m.c2.y, a22 = m.c2.z;
    const double t0 = m.c3.x, t1 = m.c3.y, t2 = m.c3.z;
    const double c00 = a11 * a22 - a12 * a21;
    const double c01 = a12 * a20 - a10 * a22;
    const double c02 = a10 * a21 - a11 * a20;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double inv = det != 0.0 ? 1.0 / det : 0.0;
    // inverse row r, column c = cofactor(c, r) / det
    const double i00 = c00 * inv;
    const double i01 = (a02 * a21 - a01 * a22) * inv;
    const double i02 = (a01 * a12 - a02 * a11) * inv;
    const double i10 = c01 * inv;
    const double i11 = (a00 * a22 - a02 * a20) * inv;
    const double i12 = (a02 * a10 - a00 * a12) * inv;
    const double i20 = c02 * inv;
    const double i21 = (a01 * a20 - a00 * a21) * inv;
    const double i22 = (a00 * a11 - a01 * a10) * inv;
    const double u0 = -(i00 * t0 + i01 * t1 + i02 * t2);
    const double u1 = -(i10 * t0 + i11 * t1 + i12 * t2);
    const double u2 = -(i20 * t0 + i21 * t1 + i22 * t2);
    mat4 r;
    r.c0 = {float(i00), float(i10), float(i20)};
    r.c1 = {float(i01), float(i11), float(i21)};
    r.c2 = {float(i02), float(i12), float(i22)};
    r.c3 = {float(u0), float(u1), float(u2)};
    return r;
}

// transpose(world_to_object) restricted to 3x3: the normal_to_world matrix
// of src/luisa/path_kernel_surface_primitive.cpp:27-29.
inline mat4 normal_matrix(const mat4 &w) {
    mat4 n;
    n.c0 = {w.c0.x, w.c1.x, w.c2.x};
    n.c1 = {w.c0.y, w.c1.y, w.c2.y};
    n.c2 = {w.c0.z, w.c1.z, w.c2.z};
    n.c3 = {0.0f, 0.0f, 0.0f};
    return n;
}

// safe_normalize of make_light_transport_callables
// (src/luisa/path_tracer_lighting.cpp:9-17).
inline float3 safe_normalize(float3 value, float3 fallback) {
    const bool valid = dot(value, value) > 1.0e-20f;
    const float3 selected = valid ? value : fallback;
    return normalize(dot(selected, selected) > 1.0e-20f ? selected : f3(0.0f, 0.0f, 1.0f));
}

// normalize_or (include/psycles/luisa/spherical_geometry.h:35 and
// src/luisa/path_kernel_emissive_triangle.cpp:10).
inline float3 normalize_or(float3 value, float3 fallback) {
    const float l2 = dot(value, value);
    return l2 > 1.0e-20f ? value / std::sqrt(maxf(l2, 1.0e-20f)) : fallback;
}

// analytic_light_sampling::safe_normalize
// (include/psycles/luisa/analytic_light_sampling.h:120).
inline float3 light_safe_normalize(float3 value, float3 fallback) {
    const float m2 = dot(value, value);
    return m2 > 0.0f ? value / std::sqrt(maxf(m2, 1.0e-30f)) : fallback;
}

// Transcendentals on the sampling path are evaluated in double precision
// and rounded once to float, on the CPU here and on the GPU in the product,
// so both sides produce the same float for the same argument.
inline float sin_(float x) { return static_cast<float>(std::sin(static_cast<double>(x))); }
inline float cos_(float x) { return static_cast<float>(std::cos(static_cast<double>(x))); }
inline float acos_(float x) { return static_cast<float>(std::acos(static_cast<double>(x))); }
inline float asin_(float x) { return static_cast<float>(std::asin(static_cast<double>(x))); }
inline float pow_(float x, float y) {
    return static_cast<float>(std::pow(static_cast<double>(x), static_cast<double>(y)));
}
inline float tan_(float x) { return static_cast<float>(std::tan(static_cast<double>(x))); }
inline float exp_(float x) { return static_cast<float>(std::exp(static_cast<double>(x))); }
inline float log_(float x) { return static_cast<float>(std::log(static_cast<double>(x))); }
inline float atan2_(float y, float x) {
    return static_cast<float>(std::atan2(static_cast<double>(y), static_cast<double>(x)));
}

constexpr float kPi = 3.1415926535897932f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInvTwoPi = 0.15915494309189533577f;
constexpr uint32_t kInvalid = 0xffffffffu;

}  // namespace oracle
