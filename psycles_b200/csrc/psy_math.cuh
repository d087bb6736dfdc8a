// Device float math of the path-trace kernels.
//
// The kernels are compiled with -fmad=false, IEEE division and square root,
// so every expression below rounds exactly as written; fmaf is spelled out
// where the Psycles kernels prescribe a fused operation (Pluecker products,
// src/luisa/cycles_triangle_intersection_component.cpp:13-29, and the
// Cycles affine transform, src/luisa/cycles_transform.cpp:7-24).
// Conventions for Luisa builtins the reference calls: normalize(v) =
// v / sqrt(dot(v, v)); dot = ((x*x' + y*y') + z*z'); lerp(a, b, t) =
// a + t*(b - a); triangle_interpolate = (1-u-v)a + ub + vc.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace psy {

struct f3 {
    float x, y, z;
};
struct f2 {
    float x, y;
};

__host__ __device__ __forceinline__ f3 mk3(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ f3 mk3(float v) { return {v, v, v}; }
__host__ __device__ __forceinline__ f2 mk2(float x, float y) { return {x, y}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, f3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__host__ __device__ __forceinline__ f2 operator*(f2 a, float s) { return {a.x * s, a.y * s}; }

__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float dot(f2 a, f2 b) { return a.x * b.x + a.y * b.y; }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ float minf_(float a, float b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ float maxf_(float a, float b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ float clampf_(float v, float lo, float hi) { return minf_(maxf_(v, lo), hi); }
__host__ __device__ __forceinline__ f3 max3(f3 a, f3 b) { return {maxf_(a.x, b.x), maxf_(a.y, b.y), maxf_(a.z, b.z)}; }
__host__ __device__ __forceinline__ f3 clamp3(f3 v, float lo, float hi) {
    return {clampf_(v.x, lo, hi), clampf_(v.y, lo, hi), clampf_(v.z, lo, hi)};
}
__device__ __forceinline__ float length(f3 v) { return sqrtf(dot(v, v)); }
__device__ __forceinline__ f3 normalize(f3 v) { return v / sqrtf(dot(v, v)); }
__host__ __device__ __forceinline__ float lerpf_(float a, float b, float t) { return a + t * (b - a); }
__host__ __device__ __forceinline__ bool any_nonzero(f3 v) { return v.x != 0.0f || v.y != 0.0f || v.z != 0.0f; }
__device__ __forceinline__ bool any_nan(f3 v) { return isnan(v.x) || isnan(v.y) || isnan(v.z); }
__host__ __device__ __forceinline__ float max_component(f3 v) { return maxf_(v.x, maxf_(v.y, v.z)); }
__device__ __forceinline__ float max_abs_component(f3 v) { return maxf_(fabsf(v.x), maxf_(fabsf(v.y), fabsf(v.z))); }

// Column-major affine transform (columns c0..c2 and translation c3).
struct Xform {
    f3 c0, c1, c2, c3;
};

// cycles_transform::point / direction (src/luisa/cycles_transform.cpp:7-24).
__device__ __forceinline__ f3 xform_affine(const Xform &m, f3 v, bool translate) {
    const float tx = translate ? m.c3.x : 0.0f;
    const float ty = translate ? m.c3.y : 0.0f;
    const float tz = translate ? m.c3.z : 0.0f;
    return {fmaf(v.x, m.c0.x, fmaf(v.y, m.c1.x, fmaf(v.z, m.c2.x, tx))),
            fmaf(v.x, m.c0.y, fmaf(v.y, m.c1.y, fmaf(v.z, m.c2.y, ty))),
            fmaf(v.x, m.c0.z, fmaf(v.y, m.c1.z, fmaf(v.z, m.c2.z, tz)))};
}
__device__ __forceinline__ f3 xform_point(const Xform &m, f3 v) { return xform_affine(m, v, true); }
__device__ __forceinline__ f3 xform_direction(const Xform &m, f3 v) { return xform_affine(m, v, false); }

// safe_normalize of make_light_transport_callables (src/luisa/path_tracer_lighting.cpp:9-17).
__device__ __forceinline__ f3 safe_normalize(f3 value, f3 fallback) {
    const bool valid = dot(value, value) > 1.0e-20f;
    const f3 selected = valid ? value : fallback;
    return normalize(dot(selected, selected) > 1.0e-20f ? selected : mk3(0.0f, 0.0f, 1.0f));
}

// normalize_or (include/psycles/luisa/spherical_geometry.h:35-41).
__device__ __forceinline__ f3 normalize_or(f3 value, f3 fallback) {
    const float l2 = dot(value, value);
    return l2 > 1.0e-20f ? value / sqrtf(maxf_(l2, 1.0e-20f)) : fallback;
}

// analytic_light_sampling::safe_normalize (analytic_light_sampling.h:120-131).
__device__ __forceinline__ f3 light_safe_normalize(f3 value, f3 fallback) {
    const float m2 = dot(value, value);
    return m2 > 0.0f ? value / sqrtf(maxf_(m2, 1.0e-30f)) : fallback;
}

// Transcendentals on the sampling path are evaluated in double precision
// and rounded once to float, so the kernels and a CPU evaluation of the same
// expression agree bit for bit.  They are out of line: each double-precision
// routine is long, and one copy per call site would overflow the
// instruction cache of the shading kernel.
__device__ __noinline__ float sin_(float x) { return static_cast<float>(sin(static_cast<double>(x))); }
__device__ __noinline__ float cos_(float x) { return static_cast<float>(cos(static_cast<double>(x))); }
__device__ __noinline__ float acos_(float x) { return static_cast<float>(acos(static_cast<double>(x))); }
__device__ __noinline__ float asin_(float x) { return static_cast<float>(asin(static_cast<double>(x))); }
__device__ __noinline__ float atan2_(float y, float x) {
    return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x)));
}
__device__ __noinline__ float pow_(float x, float y) {
    return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}
__device__ __noinline__ float exp_(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
__device__ __noinline__ float log_(float x) { return static_cast<float>(log(static_cast<double>(x))); }

constexpr float kPi = 3.1415926535897932f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInvTwoPi = 0.15915494309189533577f;
constexpr uint32_t kInvalid = 0xffffffffu;

__device__ __forceinline__ f3 ld3(const float *p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ f3 ld3(float4 v) { return {v.x, v.y, v.z}; }

}  // namespace psy
