// Device building blocks of the path-trace kernels: tabulated-Sobol lookup,
// closure programs, light sampling, two-level BVH traversal with the Cycles
// closest-hit predicate, and hit reconstruction.  Each function names the
// Psycles function it implements.
#pragma once

#include <type_traits>

#include "psy_math.cuh"
#include "psy_scene.h"

namespace psy {

// ------------------------------------------------------- record sectors
// A path record's 16-byte fields pair up into its four 32-byte sectors (ray
// origin + direction, the two state words, throughput + radiance, hit + hit
// primitive).  One 256-bit access (ld / st.global.v8.b32, sm_100) moves a
// pair: a lane fills a whole sector per request instead of half of one.
// The field passed is the pair's first; its record offset is 32-byte aligned.
__device__ __forceinline__ uint4 bits4(const float4 &v) {
    return make_uint4(__float_as_uint(v.x), __float_as_uint(v.y), __float_as_uint(v.z), __float_as_uint(v.w));
}
__device__ __forceinline__ float4 floats4(const uint4 &v) {
    return make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w));
}
__device__ __forceinline__ void load_sector(const void *p, uint4 &a, uint4 &b) {
    asm volatile("ld.global.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
                 : "l"(p));
}
__device__ __forceinline__ void store_sector(void *p, const uint4 &a, const uint4 &b) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(a.x), "r"(a.y), "r"(a.z),
                 "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
                 : "memory");
}
template <class A, class B>
__device__ __forceinline__ void load_pair(const PathField<A> &first, size_t i, A &a, B &b) {
    uint4 ua, ub;
    load_sector(&first[i], ua, ub);
    if constexpr (std::is_same<A, float4>::value) a = floats4(ua);
    else a = ua;
    if constexpr (std::is_same<B, float4>::value) b = floats4(ub);
    else b = ub;
}
__device__ __forceinline__ uint4 as_bits(const float4 &v) { return bits4(v); }
__device__ __forceinline__ uint4 as_bits(const uint4 &v) { return v; }
template <class A, class B>
__device__ __forceinline__ void store_pair(const PathField<A> &first, size_t i, const A &a, const B &b) {
    store_sector(&first[i], as_bits(a), as_bits(b));
}

// ------------------------------------------------------------- sampler
// include/psycles/luisa/cycles_sampler.h:36-339.

__device__ __forceinline__ uint32_t reverse_bits(uint32_t v) { return __brev(v); }

__device__ __forceinline__ uint32_t reversed_bit_owen(uint32_t v, uint32_t seed) {
    v ^= v * 0x3d20adeau;
    v += seed;
    v *= (seed >> 16u) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return v;
}

__device__ __forceinline__ uint32_t hash_wang_seeded_uint(uint32_t v, uint32_t seed) {
    v = (v ^ 61u) ^ seed;
    v += v << 3u;
    v ^= v >> 4u;
    v *= 0x27d4eb2du;
    return v;
}

__device__ __forceinline__ uint32_t shuffled_pattern_index(uint32_t dimension, uint32_t seed) {
    uint32_t v = dimension & 0xffu;
    const uint32_t mask = 0xffu;
    v ^= seed;
    v *= 0xe170893du;
    v ^= seed >> 16u;
    v ^= (v & mask) >> 4u;
    v ^= seed >> 8u;
    v *= 0x0929eb3fu;
    v ^= seed >> 23u;
    v ^= (v & mask) >> 1u;
    v *= 1u | (seed >> 27u);
    v *= 0x6935fa69u;
    v ^= (v & mask) >> 11u;
    v *= 0x74dcb303u;
    v ^= (v & mask) >> 2u;
    v *= 0x9e501cc3u;
    v ^= (v & mask) >> 2u;
    v *= 0xc860a3dfu;
    v &= mask;
    v ^= v >> 5u;
    return v;
}

__device__ __forceinline__ uint32_t pixel_hash(uint32_t x, uint32_t y, uint32_t seed) {
    const uint32_t qx = 1103515245u * ((x >> 1u) ^ y);
    const uint32_t qy = 1103515245u * ((y >> 1u) ^ x);
    const uint32_t h = 1103515245u * (qx ^ (qy >> 3u));
    return h ^ seed;
}

__device__ __forceinline__ uint32_t shuffled_sample_index(uint32_t sample, uint32_t dimension, uint32_t seed,
                                                          uint32_t size) {
    const uint32_t pattern = shuffled_pattern_index(dimension, seed);
    const uint32_t mask = size - 1u;
    const uint32_t shuffled =
        reverse_bits(reversed_bit_owen(reverse_bits(sample), hash_wang_seeded_uint(dimension, seed)));
    sample = (sample & ~mask) | (shuffled & mask);
    return ((pattern * size) + sample) % (size * 256u);
}

__device__ __forceinline__ float4 sample_4d(const RenderParams &p, uint32_t sample, uint32_t rng_hash, uint32_t dim) {
    return __ldg(&p.sobol[shuffled_sample_index(sample, dim, rng_hash, p.sobol_size)]);
}

// pixel_filter::sample (include/psycles/luisa/pixel_filter.h:17-29).
__device__ __forceinline__ float pixel_filter_sample(const float *table, float random) {
    const uint32_t last = 1023u;
    const float coordinate = clampf_(random, 0.0f, 1.0f) * static_cast<float>(last);
    const uint32_t index = min(static_cast<uint32_t>(coordinate), last);
    const uint32_t next = min(index + 1u, last);
    const float t = coordinate - static_cast<float>(index);
    return lerpf_(__ldg(&table[index]), __ldg(&table[next]), t);
}

// ---------------------------------------------------------- sample maps
// include/psycles/luisa/cycles_sample_mapping.h:49-339.

__device__ __forceinline__ f2 sample_uniform_disk(f2 r) {
    const float a = 2.0f * r.x - 1.0f;
    const float b = 2.0f * r.y - 1.0f;
    const bool x_major = a * a > b * b;
    const float safe_a = a != 0.0f ? a : 1.0f;
    const float safe_b = b != 0.0f ? b : 1.0f;
    const float radius = x_major ? a : b;
    const float angle = x_major ? 0.25f * kPi * (b / safe_a) : 0.5f * kPi - 0.25f * kPi * (a / safe_b);
    if (a == 0.0f && b == 0.0f) return {0.0f, 0.0f};
    return {cos_(angle) * radius, sin_(angle) * radius};
}

struct Basis {
    f3 tangent, bitangent;
};

__device__ __forceinline__ Basis make_orthonormals(f3 n) {
    const f3 general = mk3(n.z - n.y, n.x - n.z, n.y - n.x);
    const f3 equal = mk3(n.z - n.y, n.x + n.z, -n.y - n.x);
    const bool use_general = (n.x != n.y) || (n.x != n.z);
    const f3 t = normalize(use_general ? general : equal);
    return {t, cross(n, t)};
}

__device__ __forceinline__ f3 sample_cosine_hemisphere(f3 n, f2 r, float *pdf) {
    const f2 d = sample_uniform_disk(r);
    const float c = sqrtf(maxf_(1.0f - dot(d, d), 0.0f));
    const Basis b = make_orthonormals(n);
    if (pdf) *pdf = c * kInvPi;
    return b.tangent * d.x + b.bitangent * d.y + n * c;
}

struct ConeSample {
    f3 direction;
    float cosine, pdf;
};

__device__ __forceinline__ ConeSample sample_uniform_cone(f3 axis, float one_minus_cosine, f2 r) {
    const f2 disk = sample_uniform_disk(r);
    const float r2 = dot(disk, disk);
    const float cosine = 1.0f - r2 * one_minus_cosine;
    const float scale = sqrtf(maxf_(one_minus_cosine * (2.0f - one_minus_cosine * r2), 0.0f));
    const f2 mapped = disk * scale;
    const Basis b = make_orthonormals(axis);
    const f3 finite_dir = b.tangent * mapped.x + b.bitangent * mapped.y + axis * cosine;
    if (one_minus_cosine > 0.0f) return {finite_dir, cosine, kInvTwoPi / one_minus_cosine};
    return {axis, 1.0f, 1.0f};
}

// sample_ggx_visible_normal (cycles_sample_mapping.h:131-183): Heitz 2018,
// "Sampling the GGX Distribution of Visible Normals", in the frame of
// make_orthonormals(normal) with the concentric disk map; the half vector
// is not renormalised in world space.
__device__ __noinline__ f3 sample_ggx_visible_normal(f3 normal, f3 incoming, float alpha, f2 random) {
    const Basis w = make_orthonormals(normal);
    const f3 li = mk3(dot(w.tangent, incoming), dot(w.bitangent, incoming), dot(normal, incoming));
    const f3 si = normalize(mk3(alpha * li.x, alpha * li.y, li.z));
    const float pl2 = si.x * si.x + si.y * si.y;
    const f3 pt = mk3(-si.y, si.x, 0.0f) / sqrtf(maxf_(pl2, 1.0e-20f));
    const f3 bx = pl2 > 1.0e-7f ? pt : mk3(1.0f, 0.0f, 0.0f);
    const f3 by = cross(si, bx);
    f2 disk = sample_uniform_disk(random);
    const float projected_area = 0.5f * (1.0f + si.z);
    disk.y = lerpf_(sqrtf(maxf_(1.0f - disk.x * disk.x, 0.0f)), disk.y, projected_area);
    const float hz = sqrtf(maxf_(1.0f - disk.x * disk.x - disk.y * disk.y, 0.0f));
    const f3 sh = bx * disk.x + by * disk.y + si * hz;
    const f3 lh = normalize(mk3(alpha * sh.x, alpha * sh.y, maxf_(sh.z, 0.0f)));
    return w.tangent * lh.x + w.bitangent * lh.y + normal * lh.z;
}

// erf of Abramowitz & Stegun 7.1.28 (1 - 1 / (1 + a1 x + ... + a6 x^6)^16,
// |error| <= 3e-7) as Cycles evaluates it (cycles_sample_mapping.h:188-208):
// Horner steps as fused multiply-adds, +-1 beyond |x| = 12.3.
__device__ __forceinline__ float fast_erf(float value) {
    const float magnitude = fabsf(value);
    const float crushed = 1.0f - (1.0f - magnitude);
    float p = fmaf(0.0000430638f, crushed, 0.0002765672f);
    p = fmaf(p, crushed, 0.0001520143f);
    p = fmaf(p, crushed, 0.0092705272f);
    p = fmaf(p, crushed, 0.0422820123f);
    p = fmaf(p, crushed, 0.0705230784f);
    p = fmaf(p, crushed, 1.0f);
    const float square = p * p;
    const float fourth = square * square;
    const float eighth = fourth * fourth;
    const float sixteenth = eighth * eighth;
    const float unsigned_result = 1.0f - 1.0f / sixteenth;
    if (magnitude >= 12.3f) return value >= 0.0f ? 1.0f : -1.0f;
    return value >= 0.0f ? unsigned_result : -unsigned_result;
}

// erfinv of Giles, "Approximating the erfinv function" (GPU Computing Gems,
// 2011), single-precision branch pair on w = -log((1 - x)(1 + x)), as
// Cycles evaluates it (cycles_sample_mapping.h:210-237).
__device__ __forceinline__ float fast_inverse_erf(float value) {
    const float magnitude = minf_(fabsf(value), 0.99999994f);
    const float base = -log_((1.0f - magnitude) * (1.0f + magnitude));
    const float cx = base - 2.5f;
    float central = fmaf(2.81022636e-08f, cx, 3.43273939e-07f);
    central = fmaf(central, cx, -3.5233877e-06f);
    central = fmaf(central, cx, -4.39150654e-06f);
    central = fmaf(central, cx, 0.00021858087f);
    central = fmaf(central, cx, -0.00125372503f);
    central = fmaf(central, cx, -0.00417768164f);
    central = fmaf(central, cx, 0.246640727f);
    central = fmaf(central, cx, 1.50140941f);
    const float tx = sqrtf(base) - 3.0f;
    float tail = fmaf(-0.000200214257f, tx, 0.000100950558f);
    tail = fmaf(tail, tx, 0.00134934322f);
    tail = fmaf(tail, tx, -0.00367342844f);
    tail = fmaf(tail, tx, 0.00573950773f);
    tail = fmaf(tail, tx, -0.0076224613f);
    tail = fmaf(tail, tx, 0.00943887047f);
    tail = fmaf(tail, tx, 1.00167406f);
    tail = fmaf(tail, tx, 2.83297682f);
    return (base < 5.0f ? central : tail) * value;
}

// sample_beckmann_visible_normal (cycles_sample_mapping.h:239-310): the
// visible-slope sampler of Heitz and d'Eon (2014) with Cycles' root solve
// -- a quadratic first guess, at most three Newton steps kept inside the
// bracket (bisection otherwise) -- in the frame of make_orthonormals(normal).
__device__ __noinline__ f3 sample_beckmann_visible_normal(f3 normal, f3 incoming, float alpha, f2 random) {
    const Basis w = make_orthonormals(normal);
    const f3 li = mk3(dot(w.tangent, incoming), dot(w.bitangent, incoming), dot(normal, incoming));
    const f3 si = normalize(mk3(alpha * li.x, alpha * li.y, li.z));
    const float normal_radius = sqrtf(-log_(random.x));
    const float normal_phi = 2.0f * kPi * random.y;
    const f2 normal_slope = mk2(normal_radius * cos_(normal_phi), normal_radius * sin_(normal_phi));
    const float cosine = si.z;
    const float sine = sqrtf(maxf_(1.0f - cosine * cosine, 0.0f));
    const float safe_cosine = cosine != 0.0f ? cosine : 1.0f;
    const float safe_sine = sine != 0.0f ? sine : 1.0f;
    const float tangent = sine / safe_cosine;
    const float safe_tangent = tangent != 0.0f ? tangent : 1.0f;
    const float cotangent = 1.0f / safe_tangent;
    const float erf_a = fast_erf(cotangent);
    const float exponential = exp_(-cotangent * cotangent);
    const float cosine_phi = sine != 0.0f ? si.x / safe_sine : 1.0f;
    const float sine_phi = sine != 0.0f ? si.y / safe_sine : 0.0f;
    const float k = tangent * 0.56418958354f;
    const float approximate_y = random.x * (1.0f + erf_a + k * (1.0f - erf_a * erf_a));
    const float exact_y = random.x * (1.0f + erf_a + k * exponential);
    const float safe_k = k > 0.0f ? k : 1.0f;
    const float quadratic_b = (0.5f - sqrtf(maxf_(k * (k - approximate_y + 1.0f) + 0.25f, 0.0f))) / safe_k;
    const float b = k > 0.0f ? quadratic_b : approximate_y - 1.0f;
    float inverse_erf = fast_inverse_erf(b);
    f2 begin = mk2(-1.0f, -exact_y);
    f2 end = mk2(erf_a, 1.0f + erf_a + k * exponential - exact_y);
    f2 current = mk2(b, 1.0f + b + k * exp_(-inverse_erf * inverse_erf) - exact_y);
    for (uint32_t iteration = 0; fabsf(current.y) > 1.0e-6f && iteration < 3u; ++iteration) {
        const bool same_sign = (begin.y < 0.0f) == (current.y < 0.0f);
        if (same_sign) begin = current;
        else end.x = current.x;
        const float newton = current.x - current.y / (1.0f - inverse_erf * tangent);
        const bool inside = newton >= begin.x && newton <= end.x;
        current.x = inside ? newton : 0.5f * (begin.x + end.x);
        inverse_erf = fast_inverse_erf(current.x);
        current.y = 1.0f + current.x + k * exp_(-inverse_erf * inverse_erf) - exact_y;
    }
    const f2 general_slope = mk2(inverse_erf, fast_inverse_erf(2.0f * random.y - 1.0f));
    const f2 slope = si.z >= 0.99999f ? normal_slope : general_slope;
    const f2 rotated = mk2(cosine_phi * slope.x - sine_phi * slope.y, sine_phi * slope.x + cosine_phi * slope.y) * alpha;
    const f3 lh = normalize(mk3(-rotated.x, -rotated.y, 1.0f));
    return w.tangent * lh.x + w.bitangent * lh.y + normal * lh.z;
}

// ------------------------------------------------------ closure programs
// GraphSurfaceImplementation::for_each_closure (src/luisa/graph_surface_closures.cpp:5-356)
// with allocation (src/luisa/graph_surface_state.cpp:19-48).

constexpr uint32_t kMaxClosures = 16u;
constexpr uint32_t kMaxClosureStack = 32u;

// One allocated closure.  Diffuse closures keep their authored colour and
// roughness for the Oren-Nayar evaluation (roughness below 1e-5: Lambert).
// The in-scope closures have no Normal input, so every diffuse closure
// shares the normalised shading normal (SurfaceClosures::normal) and a
// transparent closure never reads one.  A glossy closure's `color` holds
// its normal after setup's specular-reflection correction (its colour is
// in its weight), `roughness` its roughness (microfacet alpha = roughness^2),
// and its op carries kGlossyBeckmann for the Beckmann distribution.  A glass
// closure's `color` is its Fresnel tint (its normal is recomputed where it
// is used); a refraction closure's `color` holds its normal like a glossy
// one (its colour is in its weight).
struct PhysicalClosure {
    f3 weight;
    float sample_weight;
    uint32_t op;
    f3 color;
    float roughness;
};

// The closure of the glossy-capable shading variant: glass and refraction
// closures add their IORs.  The variant without glossy closures keeps the
// 36-byte closure, so its shading point stores no IOR it never reads.
struct DielectricClosure : PhysicalClosure {
    float ior;  // relative IOR (inverted on a back face)
    float f0;   // glass: F0 of the authored IOR
};
template <bool kGlossy> struct ClosureSlot {
    using type = PhysicalClosure;
};
template <> struct ClosureSlot<true> {
    using type = DielectricClosure;
};

constexpr uint32_t kGlossyBeckmann = 0x100u;
// A glossy op with kGlossyMultiscatter is MULTI_GGX: GGX with Cycles' tabulated
// multiple-scattering energy preservation; its closure keeps the evaluation
// scale 1 / E in `f0`.
constexpr uint32_t kGlossyMultiscatter = 0x200u;
__device__ __forceinline__ bool is_glossy(uint32_t op) { return (op & 0xffu) == PSY_CLOSURE_GLOSSY; }
__device__ __forceinline__ bool is_glass(uint32_t op) { return (op & 0xffu) == PSY_CLOSURE_GLASS; }
__device__ __forceinline__ bool is_refraction(uint32_t op) { return (op & 0xffu) == PSY_CLOSURE_REFRACTION; }
__device__ __forceinline__ bool is_dielectric(uint32_t op) { return is_glass(op) || is_refraction(op); }

// The surface point's inputs to closure setup, evaluation and sampling.
// `view` is the normalised incoming direction every closure routine of
// the reference takes (safe_normalize(point.incoming, ...): the fallback
// never applies to a ray direction), normalised once per shading point.
struct ClosurePoint {
    f3 shading_normal;    // SurfacePoint::shading_normal
    f3 geometric_normal;  // SurfacePoint::geometric_normal (facing the incoming ray)
    f3 incoming;          // SurfacePoint::incoming (-ray direction)
    f3 view;              // normalize(incoming)
    bool bump_correction; // SurfacePoint::use_bump_map_correction
    bool back_facing;     // SurfacePoint::back_facing
};

// Shading routines are instantiated with and without glossy closures
// (kGlossy): a scene without them runs code with no glossy branch, which
// keeps the shading kernel's register budget where it was before them.
constexpr uint32_t kLeavesOf(bool glossy) { return glossy ? 15u : 7u; }

template <bool kGlossy>
struct SurfaceClosures {
    f3 normal;          // the diffuse closures' normal
    bool normal_exact;  // it equals the shading normal bit for bit (bump term one)
    typename ClosureSlot<kGlossy>::type c[kMaxClosures];
    uint32_t count;
    f3 emission;
};

__device__ __forceinline__ float closure_sample_weight(f3 w) { return fabsf((w.x + w.y + w.z) / 3.0f); }

__device__ __forceinline__ f3 bsdf_allocated_weight(f3 v) {
    v = max3(v, mk3(0.0f));
    const float average = (v.x + v.y + v.z) / 3.0f;
    return average >= 1.0e-5f ? v : mk3(0.0f);
}

__device__ __forceinline__ f3 ld_vector(const SceneView &s, const MaterialGpu &m, uint32_t slot) {
    return ld3(s.vectors + 3u * (m.vector_offset + slot));
}
__device__ __forceinline__ float ld_scalar(const SceneView &s, const MaterialGpu &m, uint32_t slot) {
    return s.scalars[m.scalar_offset + slot];
}

// Film::rgb_to_y of Blender 4.5's default scene-linear space, the
// coefficients of color_to_scalar (src/luisa/graph_surface_value_math.cpp:91-103).
constexpr float kRgbToYR = 0.21267404f, kRgbToYG = 0.7151516f, kRgbToYB = 0.07217542f;

__device__ __forceinline__ f3 lerp3(f3 a, f3 b, f3 t) {
    return {lerpf_(a.x, b.x, t.x), lerpf_(a.y, b.y, t.y), lerpf_(a.z, b.z, t.z)};
}

// cast<int>(x) != 0 of scalar_to_boolean: truncation toward zero, with the
// saturating conversion of the hardware (NaN converts to 0).
__device__ __forceinline__ bool truncates_nonzero(float x) { return __float2int_rz(x) != 0; }

// The value stream of a SurfaceProgram (GraphSurfaceImplementation::
// trace_value_stage, src/luisa/graph_surface_values.cpp:70-100): instructions
// 0..id in order, each reading earlier results; scalars are held in x.
// Operations: src/luisa/graph_surface_value_math.cpp:54-880,
// graph_surface_value_context.cpp:80-108, graph_surface_value_procedural.cpp:
// 568-600.  Scene compile checks the operations, operand order, types and
// parameter slots.  Out of line: only linked closure inputs reach it.
__device__ __noinline__ f3 eval_value(const SceneView &s, const MaterialGpu &m, uint32_t id) {
    f3 v[kMaxValues];
    const uint32_t n = min(id + 1u, min(m.value_count, kMaxValues));
    for (uint32_t i = 0; i < n; ++i) {
        const psy_value_instruction in = s.values[m.value_offset + i];
        const f3 a = in.a < i ? v[in.a] : mk3(0.0f);
        const f3 b = in.b < i ? v[in.b] : mk3(0.0f);
        const f3 c = in.c < i ? v[in.c] : mk3(0.0f);
        f3 r = mk3(0.0f);
        switch (in.op) {
        case PSY_VALUE_PARAMETER:
            r = in.type == PSY_VALUE_TYPE_SCALAR ? mk3(ld_scalar(s, m, in.parameter), 0.0f, 0.0f)
                                                 : ld_vector(s, m, in.parameter);
            break;
        case PSY_VALUE_PASSTHROUGH: r = a; break;
        case PSY_VALUE_SCALAR_TO_COLOR: r = mk3(a.x); break;
        case PSY_VALUE_SCALAR_TO_BOOLEAN: r.x = truncates_nonzero(a.x) ? 1.0f : 0.0f; break;
        case PSY_VALUE_COLOR_TO_SCALAR: r.x = a.x * kRgbToYR + a.y * kRgbToYG + a.z * kRgbToYB; break;
        case PSY_VALUE_VECTOR_TO_SCALAR: r.x = (a.x + a.y + a.z) / 3.0f; break;
        case PSY_VALUE_ADD: r.x = a.x + b.x; break;
        case PSY_VALUE_SUBTRACT: r.x = a.x - b.x; break;
        case PSY_VALUE_MULTIPLY: r.x = a.x * b.x; break;
        case PSY_VALUE_DIVIDE: r.x = fabsf(b.x) > 1.0e-20f ? a.x / b.x : 0.0f; break;
        case PSY_VALUE_MINIMUM: r.x = fminf(a.x, b.x); break;
        case PSY_VALUE_MAXIMUM: r.x = fmaxf(a.x, b.x); break;
        case PSY_VALUE_POWER: r.x = pow_(fmaxf(a.x, 0.0f), b.x); break;
        case PSY_VALUE_ABSOLUTE: r.x = fabsf(a.x); break;
        case PSY_VALUE_CLAMP01: r.x = fminf(fmaxf(a.x, 0.0f), 1.0f); break;
        case PSY_VALUE_CLAMP_RANGE: {
            float lo = b.x, hi = c.x;
            if (in.static_u0 == 1u && lo > hi) {
                lo = c.x;
                hi = b.x;
            }
            r.x = fminf(fmaxf(a.x, lo), hi);
            break;
        }
        case PSY_VALUE_MIX_FLOAT: {
            const float t = in.static_u0 != 0u ? fminf(fmaxf(c.x, 0.0f), 1.0f) : c.x;
            r.x = lerpf_(a.x, b.x, t);
            break;
        }
        case PSY_VALUE_MIX_VECTOR: {
            f3 t = in.static_u0 != 0u ? c : mk3(c.x);
            if (in.static_u1 != 0u) t = clamp3(t, 0.0f, 1.0f);
            r = lerp3(a, b, t);
            break;
        }
        case PSY_VALUE_MIX: {
            const float t = (in.static_u1 & 1u) != 0u ? fminf(fmaxf(c.x, 0.0f), 1.0f) : c.x;
            const f3 tt = mk3(t);
            switch (in.static_u0) {
            case PSY_BLEND_DARKEN: r = lerp3(a, mk3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)), tt); break;
            case PSY_BLEND_MULTIPLY: r = lerp3(a, a * b, tt); break;
            case PSY_BLEND_LIGHTEN: r = lerp3(a, mk3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)), tt); break;
            case PSY_BLEND_SCREEN: {
                const float k = 1.0f - t;
                r = mk3(1.0f - (k + t * (1.0f - b.x)) * (1.0f - a.x), 1.0f - (k + t * (1.0f - b.y)) * (1.0f - a.y),
                        1.0f - (k + t * (1.0f - b.z)) * (1.0f - a.z));
                break;
            }
            case PSY_BLEND_ADD: r = lerp3(a, a + b, tt); break;
            case PSY_BLEND_DIFFERENCE:
                r = lerp3(a, mk3(fabsf(a.x - b.x), fabsf(a.y - b.y), fabsf(a.z - b.z)), tt);
                break;
            case PSY_BLEND_SUBTRACT: r = lerp3(a, a - b, tt); break;
            default: r = lerp3(a, b, tt); break;  // PSY_BLEND_MIX
            }
            break;
        }
        case PSY_VALUE_MULTIPLY_COLOR: r = lerp3(a, a * b, mk3(fminf(fmaxf(c.x, 0.0f), 1.0f))); break;
        case PSY_VALUE_INVERT: r = lerp3(a, mk3(1.0f) - a, mk3(b.x)); break;
        case PSY_VALUE_SEPARATE_R: r.x = a.x; break;
        case PSY_VALUE_SEPARATE_G: r.x = a.y; break;
        case PSY_VALUE_SEPARATE_B: r.x = a.z; break;
        case PSY_VALUE_COMBINE_COLOR: r = mk3(a.x, b.x, c.x); break;
        default: break;
        }
        v[i] = r;
    }
    return n > id ? v[id] : mk3(0.0f);
}

// A closure input: the closure node's own parameter slot, or a value of the
// stream (PSY_INPUT_VALUE).
__device__ __forceinline__ f3 input_vector(const SceneView &s, const MaterialGpu &m, uint32_t ref) {
    if ((ref & PSY_INPUT_VALUE) == 0u) return ld_vector(s, m, ref);
    return eval_value(s, m, ref & ~PSY_INPUT_VALUE);
}
__device__ __forceinline__ float input_scalar(const SceneView &s, const MaterialGpu &m, uint32_t ref) {
    if (ref == PSY_INPUT_NONE) return 0.0f;
    if ((ref & PSY_INPUT_VALUE) == 0u) return ld_scalar(s, m, ref);
    return eval_value(s, m, ref & ~PSY_INPUT_VALUE).x;
}

// Leaf kinds a closure walk reports (kLeaves of walk_closures).
constexpr uint32_t kLeafDiffuse = 1u, kLeafTransparent = 2u, kLeafEmission = 4u, kLeafGlossy = 8u, kLeafAll = 15u;

// Visits closure leaves depth-first, `a` before `b`, with the add / mix
// weight rule; `visit(op, weight, color, roughness, ior)` receives the
// diffuse / microfacet / transparent / emission leaves selected by kLeaves
// with their authored colour (x strength for emission), the roughness input
// of diffuse and microfacet leaves, and the IOR of glass and refraction (a
// Beckmann leaf's op carries kGlossyBeckmann).  Glass is allocated with the
// mix weight and takes its colour as a tint; refraction's weight is colour x
// mix weight (graph_surface_closures.cpp:290-320).
// Unselected leaves read no inputs (a shadow ray's extinction needs only
// the transparent ones).
template <uint32_t kLeaves = kLeafAll, typename Visit>
__device__ __forceinline__ void walk_closures(const SceneView &s, const MaterialGpu &m, Visit visit) {
    uint32_t stack_id[kMaxClosureStack];
    float stack_w[kMaxClosureStack];
    int sp = 0;
    stack_id[sp] = m.root;
    stack_w[sp] = 1.0f;
    ++sp;
    while (sp > 0) {
        --sp;
        const uint32_t id = stack_id[sp];
        const float w = stack_w[sp];
        if (id >= m.code_count) continue;
        const psy_closure_instruction c = s.code[m.code_offset + id];
        if (c.op == PSY_CLOSURE_ADD) {
            if (sp + 2 > int(kMaxClosureStack)) continue;
            stack_id[sp] = c.b; stack_w[sp] = w; ++sp;
            stack_id[sp] = c.a; stack_w[sp] = w; ++sp;
        } else if (c.op == PSY_CLOSURE_MIX) {
            if (sp + 2 > int(kMaxClosureStack)) continue;
            const float f = clampf_(input_scalar(s, m, c.scalar), 0.0f, 1.0f);
            stack_id[sp] = c.b; stack_w[sp] = w * f; ++sp;
            stack_id[sp] = c.a; stack_w[sp] = w * (1.0f - f); ++sp;
        } else if (c.op == PSY_CLOSURE_DIFFUSE) {
            if constexpr ((kLeaves & kLeafDiffuse) != 0u) {
                const f3 color = input_vector(s, m, c.color);
                visit(c.op, color * w, color, input_scalar(s, m, c.roughness), 1.0f);
            }
        } else if (c.op == PSY_CLOSURE_TRANSPARENT) {
            if constexpr ((kLeaves & kLeafTransparent) != 0u) {
                const f3 color = input_vector(s, m, c.color);
                visit(c.op, color * w, color, 0.0f, 1.0f);
            }
        } else if (c.op == PSY_CLOSURE_GLOSSY) {
            if constexpr ((kLeaves & kLeafGlossy) != 0u) {
                const f3 color = input_vector(s, m, c.color);
                const uint32_t op = c.a == PSY_GLOSSY_BECKMANN    ? (uint32_t(PSY_CLOSURE_GLOSSY) | kGlossyBeckmann)
                                    : c.a == PSY_GLOSSY_MULTI_GGX ? (uint32_t(PSY_CLOSURE_GLOSSY) | kGlossyMultiscatter)
                                                                  : uint32_t(PSY_CLOSURE_GLOSSY);
                visit(op, color * w, color, input_scalar(s, m, c.roughness), 1.0f);
            }
        } else if (c.op == PSY_CLOSURE_GLASS || c.op == PSY_CLOSURE_REFRACTION) {
            if constexpr ((kLeaves & kLeafGlossy) != 0u) {
                const f3 color = max3(input_vector(s, m, c.color), mk3(0.0f));
                const uint32_t op = uint32_t(c.op) | (c.a == PSY_GLOSSY_BECKMANN ? kGlossyBeckmann : 0u);
                visit(op, c.op == PSY_CLOSURE_GLASS ? mk3(w) : color * w, color, input_scalar(s, m, c.roughness),
                      maxf_(input_scalar(s, m, c.scalar), 1.0e-5f));
            }
        } else if (c.op == PSY_CLOSURE_EMISSION && (kLeaves & kLeafEmission) != 0u) {
            const f3 color = input_vector(s, m, c.color) * input_scalar(s, m, c.scalar);
            visit(c.op, color * w, color, 0.0f, 1.0f);
        }
    }
}

// ensure_valid_specular_reflection (src/luisa/graph_surface_scattering.cpp:119-155):
// a shading normal whose mirror direction of `incoming` would dip below the
// geometric surface is tilted toward the geometric normal until the
// reflection clears it by min(0.9 cos_i, 0.01).
__device__ __noinline__ f3 ensure_valid_specular_reflection(f3 ng, f3 incoming, f3 n) {
    const f3 reflected = n * (2.0f * dot(n, incoming)) - incoming;
    const float ig = maxf_(dot(incoming, ng), 0.0f);
    const float threshold = minf_(0.9f * ig, 0.01f);
    const bool valid = dot(ng, reflected) >= threshold;
    const f3 tangent = safe_normalize(n - ng * dot(n, ng), n);
    const float it = dot(incoming, tangent);
    const float a = it * it + ig * ig;
    const float b = 2.0f * (a + ig * threshold);
    const float c = (threshold + ig) * (threshold + ig);
    const float disc = maxf_(b * b - 4.0f * a * c, 0.0f);
    const float signed_root = it < 0.0f ? b + sqrtf(disc) : b - sqrtf(disc);
    const float nz2 = clampf_(0.25f * signed_root / maxf_(a, 1.0e-20f), 0.0f, 1.0f);
    const f3 corrected = safe_normalize(tangent * sqrtf(maxf_(1.0f - nz2, 0.0f)) + ng * sqrtf(nz2), ng);
    return (!valid && a > 1.0e-20f) ? corrected : n;
}

// maybe_ensure_valid_specular_reflection (graph_surface_scattering.cpp:157-168).
__device__ __forceinline__ f3 specular_normal(bool correction, f3 ng, f3 incoming, f3 n) {
    const bool equal = ng.x == n.x && ng.y == n.y && ng.z == n.z;
    return correction && !equal ? ensure_valid_specular_reflection(ng, incoming, n) : n;
}

// fresnel_dielectric_cos / f0_from_ior (graph_surface_scattering.cpp:42-58).
__device__ __forceinline__ float fresnel_dielectric_cos(float cosine, float eta) {
    const float c = fabsf(cosine);
    const float g2 = eta * eta - 1.0f + c * c;
    const float g = sqrtf(maxf_(g2, 0.0f));
    const float a = (g - c) / maxf_(g + c, 1.0e-20f);
    const float den = c * (g - c) + 1.0f;
    const float b = (c * (g + c) - 1.0f) / (fabsf(den) > 1.0e-20f ? den : 1.0e-20f);
    const float regular = 0.5f * a * a * (1.0f + b * b);
    return g2 > 0.0f ? regular : 1.0f;
}
// Cycles' table lookups (cycles_table_1d / cycles_table_2d,
// src/luisa/graph_surface_state.cpp:84-130): x and y clamped to [0, 1],
// linear between the two nearest entries; a 2-D table is y_size rows of
// x_size entries.
__device__ __forceinline__ float cycles_table_1d(const float *table, float x, uint32_t size) {
    const float coordinate = clampf_(x, 0.0f, 1.0f) * float(size - 1u);
    const uint32_t index = min(uint32_t(coordinate), size - 1u);
    const uint32_t next = min(index + 1u, size - 1u);
    const float t = coordinate - float(index);
    return lerpf_(__ldg(table + index), __ldg(table + next), t);
}
__device__ __forceinline__ float cycles_table_2d(const float *table, float x, float y, uint32_t x_size,
                                                 uint32_t y_size) {
    const float coordinate = clampf_(y, 0.0f, 1.0f) * float(y_size - 1u);
    const uint32_t index = min(uint32_t(coordinate), y_size - 1u);
    const uint32_t next = min(index + 1u, y_size - 1u);
    const float t = coordinate - float(index);
    const float d0 = cycles_table_1d(table + x_size * index, x, x_size);
    const float d1 = cycles_table_1d(table + x_size * next, x, x_size);
    return lerpf_(d0, d1, t);
}

struct GgxEnergy {
    f3 darkening;
    float energy_scale;
};

// ggx_energy (src/luisa/graph_surface_scattering.cpp:170-198): GGX's
// directional albedo E(roughness, cos) and its average, the single-scattering
// Fresnel albedo `fss` turned into the multiple-scattering one, the weight's
// darkening (1 + Fms (1 - E) / E) E and the evaluation scale 1 / E.
__device__ __noinline__ GgxEnergy ggx_energy(const SceneView &s, float roughness, float incoming_cosine, f3 fss) {
    const float energy = maxf_(cycles_table_2d(s.ggx_e, roughness, incoming_cosine, 32u, 32u), 1.0e-20f);
    const float average = cycles_table_1d(s.ggx_eavg, roughness, 32u);
    const float missing = (1.0f - energy) / energy;
    const float scale = 1.0f / energy;
    const f3 fms = mk3(fss.x * average / maxf_(1.0f - fss.x * (1.0f - average), 1.0e-20f),
                       fss.y * average / maxf_(1.0f - fss.y * (1.0f - average), 1.0e-20f),
                       fss.z * average / maxf_(1.0f - fss.z * (1.0f - average), 1.0e-20f));
    GgxEnergy r;
    r.darkening = mk3((1.0f + fms.x * missing) / scale, (1.0f + fms.y * missing) / scale,
                      (1.0f + fms.z * missing) / scale);
    r.energy_scale = scale;
    return r;
}

__device__ __forceinline__ float f0_from_ior(float ior) {
    const float r = (ior - 1.0f) / maxf_(ior + 1.0f, 1.0e-20f);
    return r * r;
}

// Closure allocation (graph_surface_state.cpp:26-48,
// graph_surface_physical_closures.cpp:158-520): diffuse goes through
// bsdf_alloc (negative weight clamped, average cutoff 1e-5); glossy is
// allocated the same way (reflective caustics on), its normal corrected for
// a valid specular reflection and its weight kept (GGX / Beckmann without
// energy preservation: darkening and evaluation scale one); transparent
// keeps its signed weight, uses the cutoff on |average|, and every
// allocated transparent contribution merges into the first one
// (bsdf_transparent_setup, :483-518: summed weights and sample weights).
template <bool kGlossy>
__device__ __forceinline__ void collect_surface(const SceneView &s, const MaterialGpu &m, const ClosurePoint &pt,
                                    SurfaceClosures<kGlossy> &out) {
    out.count = 0u;
    out.emission = mk3(0.0f);
    out.normal = safe_normalize(pt.shading_normal, pt.shading_normal);
    out.normal_exact = out.normal.x == pt.shading_normal.x && out.normal.y == pt.shading_normal.y &&
                       out.normal.z == pt.shading_normal.z;
    int transparent_slot = -1;
    walk_closures<kLeavesOf(kGlossy)>(s, m, [&](uint32_t op, f3 w, f3 color, float roughness, float ior) {
        if (op == PSY_CLOSURE_EMISSION) {
            out.emission = out.emission + w;
            return;
        }
        typename ClosureSlot<kGlossy>::type p;
        p.op = op;
        p.color = color;
        p.roughness = roughness;
        if constexpr (kGlossy) {
            p.ior = 1.0f;
            p.f0 = 0.0f;
        }
        if (op == PSY_CLOSURE_DIFFUSE) {
            p.weight = bsdf_allocated_weight(w);
            p.sample_weight = closure_sample_weight(p.weight);
            if (!any_nonzero(p.weight)) return;
        } else if (kGlossy && is_glossy(op)) {
            const f3 allocated = max3(w, mk3(0.0f));
            const float allocation = closure_sample_weight(allocated);
            if (!(allocation >= 1.0e-5f)) return;
            p.weight = allocated;
            p.sample_weight = allocation * closure_sample_weight(mk3(1.0f));
            p.color = specular_normal(pt.bump_correction, pt.geometric_normal, pt.view, out.normal);
            if constexpr (kGlossy) {
                if ((op & kGlossyMultiscatter) != 0u) {
                    // ggx_energy (graph_surface_scattering.cpp:170-198) with the Fresnel
                    // single-scattering albedo max(colour, 0); the weight takes the
                    // darkening, evaluations the scale 1 / E
                    const GgxEnergy e = ggx_energy(s, clampf_(roughness, 0.0f, 1.0f),
                                                   clampf_(dot(p.color, pt.view), 0.0f, 1.0f), max3(color, mk3(0.0f)));
                    p.weight = allocated * e.darkening;
                    p.sample_weight = allocation * closure_sample_weight(e.darkening);
                    p.f0 = e.energy_scale;
                }
            }
        } else if (kGlossy && is_dielectric(op)) {
            // MicrofacetGlassComponent::setup (microfacet_glass_component.cpp:180-232): the
            // corrected normal, roughness sqrt(clamp(r^2)), the IOR inverted on a back
            // face, weight max(weight, 0) (no energy preservation).  A glass closure's
            // selection weight would also carry Cycles' tabulated Fresnel albedo; it is
            // the only BSDF closure of its material (compile refuses other mixes), where
            // that factor only rescales weighted_pdf / total, and is taken as one.
            const f3 allocated = max3(w, mk3(0.0f));
            const float allocation = closure_sample_weight(allocated);
            if (!(allocation >= 1.0e-5f)) return;
            p.weight = allocated;
            p.sample_weight = allocation * 1.0f * closure_sample_weight(mk3(1.0f));
            p.roughness = sqrtf(clampf_(roughness * roughness, 0.0f, 1.0f));
            if constexpr (kGlossy) {
                p.ior = pt.back_facing ? 1.0f / ior : ior;
                p.f0 = clampf_(f0_from_ior(ior), 0.0f, 1.0f);
            }
            if (is_refraction(op)) p.color = specular_normal(pt.bump_correction, pt.geometric_normal, pt.view, out.normal);
        } else {
            const float sw = closure_sample_weight(w);
            if (!(sw >= 1.0e-5f)) return;
            if (transparent_slot >= 0) {
                out.c[transparent_slot].weight = out.c[transparent_slot].weight + w;
                out.c[transparent_slot].sample_weight += sw;
                return;
            }
            p.weight = w;
            p.sample_weight = sw;
        }
        if (out.count >= kMaxClosures) return;
        if (op == PSY_CLOSURE_TRANSPARENT) transparent_slot = int(out.count);
        out.c[out.count++] = p;
    });
}

__device__ __forceinline__ f3 material_emission(const SceneView &s, const MaterialGpu &m) {
    f3 r = mk3(0.0f);
    walk_closures<kLeafEmission>(s, m, [&](uint32_t op, f3 w, f3, float, float) {
        if (op == PSY_CLOSURE_EMISSION) r = r + w;
    });
    return r;
}

// transparent_extinction (src/luisa/graph_surface_implementation.cpp:354-372).
__device__ __forceinline__ f3 transparent_extinction(const SceneView &s, const MaterialGpu &m) {
    f3 r = mk3(0.0f);
    walk_closures<kLeafTransparent>(s, m, [&](uint32_t op, f3 w, f3, float, float) {
        if (op == PSY_CLOSURE_TRANSPARENT && closure_sample_weight(w) >= 1.0e-5f) r = r + w;
    });
    return r;
}

constexpr uint32_t kEventReflection = 1u, kEventTransmission = 2u, kEventDiffuse = 4u, kEventGlossy = 8u,
                   kEventSingular = 16u, kEventTransparent = 32u;
constexpr uint32_t kLabelTransmit = 1u, kLabelReflect = 2u, kLabelDiffuse = 4u, kLabelGlossy = 8u,
                   kLabelSingular = 16u, kLabelTransparent = 32u;
constexpr uint32_t kRuntimeBackfacing = 1u, kRuntimeBsdf = 8u, kRuntimeBsdfHasEval = 16u,
                   kRuntimeTransparent = 1024u, kRuntimeBsdfHasTransmission = 2048u;

__device__ __forceinline__ uint32_t label_from_events(uint32_t e) {
    uint32_t l = 0u;
    if (e & kEventTransmission) l |= kLabelTransmit;
    if (e & kEventReflection) l |= kLabelReflect;
    if (e & kEventDiffuse) l |= kLabelDiffuse;
    if (e & kEventGlossy) l |= kLabelGlossy;
    if (e & kEventSingular) l |= kLabelSingular;
    if (e & kEventTransparent) l |= kLabelTransparent;
    return l;
}

constexpr float kMicrofacetSingularAlphaProduct = 2.0e-10f;

// microfacet_alpha / microfacet_is_singular (graph_surface_scattering.cpp:549-568)
// without the glossy filter (its roughness is zero: Filter Glossy off).
__device__ __forceinline__ float microfacet_alpha(float roughness) {
    const float a = clampf_(roughness, 0.0f, 1.0f);
    return a * a;
}
__device__ __forceinline__ bool microfacet_singular(float roughness) {
    const float a = microfacet_alpha(roughness);
    return a * a <= kMicrofacetSingularAlphaProduct;
}

// cycles_runtime_flags (src/luisa/graph_surface_scattering.cpp:292-365).
template <bool kGlossy>
__device__ __forceinline__ uint32_t runtime_flags(const SurfaceClosures<kGlossy> &s, bool back_facing) {
    uint32_t f = back_facing ? kRuntimeBackfacing : 0u;
    for (uint32_t i = 0; i < s.count; ++i) {
        const auto &c = s.c[i];
        if (c.op == PSY_CLOSURE_DIFFUSE) f |= kRuntimeBsdf | kRuntimeBsdfHasEval;
        else if (is_glossy(c.op)) f |= kRuntimeBsdf | (microfacet_singular(c.roughness) ? 0u : kRuntimeBsdfHasEval);
        else if (is_dielectric(c.op))
            f |= kRuntimeBsdf | (microfacet_singular(c.roughness) ? 0u : kRuntimeBsdfHasEval) | kRuntimeBsdfHasTransmission;
        else f |= kRuntimeBsdf | kRuntimeTransparent;
    }
    return f;
}

// bump_shadowing_term (src/luisa/graph_surface_scattering.cpp:219-281) of a
// diffuse or glossy closure whose normal is `cn`: one when it is the
// smooth shading normal; otherwise a direction on the wrong side of the
// smooth surface is rejected during evaluation (and, for diffuse closures,
// also when sampling), and a diffuse closure under bump correction gets the
// smoothed shadowing factor.  The in-scope diffuse closures have the
// shading normal, so only glossy closures reach the general case.
__device__ __noinline__ float bump_shadowing_general(f3 smooth, f3 cn, f3 dir, bool is_evaluation, bool diffuse,
                                                     bool bump_correction) {
    const float csd = dot(smooth, dir);
    const float csc = dot(smooth, cn);
    const float ccd = dot(cn, dir);
    const bool reject = csd * csc * ccd < 0.0f && (is_evaluation || diffuse);
    const float cos_i = fabsf(csd);
    const float cos_d = fabsf(csc);
    const float tan_d2 = maxf_(1.0f / maxf_(cos_d * cos_d, 1.0e-20f) - 1.0f, 0.0f);
    const float bump_alpha2 = clampf_(0.125f * tan_d2, 0.0f, 1.0f);
    const float tan_i2 = maxf_(1.0f / maxf_(cos_i * cos_i, 1.0e-20f) - 1.0f, 0.0f);
    const float lambda = 0.5f * (sqrtf(1.0f + bump_alpha2 * tan_i2) - 1.0f);
    const float smoothed = 1.0f / (1.0f + lambda);
    const bool domain = diffuse && bump_correction && cos_d < 1.0f && cos_i < 1.0f;
    const bool grazing = domain && cos_i < 1.0e-6f;
    float result = domain && !grazing ? smoothed : 1.0f;
    if (reject || grazing) result = 0.0f;
    return result;
}
__device__ __forceinline__ float bump_shadowing(f3 smooth, f3 cn, f3 dir, bool is_evaluation, bool diffuse,
                                                bool bump_correction) {
    if (cn.x == smooth.x && cn.y == smooth.y && cn.z == smooth.z) return 1.0f;
    return bump_shadowing_general(smooth, cn, dir, is_evaluation, diffuse, bump_correction);
}

// microfacet_distribution / microfacet_lambda (graph_surface_scattering.cpp:508-547).
__device__ __forceinline__ float microfacet_distribution(bool beckmann, float n_dot_h, float alpha) {
    const float alpha2 = alpha * alpha;
    const float cosine2 = minf_(n_dot_h * n_dot_h, 1.0f);
    const float one_minus = 1.0f - cosine2;
    if (!beckmann) {
        const float den = one_minus + alpha2 * cosine2;
        return alpha2 / maxf_(kPi * den * den, 1.0e-20f);
    }
    const float exponent = one_minus / (cosine2 * alpha2);
    return 1.0f / (exp_(exponent) * kPi * alpha2 * cosine2 * cosine2);
}
__device__ __forceinline__ float microfacet_lambda(bool beckmann, float n_dot_v, float alpha) {
    const float cosine2 = n_dot_v * n_dot_v;
    const float sat = alpha * alpha * maxf_(1.0f / cosine2 - 1.0f, 0.0f);
    if (!beckmann) return 0.5f * (sqrtf(1.0f + sat) - 1.0f);
    const float a = 1.0f / sqrtf(sat);
    const float approximation = ((0.396f * a - 1.259f) * a + 1.0f) / ((2.181f * a + 3.535f) * a);
    return sat < 0.39f ? 0.0f : approximation;
}

// microfacet_intensity and microfacet_pdf (graph_surface_scattering.cpp:665-728)
// of a standalone glossy closure (Fresnel constant one: its colour is in
// the closure weight), in the corrected normal `gn`.
struct Microfacet {
    float intensity, pdf;
};
__device__ __noinline__ Microfacet microfacet_eval(uint32_t op, float roughness, f3 incoming, f3 outgoing, f3 gn,
                                                   float fresnel) {
    const bool beckmann = (op & kGlossyBeckmann) != 0u;
    const float ndv = maxf_(dot(gn, incoming), 0.0f);
    const float ndl = maxf_(dot(gn, outgoing), 0.0f);
    const f3 h = safe_normalize(incoming + outgoing, gn);
    const float ndh = maxf_(dot(gn, h), 0.0f);
    const float vdh = maxf_(dot(incoming, h), 0.0f);
    const bool singular = microfacet_singular(roughness);
    const float alpha = maxf_(microfacet_alpha(roughness), 1.0e-10f);
    const float d = microfacet_distribution(beckmann, ndh, alpha);
    const float lv = microfacet_lambda(beckmann, ndv, alpha);
    const float g = 1.0f / (1.0f + lv + microfacet_lambda(beckmann, ndl, alpha));
    const bool valid = ndv > 0.0f && ndl > 0.0f && ndh > 0.0f && vdh > 0.0f && !singular;
    Microfacet r;
    r.intensity = valid ? fresnel * d * g / maxf_(4.0f * ndv, 1.0e-20f) : 0.0f;
    r.pdf = valid ? d / maxf_(4.0f * ndv, 1.0e-20f) / (1.0f + lv) : 0.0f;
    return r;
}

// ---- glass and refraction (src/luisa/microfacet_glass_component.cpp) ----

// The closure normal of a glossy, glass or refraction closure after setup's
// specular-reflection correction (glass recomputes it: its `color` holds the tint).
__device__ __forceinline__ f3 microfacet_setup_normal(const PhysicalClosure &c, f3 diffuse_normal,
                                                      const ClosurePoint &pt) {
    return is_glass(c.op) ? specular_normal(pt.bump_correction, pt.geometric_normal, pt.view, diffuse_normal) : c.color;
}

struct GlassFresnel {
    f3 reflection, transmission;
};

// glass_fresnel / masked_fresnel (microfacet_glass_component.cpp:32-77) of a
// standalone Glass closure (F0 of its IOR, F90 one, both tints its colour:
// caustics on) or Refraction closure (no reflection; transmission one unless
// totally reflected).
__device__ __forceinline__ GlassFresnel glass_fresnel(const DielectricClosure &c, float cos_hi, bool reflection_allowed,
                                                      bool transmission_allowed) {
    const float real = fresnel_dielectric_cos(cos_hi, c.ior);
    GlassFresnel r;
    if (is_refraction(c.op)) {
        r.reflection = mk3(0.0f);
        r.transmission = real == 1.0f ? mk3(0.0f) : mk3(1.0f);
    } else {
        const float real_f0 = f0_from_ior(c.ior);
        const float t = clampf_((real - real_f0) / (1.0f - real_f0), 0.0f, 1.0f);
        const f3 fresnel = mk3(lerpf_(c.f0, 1.0f, t));
        r.reflection = fresnel * c.color;
        r.transmission = (mk3(1.0f) - fresnel) * c.color;
    }
    if (!reflection_allowed) r.reflection = mk3(0.0f);
    if (!transmission_allowed) r.transmission = mk3(0.0f);
    return r;
}

__device__ __forceinline__ float reflection_probability(const GlassFresnel &f) {
    const float r = closure_sample_weight(f.reflection);
    const float t = closure_sample_weight(f.transmission);
    return r / maxf_(r + t, 1.0e-20f);
}

// MicrofacetGlassComponent::intensity and ::pdf (microfacet_glass_component.cpp:79-109,
// 234-320): glass_geometry's half vector (the refractive one oriented by the
// IOR), D, Lambda, the Fresnel lobe of the side `outgoing` lies on, and the
// refraction Jacobian.
__device__ __noinline__ Microfacet glass_eval(const DielectricClosure &c, f3 incoming, f3 outgoing, f3 n,
                                              bool reflection_allowed, bool transmission_allowed, f3 &value) {
    const bool beckmann = (c.op & kGlossyBeckmann) != 0u;
    const float cos_o = dot(n, outgoing);
    const bool transmission = cos_o < 0.0f;
    const f3 uh = transmission ? -(outgoing * c.ior + incoming) : incoming + outgoing;
    const float hl = sqrtf(dot(uh, uh));
    const bool finite = hl != 0.0f && !(transmission && c.ior == 1.0f);
    const float inv_hl = finite ? 1.0f / hl : 0.0f;
    const f3 h = uh * inv_hl;
    const float cos_i = dot(n, incoming), cos_hi = dot(h, incoming), cos_nh = dot(n, h), cos_ho = dot(h, outgoing);
    const float setup_alpha = microfacet_alpha(c.roughness);
    const float alpha = maxf_(setup_alpha, 1.0e-7f);
    const float d = microfacet_distribution(beckmann, cos_nh, alpha);
    const float li = microfacet_lambda(beckmann, cos_i, alpha);
    const float lo = microfacet_lambda(beckmann, cos_o, alpha);
    const float jacobian = c.ior * c.ior * inv_hl * inv_hl * fabsf(cos_hi * cos_ho);
    const float common = d / cos_i * (transmission ? jacobian : 0.25f);
    const bool regular = setup_alpha * setup_alpha > kMicrofacetSingularAlphaProduct;
    // intensity (unmasked Fresnel)
    const GlassFresnel full = glass_fresnel(c, cos_hi, true, true);
    const f3 lobe = transmission ? full.transmission : full.reflection;
    value = (cos_i > 0.0f && regular) ? lobe * common / (1.0f + li + lo) * 1.0f : mk3(0.0f);
    // pdf (Fresnel masked by the enabled lobes)
    const GlassFresnel f = glass_fresnel(c, cos_hi, reflection_allowed, transmission_allowed);
    const float probability = reflection_probability(f);
    const float lobe_probability = transmission ? 1.0f - probability : probability;
    const float lobe_energy = transmission ? closure_sample_weight(f.transmission) : closure_sample_weight(f.reflection);
    Microfacet m;
    m.intensity = 0.0f;
    m.pdf = (cos_i > 0.0f && lobe_energy > 0.0f && regular) ? common / (1.0f + li) * lobe_probability : 0.0f;
    return m;
}

struct GlassSample {
    f3 direction, singular_evaluation;
    float singular_pdf;
    bool transmission, singular, valid;
};

// MicrofacetGlassComponent::sample (microfacet_glass_component.cpp:322-395).
__device__ __noinline__ GlassSample glass_sample(const DielectricClosure &c, f3 incoming, f3 gn, f3 ng, f2 random,
                                                 float random_lobe, bool reflection_allowed, bool transmission_allowed) {
    const float alpha = microfacet_alpha(c.roughness);
    bool singular = alpha * alpha <= kMicrofacetSingularAlphaProduct;
    const float sampling_alpha = maxf_(alpha, 1.0e-7f);
    f3 h = gn;
    if (!singular)
        h = (c.op & kGlossyBeckmann) != 0u ? sample_beckmann_visible_normal(gn, incoming, sampling_alpha, random)
                                           : sample_ggx_visible_normal(gn, incoming, sampling_alpha, random);
    const float cos_hi = dot(h, incoming);
    const GlassFresnel f = glass_fresnel(c, cos_hi, reflection_allowed, transmission_allowed);
    const float probability = reflection_probability(f);
    GlassSample r;
    r.transmission = random_lobe >= probability;
    const f3 reflected = h * (2.0f * cos_hi) - incoming;
    const float e2 = c.ior * c.ior - (1.0f - cos_hi * cos_hi);
    const float cos_ho = -sqrtf(maxf_(e2, 0.0f)) / c.ior;
    const float inverse_eta = 1.0f / c.ior;
    const f3 transmitted = h * (inverse_eta * cos_hi + cos_ho) - incoming * inverse_eta;
    r.direction = r.transmission ? transmitted : reflected;
    const f3 selected = r.transmission ? f.transmission : f.reflection;
    const float lobe_probability = r.transmission ? 1.0f - probability : probability;
    const bool shading_negative = dot(gn, r.direction) < 0.0f;
    const bool geometric_negative = dot(ng, r.direction) < 0.0f;
    const bool shading_ok = r.transmission ? shading_negative : !shading_negative;
    const bool geometric_ok = r.transmission ? geometric_negative : !geometric_negative;
    const bool has_energy = closure_sample_weight(f.reflection + f.transmission) > 0.0f;
    r.valid = has_energy && cos_hi > 0.0f && shading_ok && geometric_ok;
    r.singular = singular || (r.transmission && fabsf(c.ior - 1.0f) < 1.0e-4f);
    r.singular_evaluation = c.weight * selected * 1.0f * 1.0e6f;
    r.singular_pdf = lobe_probability * 1.0e6f;
    return r;
}

struct Evaluation {
    f3 f;
    float pdf;
    uint32_t events;
};

// oren_nayar_g (src/luisa/graph_surface_scattering.cpp:463-473).
__device__ __noinline__ float oren_nayar_g(float cosine) {
    const float c = clampf_(cosine, 0.0f, 1.0f);
    const float sine = sqrtf(maxf_(1.0f - c * c, 0.0f));
    const float theta = acos_(c);
    const float safe_cosine = maxf_(c, 1.0e-6f);
    const float regular = sine * (theta - 2.0f / 3.0f - sine * c) +
                          2.0f / 3.0f * (sine / safe_cosine) * (1.0f - sine * sine * sine);
    const float taylor = (kPi * 0.5f - 2.0f / 3.0f) - c;
    return c < 1.0e-6f ? taylor : regular;
}

// diffuse_intensity (src/luisa/graph_surface_scattering.cpp:475-506) of a
// closure whose clamped roughness `sigma` is at least 1e-5: Cycles'
// energy-compensated Oren-Nayar model (single scattering plus a multiple-
// scattering term from the clamped albedo).  `n` is the closure normal,
// `incoming` points to the viewer, `outgoing` to the light, nl = max(n.outgoing, 0).
// Below the cutoff the intensity is Lambert's nl / pi, which the callers
// evaluate inline.
__device__ __noinline__ f3 oren_nayar_intensity(const PhysicalClosure &c, float sigma, f3 n, f3 incoming,
                                                f3 outgoing, float nl) {
    const float a = 1.0f / (kPi + sigma * (kPi * 0.5f - 2.0f / 3.0f));
    const float b = sigma * a;
    const float nv = maxf_(dot(n, incoming), 0.0f);
    float t = dot(outgoing, incoming) - nl * nv;
    if (t > 0.0f) t = t / (maxf_(nl, nv) + 1.17549435e-38f);
    const float single_scatter = a + b * t;
    const f3 albedo = clamp3(c.color, 0.0f, 1.0f);
    const float e_average = a * kPi + ((2.0f * kPi - 5.6f) / 3.0f) * b;
    const float ratio = e_average / (1.0f - e_average);
    const float keep = 1.0f - e_average;
    const f3 e_ms = mk3(kInvPi * (albedo.x * albedo.x) * ratio / (1.0f - albedo.x * keep),
                        kInvPi * (albedo.y * albedo.y) * ratio / (1.0f - albedo.y * keep),
                        kInvPi * (albedo.z * albedo.z) * ratio / (1.0f - albedo.z * keep));
    const float e_incoming = a * kPi + b * oren_nayar_g(nv);
    const f3 multiscatter = e_ms * (1.0f - e_incoming);
    const float e_outgoing = a * kPi + b * oren_nayar_g(nl);
    return (mk3(single_scatter) + multiscatter * (1.0f - e_outgoing)) * nl;
}

// surface_closure_evaluation_contribution + accumulator
// (src/luisa/surface_closure_evaluation.cpp:61-438).  Every diffuse closure
// shares the closure normal, so the cosine, pdf and bump term are taken
// once; a glossy closure is evaluated in its corrected normal, and its bump
// term (which rejects a direction on the wrong side of the smooth surface
// unless the closure produced it) is its own.  Out of line: the shading
// kernel calls it for the light sample and for the BSDF sample, and a
// single copy keeps the kernel's code within the instruction cache.
template <bool kGlossy>
__device__ __noinline__ Evaluation evaluate_mixture(const SurfaceClosures<kGlossy> &s, const ClosurePoint &pt,
                                                    f3 outgoing_raw, uint32_t lobe_mask, int selected) {
    const f3 outgoing = safe_normalize(outgoing_raw, pt.shading_normal);
    // make_surface_closure_evaluation_directions (surface_closure_evaluation.cpp:61-70)
    const f3 incoming = pt.view;
    Evaluation e{mk3(0.0f), 0.0f, 0u};
    float total = 0.0f, weighted_pdf = 0.0f;
    const bool diffuse_enabled = (lobe_mask & kEventDiffuse) != 0u;
    const bool glossy_enabled = (lobe_mask & kEventGlossy) != 0u;
    const bool transparent_enabled = (lobe_mask & kEventTransparent) != 0u;
    const bool transmission_enabled = (lobe_mask & kEventTransmission) != 0u;
    const f3 n = s.normal;
    const float nl = maxf_(dot(n, outgoing), 0.0f);
    const float bump =
        s.normal_exact ? 1.0f : bump_shadowing_general(pt.shading_normal, n, outgoing, true, true, pt.bump_correction);
    const float lambert = nl * kInvPi;
    for (uint32_t i = 0; i < s.count; ++i) {
        const auto &c = s.c[i];
        if (c.op == PSY_CLOSURE_TRANSPARENT) {
            if (transparent_enabled) total += c.sample_weight;
            continue;
        }
        if constexpr (kGlossy) if (is_dielectric(c.op)) {
            // glass / refraction (surface_closure_evaluation.cpp:134-394): the side of
            // `outgoing` picks reflection or transmission; a selected transmission
            // keeps its bump term, and a selected unit-IOR transmission is a delta
            const bool is_selected = int(i) == selected;
            const f3 cn = microfacet_setup_normal(c, s.normal, pt);
            const f3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, cn);
            const bool transmission = dot(gn, outgoing) < 0.0f;
            const bool unit_ior_delta = is_selected && transmission && fabsf(c.ior - 1.0f) < 1.0e-4f;
            float gb = bump_shadowing(pt.shading_normal, cn, outgoing, !is_selected, false, pt.bump_correction);
            if (is_selected && transmission) gb = 1.0f;
            const bool allowed = is_glass(c.op) ? (transmission ? transmission_enabled : glossy_enabled)
                                                : (glossy_enabled && transmission_enabled);
            if (!allowed) continue;
            f3 intensity;
            const Microfacet m = glass_eval(c, incoming, outgoing, gn, glossy_enabled, transmission_enabled, intensity);
            const float pdf = ((gb != 0.0f || is_selected) && !unit_ior_delta) ? m.pdf : 0.0f;
            const f3 value = unit_ior_delta ? mk3(0.0f) : c.weight * intensity * gb;
            e.f = e.f + value;
            total += c.sample_weight;
            weighted_pdf += c.sample_weight * pdf;
            if (closure_sample_weight(value) > 0.0f)
                e.events |= kEventGlossy | (transmission ? kEventTransmission : kEventReflection);
            continue;
        }
        if constexpr (kGlossy) if (is_glossy(c.op)) {
            if (!glossy_enabled) continue;
            const bool is_selected = int(i) == selected;
            const float gb = bump_shadowing(pt.shading_normal, c.color, outgoing, !is_selected, false,
                                            pt.bump_correction);
            const f3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, c.color);
            // the glossy Fresnel factor: one, or MULTI_GGX's scale 1 / E
            // (microfacet_reflection_fresnel, graph_surface_scattering.cpp:632-662)
            const float fresnel = (c.op & kGlossyMultiscatter) != 0u ? c.f0 : 1.0f;
            const Microfacet m = microfacet_eval(c.op, c.roughness, incoming, outgoing, gn, fresnel);
            const float pdf = (gb != 0.0f || is_selected) ? m.pdf : 0.0f;
            const f3 value = c.weight * m.intensity * gb;
            e.f = e.f + value;
            total += c.sample_weight;
            weighted_pdf += c.sample_weight * pdf;
            if (closure_sample_weight(value) > 0.0f) e.events |= kEventGlossy | kEventReflection;
            continue;
        }
        const bool pdf_valid = bump != 0.0f || int(i) == selected;
        const float pdf = pdf_valid ? lambert : 0.0f;
        if (!diffuse_enabled) continue;
        const float sigma = clampf_(c.roughness, 0.0f, 1.0f);
        const f3 intensity = sigma < 1.0e-5f ? mk3(lambert) : oren_nayar_intensity(c, sigma, n, incoming, outgoing, nl);
        const f3 value = c.weight * intensity * bump;
        e.f = e.f + value;
        total += c.sample_weight;
        weighted_pdf += c.sample_weight * pdf;
        if (closure_sample_weight(value) > 0.0f) e.events |= kEventDiffuse | kEventReflection;
    }
    e.pdf = total > 0.0f ? weighted_pdf / maxf_(total, 1.0e-20f) : 0.0f;
    if (!(weighted_pdf > 0.0f)) e.events = 0u;
    return e;
}

struct SurfaceSample {
    bool valid;
    f3 wi;
    Evaluation eval;
    uint32_t closure_index;
};

// sample_microfacet_reflection (src/luisa/graph_surface_scattering.cpp:730-770)
// of a glossy closure with normal `cn`: the visible-normal half vector
// reflects the view, or at alpha^2 <= 2e-10 the mirror direction of the
// corrected normal; valid when the view and the direction lie above the
// corrected normal and the direction above the geometric surface.
struct GlossySample {
    f3 direction;
    bool valid, singular;
};
__device__ __noinline__ GlossySample sample_glossy(uint32_t op, float roughness, f3 cn, const ClosurePoint &pt,
                                                   f2 u_dir) {
    const f3 incoming = pt.view;
    const f3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, cn);
    const float alpha = microfacet_alpha(roughness);
    const float sampling_alpha = maxf_(alpha, 1.0e-10f);
    GlossySample g;
    g.singular = alpha * alpha <= kMicrofacetSingularAlphaProduct;
    if (g.singular) {
        g.direction = gn * (2.0f * dot(gn, incoming)) - incoming;
    } else {
        const f3 h = (op & kGlossyBeckmann) != 0u ? sample_beckmann_visible_normal(gn, incoming, sampling_alpha, u_dir)
                                                  : sample_ggx_visible_normal(gn, incoming, sampling_alpha, u_dir);
        g.direction = h * (2.0f * dot(incoming, h)) - incoming;
    }
    g.valid = dot(gn, incoming) > 0.0f && dot(gn, g.direction) > 0.0f && dot(pt.geometric_normal, g.direction) > 0.0f;
    return g;
}

__device__ __forceinline__ bool closure_eligible(uint32_t op, uint32_t lobe_mask) {
    if (op == PSY_CLOSURE_DIFFUSE) return (lobe_mask & kEventDiffuse) != 0u;
    if (is_glossy(op)) return (lobe_mask & kEventGlossy) != 0u;
    if (is_glass(op)) return (lobe_mask & (kEventGlossy | kEventTransmission)) != 0u;
    if (is_refraction(op)) return (lobe_mask & kEventGlossy) != 0u && (lobe_mask & kEventTransmission) != 0u;
    return (lobe_mask & kEventTransparent) != 0u;
}

// SurfaceClosureSamplingVisitor::visit (src/luisa/surface_closure_sampling_core.cpp:744-812;
// selection :97-214, categorical inversion :420-437, conditional sample
// :216-337 with the glossy sample_microfacet_reflection of
// graph_surface_scattering.cpp:730-770, finish :490-660).
template <bool kGlossy>
__device__ __forceinline__ SurfaceSample sample_surface(const SurfaceClosures<kGlossy> &s, const ClosurePoint &pt, float u_lobe,
                                                        f2 u_dir, uint32_t lobe_mask) {
    SurfaceSample out;
    out.valid = false;
    out.wi = mk3(0.0f);
    out.eval = {mk3(0.0f), 0.0f, 0u};
    out.closure_index = kInvalid;
    float total = 0.0f;
    for (uint32_t i = 0; i < s.count; ++i) total += closure_eligible(s.c[i].op, lobe_mask) ? s.c[i].sample_weight : 0.0f;
    const float random_lobe = clampf_(u_lobe, 0.0f, 0.99999994f);
    const float target = random_lobe * total;
    float accumulated = 0.0f;
    int chosen = -1;
    float chosen_weight = 0.0f, rescaled = random_lobe;
    for (uint32_t i = 0; i < s.count; ++i) {
        const float w = closure_eligible(s.c[i].op, lobe_mask) ? s.c[i].sample_weight : 0.0f;
        const float next = accumulated + w;
        if (chosen < 0 && w > 0.0f && target < next) {
            chosen = int(i);
            chosen_weight = w;
            // SurfaceClosureCategoricalInversion::consider (:420-437): the lobe
            // number rescaled into the chosen closure's interval
            if (s.count > 1u) rescaled = (target - accumulated) / maxf_(w, 1.0e-20f);
        }
        accumulated = next;
    }
    if (chosen < 0) return out;
    const auto c = s.c[chosen];
    const bool transparent = c.op == PSY_CLOSURE_TRANSPARENT;
    const bool glossy = kGlossy && is_glossy(c.op);
    const bool dielectric = kGlossy && is_dielectric(c.op);
    bool candidate_valid = true, singular = false, transmission = false;
    f3 direction, dielectric_delta = mk3(0.0f);
    float dielectric_pdf = 0.0f;
    if (transparent) {
        direction = -pt.incoming;
    } else if (glossy) {
        const GlossySample g = sample_glossy(c.op, c.roughness, c.color, pt, u_dir);
        direction = g.direction;
        candidate_valid = g.valid;
        singular = g.singular;
    } else if (!dielectric) {
        direction = sample_cosine_hemisphere(s.normal, u_dir, nullptr);
    }
    if constexpr (kGlossy) if (dielectric) {
        const f3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, pt.view,
                                      microfacet_setup_normal(c, s.normal, pt));
        const GlassSample g = glass_sample(c, pt.view, gn, pt.geometric_normal, u_dir, rescaled,
                                           (lobe_mask & kEventGlossy) != 0u, (lobe_mask & kEventTransmission) != 0u);
        direction = g.direction;
        candidate_valid = g.valid;
        singular = g.singular;
        transmission = g.transmission;
        dielectric_delta = g.singular_evaluation;
        dielectric_pdf = g.singular_pdf;
    }
    out.closure_index = uint32_t(chosen);
    out.wi = direction;
    const bool geometric_valid =
        transmission ? dot(pt.geometric_normal, direction) < 0.0f : dot(pt.geometric_normal, direction) > 0.0f;
    if (!(candidate_valid && (transparent || geometric_valid))) return out;
    const Evaluation mixture = evaluate_mixture<kGlossy>(s, pt, direction, lobe_mask, chosen);
    Evaluation r;
    r.f = mixture.f;
    float delta = 0.0f;
    if (transparent || (glossy && singular)) {
        // transparent: weight x 1e6; singular glossy: weight x Fresnel (one, or
        // MULTI_GGX's scale) x bump term (one when sampling a glossy closure) x 1e6
        if constexpr (kGlossy) {
            if (glossy && (c.op & kGlossyMultiscatter) != 0u) r.f = r.f + c.weight * c.f0 * 1.0e6f;
            else r.f = r.f + c.weight * 1.0e6f;
        } else {
            r.f = r.f + c.weight * 1.0e6f;
        }
        delta = 1.0e6f * chosen_weight;
    } else if (dielectric && singular) {
        r.f = r.f + dielectric_delta;
        delta = dielectric_pdf * chosen_weight;
    }
    r.pdf = mixture.pdf + delta / maxf_(total, 1.0e-20f);
    if (transparent) r.events = kEventTransmission | kEventTransparent;
    else if (dielectric)
        r.events = (singular ? kEventSingular : kEventGlossy) | (transmission ? kEventTransmission : kEventReflection);
    else if (glossy) r.events = singular ? (kEventSingular | kEventReflection) : (kEventGlossy | kEventReflection);
    else r.events = kEventDiffuse | kEventReflection;
    out.eval = r;
    out.valid = true;
    return out;
}

// AOV visitor (src/luisa/surface_closure_operations.cpp:40-161, 402-462):
// diffuse colour into Albedo, every diffuse and glossy normal (glossy:
// corrected) weighted by |average weight| into Normal.
template <bool kGlossy>
__device__ __forceinline__ void surface_aov(const SurfaceClosures<kGlossy> &s, const ClosurePoint &pt, f3 &albedo, f3 &normal,
                                            f3 &transparency) {
    albedo = mk3(0.0f);
    transparency = mk3(0.0f);
    f3 n = mk3(0.0f);
    float total = 0.0f;
    for (uint32_t i = 0; i < s.count; ++i) {
        const auto &c = s.c[i];
        if (c.op == PSY_CLOSURE_DIFFUSE) {
            albedo = albedo + c.weight;
            const float w = closure_sample_weight(c.weight);
            n = n + s.normal * w;
            total += w;
        } else if (kGlossy && (is_glossy(c.op) || is_dielectric(c.op))) {
            const float w = closure_sample_weight(c.weight);
            n = n + specular_normal(pt.bump_correction, pt.geometric_normal, pt.view, microfacet_setup_normal(c, s.normal, pt)) * w;
            total += w;
        } else {
            transparency = transparency + c.weight;
        }
    }
    normal = safe_normalize(total > 0.0f ? n : pt.shading_normal, pt.shading_normal);
}

// ---------------------------------------------------------- intersection

struct Ray {
    f3 o, d;
    float tmin, tmax;
};

struct Hit {
    float t, u, v;
    uint32_t instance, prim, object, cycles_prim;
};

// clamp_bvh_direction (cycles_triangle_intersection_component.cpp:31-37).
__device__ __forceinline__ float clamp_bvh_direction(float v) {
    const float m = 8.271806e-25f;
    return fabsf(v) > m ? v : copysignf(m, v);
}

__device__ __forceinline__ f3 pl_cross(f3 a, f3 b) {
    return {fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x))};
}
__device__ __forceinline__ float pl_dot(f3 a, f3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }

// PlueckerTriangleIntersectionComponent::intersect
// (cycles_triangle_intersection_component.cpp:39-105).
__device__ __forceinline__ bool intersect_triangle(f3 o, f3 d, float tmin, float tmax, f3 p0, f3 p1, f3 p2,
                                                   float &t_out, float &u_out, float &v_out) {
    const f3 v0 = p0 - o, v1 = p1 - o, v2 = p2 - o;
    const f3 e0 = v2 - v0, e1 = v0 - v1, e2 = v1 - v2;
    const float u = pl_dot(pl_cross(e0, v2 + v0), d);
    const float v = pl_dot(pl_cross(e1, v0 + v1), d);
    const float w = pl_dot(pl_cross(e2, v1 + v2), d);
    const float sum = u + v + w;
    const float tol = 1.1920928955078125e-07f * fabsf(sum);
    const float mn = minf_(u, minf_(v, w));
    const float mx = maxf_(u, maxf_(v, w));
    if (!((mn >= -tol) || (mx <= tol))) return false;
    const f3 n2 = pl_cross(e1, e0) * 2.0f;
    const float den = pl_dot(n2, d);
    if (den == 0.0f) return false;
    const float t = pl_dot(v0, n2) / den;
    if (!((t >= tmin) && (t <= tmax))) return false;
    const float rs = fabsf(sum) >= 1.0e-18f ? 1.0f / sum : 0.0f;
    t_out = t;
    u_out = minf_(u * rs, 1.0f);
    v_out = minf_(v * rs, 1.0f);
    return true;
}

__device__ __forceinline__ Xform load_xform(const float *m) {
    return {ld3(m), ld3(m + 3), ld3(m + 6), ld3(m + 9)};
}

// A wide node as one ray sees it: per axis the plane a ray of that
// direction sign enters through (near) and leaves through (far).
struct WideNodeRay {
    float4 nx, fx, ny, fy, nz, fz;
    int4 link, count;
};

// Loads a wide node with its planes ordered by the ray's direction signs
// (`neg` bit a set where the direction's component a is negative), so the
// slab test needs no min / max per axis.
__device__ __forceinline__ WideNodeRay load_wide_node(const WideNodeGpu *nodes, uint32_t idx, uint32_t neg) {
    const float4 *p = reinterpret_cast<const float4 *>(nodes + idx);
    const uint32_t sx = neg & 1u, sy = (neg >> 1) & 1u, sz = (neg >> 2) & 1u;
    WideNodeRay n;
    n.nx = __ldg(p + sx);
    n.fx = __ldg(p + (1u - sx));
    n.ny = __ldg(p + 2u + sy);
    n.fy = __ldg(p + (3u - sy));
    n.nz = __ldg(p + 4u + sz);
    n.fz = __ldg(p + (5u - sz));
    const int4 *q = reinterpret_cast<const int4 *>(p + 6);
    n.link = __ldg(q);
    n.count = __ldg(q + 1);
    return n;
}

// Slab test of the four children of a wide node, conservative as the
// boxes are padded at build time and the far bound is widened by a
// relative 2^-20.  Empty slots hold +inf planes on every axis, which give
// an entry distance of +inf or an exit distance of -inf, so they never hit.
__device__ __forceinline__ void wide_slabs(const WideNodeRay &n, f3 oinv, f3 inv, float tmin, float tmax,
                                           float near[4], bool hit[4]) {
    const float nx[4] = {n.nx.x, n.nx.y, n.nx.z, n.nx.w}, fx[4] = {n.fx.x, n.fx.y, n.fx.z, n.fx.w};
    const float ny[4] = {n.ny.x, n.ny.y, n.ny.z, n.ny.w}, fy[4] = {n.fy.x, n.fy.y, n.fy.z, n.fy.w};
    const float nz[4] = {n.nz.x, n.nz.y, n.nz.z, n.nz.w}, fz[4] = {n.fz.x, n.fz.y, n.fz.z, n.fz.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float x0 = fmaf(nx[k], inv.x, -oinv.x), x1 = fmaf(fx[k], inv.x, -oinv.x);
        const float y0 = fmaf(ny[k], inv.y, -oinv.y), y1 = fmaf(fy[k], inv.y, -oinv.y);
        const float z0 = fmaf(nz[k], inv.z, -oinv.z), z1 = fmaf(fz[k], inv.z, -oinv.z);
        const float nr = fmaxf(fmaxf(x0, y0), fmaxf(z0, tmin));
        const float fr = fminf(fminf(x1, y1), fminf(z1, tmax));
        near[k] = nr;
        hit[k] = nr <= fmaxf(fmaf(fr, 1.00000095367431640625f, 1.0e-30f), fr);
    }
}

constexpr int kStackSize = int(kTraversalStackSize);

// Scene compile bounds every tree's worst-case stack by kTraversalStackSize
// (blas_stack_need / tlas_instance_depths in psy_host.cpp) and rejects a
// scene it cannot bound, so no push can find the stack full.  A debug build
// (-DPSY_STACK_CHECK=1) also counts such pushes in g_stack_overflows, which
// fails the render; the count's atomic costs about 10 % of the frame in the
// traversal kernels, so release builds keep the plain guarded push.
#ifndef PSY_STACK_CHECK
#define PSY_STACK_CHECK 0
#endif
__device__ unsigned int g_stack_overflows;

__device__ __forceinline__ void stack_push(uint32_t *stack, uint32_t &sp, uint32_t entry) {
#if PSY_STACK_CHECK
    if (sp < uint32_t(kStackSize)) stack[sp++] = entry;
    else atomicAdd(&g_stack_overflows, 1u);
#else
    if (sp < uint32_t(kStackSize)) stack[sp++] = entry;
#endif
}


__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct SlabRay {
    f3 o, d, inv, oinv;  // origin, clamped direction, reciprocal, origin * reciprocal
    uint32_t neg;        // bit a: direction component a is negative
};

__device__ __forceinline__ SlabRay make_slab_ray(f3 o, f3 raw) {
    SlabRay r;
    r.o = o;
    r.d = mk3(clamp_bvh_direction(raw.x), clamp_bvh_direction(raw.y), clamp_bvh_direction(raw.z));
    // the slab test only has to be conservative, which its padding and far
    // widening keep with the hardware's approximate reciprocal (relative
    // error below 2^-22); the triangle test uses the clamped direction itself
    r.inv = mk3(rcp_approx(r.d.x), rcp_approx(r.d.y), rcp_approx(r.d.z));
    r.oinv = mk3(o.x * r.inv.x, o.y * r.inv.y, o.z * r.inv.z);
    r.neg = (r.d.x < 0.0f ? 1u : 0u) | (r.d.y < 0.0f ? 2u : 0u) | (r.d.z < 0.0f ? 4u : 0u);
    return r;
}

// Resumable two-level traversal.  TLAS and BLAS nodes share one loop body
// so the lanes of a warp stay on the same instruction stream while their
// rays sit at different levels; the state lives in registers (stack in
// local memory) so a persistent kernel can advance a ray a few nodes at a
// time and hand the lane a new ray when it finishes.  Every triangle
// accepted by the Pluecker predicate in [tmin, tmax] (`tmax` shrinks as the
// visitor requests) that is neither the source nor the light identity is
// handed to `on_hit(instance, local, cycles_prim, t, u, v)`; a true return
// ends the traversal.
#if PSY_BVH_WIDTH != 8
struct TraversalState {
    Ray ray;      // world ray
    SlabRay cur;  // slab ray of the current level
    float tmax;
    uint32_t node, sp, inst, prim_offset;
    uint32_t visibility, src_obj, src_prim, light_obj, light_prim;
    uint32_t stack[kStackSize];
};

__device__ __forceinline__ void traversal_begin(TraversalState &t, const SceneView &s, const Ray &ray,
                                                uint32_t visibility, uint32_t src_obj, uint32_t src_prim,
                                                uint32_t light_obj, uint32_t light_prim) {
    t.ray = ray;
    t.cur = make_slab_ray(ray.o, ray.d);
    t.tmax = ray.tmax;
    t.node = s.instance_count == 0u ? kTagLeave : kTagTlas;
    t.sp = 0u;
    t.inst = kInvalid;
    t.prim_offset = 0u;
    t.visibility = visibility;
    t.src_obj = src_obj;
    t.src_prim = src_prim;
    t.light_obj = light_obj;
    t.light_prim = light_prim;
}

// Advances at most `budget` loop iterations; true once the traversal ended.
// kNearFirst orders a node's hit children nearest first (closest hit);
// without it they are pushed in slot order (any-hit queries, which visit
// every candidate or stop at the first blocker regardless of order).
template <bool kNearFirst = true, typename OnHit>
__device__ __forceinline__ bool traversal_steps(TraversalState &t, const SceneView &s, int budget, OnHit on_hit) {
    for (int it = 0; it < budget; ++it) {
        const uint32_t tag = t.node & kTagMask;
        const uint32_t idx = t.node & ~kTagMask;
        if (tag == kTagInstance) {
            const InstanceGpu &in = s.instances[idx];
            if ((in.visibility & t.visibility) != 0u) {
                const MeshGpu mesh = s.meshes[in.mesh];
                const Xform w2o = load_xform(in.w2o);
                t.cur = make_slab_ray(xform_point(w2o, t.ray.o), xform_direction(w2o, t.ray.d));
                t.inst = idx;
                t.prim_offset = mesh.prim_offset;
                stack_push(t.stack, t.sp, kTagLeave);
                t.node = kTagBlas | mesh.node_offset;
                continue;
            }
            if (t.sp == 0u) return true;
            t.node = t.stack[--t.sp];
            continue;
        }
        if (tag == kTagLeave) {
            if (t.inst != kInvalid) {
                t.cur = make_slab_ray(t.ray.o, t.ray.d);
                t.inst = kInvalid;
            }
            if (t.sp == 0u) return true;
            t.node = t.stack[--t.sp];
            continue;
        }
        const bool blas = tag == kTagBlas;
        const WideNodeRay n = load_wide_node(blas ? s.blas : s.tlas, idx, t.cur.neg);
        float near[4];
        bool hit[4];
        wide_slabs(n, t.cur.oinv, t.cur.inv, t.ray.tmin, t.tmax, near, hit);
        // a slot's link is a ready stack entry (tagged global node index or
        // tagged instance) when its count is 0, else its first triangle
        const uint32_t lk[4] = {uint32_t(n.link.x), uint32_t(n.link.y), uint32_t(n.link.z), uint32_t(n.link.w)};
        const int ct[4] = {n.count.x, n.count.y, n.count.z, n.count.w};
        // leaves first: their triangles may shrink tmax before the inner
        // children are ordered.  The hit leaf slots are walked as a bit set
        // through one copy of the triangle test, so lanes whose leaves sit
        // in different slots test them together.
        if (blas) {
            uint32_t leaves = 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (hit[k] && ct[k] != 0) leaves |= 1u << k;
            while (leaves != 0u) {
                const uint32_t k = uint32_t(__ffs(int(leaves)) - 1);
                leaves &= leaves - 1u;
                const uint32_t first = k == 0u ? lk[0] : k == 1u ? lk[1] : k == 2u ? lk[2] : lk[3];
                const int cnt = k == 0u ? ct[0] : k == 1u ? ct[1] : k == 2u ? ct[2] : ct[3];
                for (int q = 0; q < cnt; ++q) {
                    const float4 *tp = s.tris + 3u * (first + uint32_t(q));
                    const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
                    const uint32_t local = __float_as_uint(a.w);
                    const uint32_t cp = t.prim_offset + local;
                    if ((t.src_obj == t.inst && t.src_prim == cp) || (t.light_obj == t.inst && t.light_prim == cp))
                        continue;
                    float th, u, v;
                    if (!intersect_triangle(t.cur.o, t.cur.d, t.ray.tmin, t.tmax, ld3(a), ld3(b), ld3(c), th, u, v))
                        continue;
                    if (on_hit(t.inst, local, cp, th, u, v)) return true;
                }
            }
        }
        if constexpr (!kNearFirst) {
            uint32_t next = kInvalid;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!(hit[k] && near[k] <= t.tmax && ct[k] == 0)) continue;
                if (next != kInvalid) stack_push(t.stack, t.sp, next);
                next = lk[k];
            }
            if (next == kInvalid) {
                if (t.sp == 0u) return true;
                next = t.stack[--t.sp];
            }
            t.node = next;
        } else {
            // inner children (and TLAS instances) nearest first: sort the four
            // (distance, entry) pairs, misses last
            float key[4];
            uint32_t val[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const bool take = hit[k] && near[k] <= t.tmax && ct[k] == 0;
                key[k] = take ? near[k] : __int_as_float(0x7f800000);
                val[k] = lk[k];
            }
#define PSY_CSWAP(i, j)                 \
    if (key[j] < key[i]) {              \
        const float tk = key[i];        \
        key[i] = key[j];                \
        key[j] = tk;                    \
        const uint32_t tv = val[i];     \
        val[i] = val[j];                \
        val[j] = tv;                    \
    }
            PSY_CSWAP(0, 1)
            PSY_CSWAP(2, 3)
            PSY_CSWAP(0, 2)
            PSY_CSWAP(1, 3)
            PSY_CSWAP(1, 2)
#undef PSY_CSWAP
            const float kInf = __int_as_float(0x7f800000);
            if (key[0] == kInf) {
                if (t.sp == 0u) return true;
                t.node = t.stack[--t.sp];
                continue;
            }
#pragma unroll
            for (int k = 3; k >= 1; --k)
                if (key[k] != kInf) stack_push(t.stack, t.sp, val[k]);
            t.node = val[0];
        }
    }
    return false;
}

#else  // PSY_BVH_WIDTH == 8

// Group-stack traversal of the compressed 8-wide trees (after Ylitie,
// Karras and Laine 2017).  A visit tests the node's eight quantised boxes
// one child at a time (one FMA per plane after a per-node change of
// variables), tests hit leaf triangles at once, and continues into the hit
// inner child of lowest octant-remapped bit (near first for the ray's
// direction octant), leaving the node's other hit children as ONE stack
// entry (base, hit bits, inner mask).  In the TLAS the hit instances are
// entered one by one from an instance-group entry, each behind a marker
// that returns to the world ray.  Every triangle whose box the ray reaches
// within [tmin, tmax] is tested, as in the 4-wide traversal, so the closest
// hit does not depend on the order.
constexpr int kStackSize8 = int(kTraversalStackSize8);
constexpr uint32_t kNoNode = 0xffffffffu;

struct TraversalState {
    Ray ray;      // world ray
    SlabRay cur;  // slab ray of the current level
    float tmax;
    uint32_t node, sp, inst, prim_offset;  // node: tagged node to visit, or kNoNode (pop)
    uint32_t visibility, src_obj, src_prim, light_obj, light_prim;
    uint2 stack[kStackSize8];  // x: tag | base index, y: hit bits (0-7) | child or leaf mask (8-15)
};

__device__ __forceinline__ void traversal_begin(TraversalState &t, const SceneView &s, const Ray &ray,
                                                uint32_t visibility, uint32_t src_obj, uint32_t src_prim,
                                                uint32_t light_obj, uint32_t light_prim) {
    t.ray = ray;
    t.cur = make_slab_ray(ray.o, ray.d);
    t.tmax = ray.tmax;
    t.node = s.instance_count == 0u ? kNoNode : kTagTlas;
    t.sp = 0u;
    t.inst = kInvalid;
    t.prim_offset = 0u;
    t.visibility = visibility;
    t.src_obj = src_obj;
    t.src_prim = src_prim;
    t.light_obj = light_obj;
    t.light_prim = light_prim;
}

__device__ __forceinline__ void stack_push8(TraversalState &t, uint32_t x, uint32_t y) {
    if (t.sp < uint32_t(kStackSize8)) t.stack[t.sp++] = make_uint2(x, y);
}

// Enters instance `i` (object-space slab ray, return marker) when the ray
// may see it; otherwise the next entry is popped.
__device__ __forceinline__ void enter_instance8(TraversalState &t, const SceneView &s, uint32_t i) {
    const InstanceGpu &in = s.instances[i];
    if ((in.visibility & t.visibility) == 0u) {
        t.node = kNoNode;
        return;
    }
    const MeshGpu mesh = s.meshes[in.mesh];
    const Xform w2o = load_xform(in.w2o);
    t.cur = make_slab_ray(xform_point(w2o, t.ray.o), xform_direction(w2o, t.ray.d));
    t.inst = i;
    t.prim_offset = mesh.prim_offset;
    stack_push8(t, kTagLeave, 0u);
    t.node = kTagBlas | mesh.node_offset;
}

__device__ __forceinline__ uint32_t below(uint32_t mask, uint32_t bit) { return __popc(mask & ((1u << bit) - 1u)); }

// Advances at most `budget` loop iterations; true once the traversal ended.
// The octant order serves closest-hit and any-hit queries alike.
template <bool kNearFirst = true, typename OnHit>
__device__ __forceinline__ bool traversal_steps(TraversalState &t, const SceneView &s, int budget, OnHit on_hit) {
    for (int it = 0; it < budget; ++it) {
        if (t.node == kNoNode) {
            if (t.sp == 0u) return true;
            const uint2 e = t.stack[t.sp - 1u];
            const uint32_t tag = e.x & kTagMask;
            if (tag == kTagLeave) {
                t.cur = make_slab_ray(t.ray.o, t.ray.d);
                t.inst = kInvalid;
                --t.sp;
                continue;
            }
            const uint32_t bits = e.y & 0xffu, mask = (e.y >> 8) & 0xffu;
            const uint32_t b = uint32_t(__ffs(int(bits)) - 1);
            const uint32_t rest = bits & (bits - 1u);
            if (rest != 0u) t.stack[t.sp - 1u].y = rest | (mask << 8);
            else --t.sp;
            if (tag == kTagInstance) {
                enter_instance8(t, s, s.tlas_ids[(e.x & ~kTagMask) + below(mask, b)]);
            } else {
                t.node = tag | ((e.x & ~kTagMask) + below(mask, b ^ t.cur.neg));
            }
            continue;
        }
        const uint32_t tag = t.node & kTagMask;
        const bool blas = tag == kTagBlas;
        const float4 *np = reinterpret_cast<const float4 *>((blas ? s.blas8 : s.tlas8) + (t.node & ~kTagMask));
        const float4 w0 = __ldg(np);
        const uint4 w1 = __ldg(reinterpret_cast<const uint4 *>(np + 1));
        const uint4 w2 = __ldg(reinterpret_cast<const uint4 *>(np + 2));
        const uint4 w3 = __ldg(reinterpret_cast<const uint4 *>(np + 3));
        const uint4 w4 = __ldg(reinterpret_cast<const uint4 *>(np + 4));
        const uint32_t em = __float_as_uint(w0.w);
        const uint32_t imask = em >> 24, leafmask = w1.z;
        // slab distances of child k: t = q * (cell * inv) + (p - o) * inv
        const SlabRay &r = t.cur;
        const float ax = __uint_as_float((em & 0xffu) << 23) * r.inv.x;
        const float ay = __uint_as_float(((em >> 8) & 0xffu) << 23) * r.inv.y;
        const float az = __uint_as_float(((em >> 16) & 0xffu) << 23) * r.inv.z;
        const float bx = (w0.x - r.o.x) * r.inv.x;
        const float by = (w0.y - r.o.y) * r.inv.y;
        const float bz = (w0.z - r.o.z) * r.inv.z;
        // near / far byte planes by direction sign: lo x (w2.x, w2.y), lo y
        // (w2.z, w2.w), lo z (w3.x, w3.y), hi x (w3.z, w3.w), hi y (w4.x,
        // w4.y), hi z (w4.z, w4.w)
        const bool nx = (r.neg & 1u) != 0u, ny = (r.neg & 2u) != 0u, nz = (r.neg & 4u) != 0u;
        const uint32_t nx0 = nx ? w3.z : w2.x, nx1 = nx ? w3.w : w2.y, fx0 = nx ? w2.x : w3.z, fx1 = nx ? w2.y : w3.w;
        const uint32_t ny0 = ny ? w4.x : w2.z, ny1 = ny ? w4.y : w2.w, fy0 = ny ? w2.z : w4.x, fy1 = ny ? w2.w : w4.y;
        const uint32_t nz0 = nz ? w4.z : w3.x, nz1 = nz ? w4.w : w3.y, fz0 = nz ? w3.x : w4.z, fz1 = nz ? w3.y : w4.w;
        const uint32_t occupied = imask | leafmask;
        uint32_t hit_inner = 0u, hit_leaf = 0u;
        const float tmin = t.ray.tmin, tmax = t.tmax;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (((occupied >> k) & 1u) == 0u) continue;
            const int sh = 8 * (k & 3);
            const bool hi_word = k >= 4;
            const float qnx = float(((hi_word ? nx1 : nx0) >> sh) & 0xffu);
            const float qfx = float(((hi_word ? fx1 : fx0) >> sh) & 0xffu);
            const float qny = float(((hi_word ? ny1 : ny0) >> sh) & 0xffu);
            const float qfy = float(((hi_word ? fy1 : fy0) >> sh) & 0xffu);
            const float qnz = float(((hi_word ? nz1 : nz0) >> sh) & 0xffu);
            const float qfz = float(((hi_word ? fz1 : fz0) >> sh) & 0xffu);
            const float nr = fmaxf(fmaxf(fmaf(qnx, ax, bx), fmaf(qny, ay, by)), fmaxf(fmaf(qnz, az, bz), tmin));
            const float fr = fminf(fminf(fmaf(qfx, ax, bx), fmaf(qfy, ay, by)), fminf(fmaf(qfz, az, bz), tmax));
            if (nr <= fmaxf(fmaf(fr, 1.00000095367431640625f, 1.0e-30f), fr)) {
                if ((imask >> k) & 1u) hit_inner |= 1u << (uint32_t(k) ^ r.neg);
                else hit_leaf |= 1u << k;
            }
        }
        if (blas) {
            // leaves first: their triangles may shrink tmax
            while (hit_leaf != 0u) {
                const uint32_t k = uint32_t(__ffs(int(hit_leaf)) - 1);
                hit_leaf &= hit_leaf - 1u;
                const float4 *tp = s.tris + 3u * (w1.y + below(leafmask, k));
                const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
                const uint32_t local = __float_as_uint(a.w);
                const uint32_t cp = t.prim_offset + local;
                if ((t.src_obj == t.inst && t.src_prim == cp) || (t.light_obj == t.inst && t.light_prim == cp)) continue;
                float th, u, v;
                if (!intersect_triangle(t.cur.o, t.cur.d, t.ray.tmin, t.tmax, ld3(a), ld3(b), ld3(c), th, u, v))
                    continue;
                if (on_hit(t.inst, local, cp, th, u, v)) return true;
            }
        } else if (hit_leaf != 0u) {
            // TLAS: stack the inner hits, then enter the hit instances one by one
            if (hit_inner != 0u) stack_push8(t, kTagTlas | w1.x, hit_inner | (imask << 8));
            const uint32_t k = uint32_t(__ffs(int(hit_leaf)) - 1);
            const uint32_t rest = hit_leaf & (hit_leaf - 1u);
            if (rest != 0u) stack_push8(t, kTagInstance | w1.y, rest | (leafmask << 8));
            enter_instance8(t, s, s.tlas_ids[w1.y + below(leafmask, k)]);
            continue;
        }
        if (hit_inner == 0u) {
            t.node = kNoNode;
            continue;
        }
        const uint32_t b = uint32_t(__ffs(int(hit_inner)) - 1);
        const uint32_t rest = hit_inner & (hit_inner - 1u);
        if (rest != 0u) stack_push8(t, tag | w1.x, rest | (imask << 8));
        t.node = tag | (w1.x + below(imask, b ^ r.neg));
    }
    return false;
}

#endif  // PSY_BVH_WIDTH

// Whole traversal in one call.
template <typename OnHit>
__device__ __forceinline__ void traverse_scene(const SceneView &s, const Ray &ray, uint32_t visibility,
                                               uint32_t src_obj, uint32_t src_prim, uint32_t light_obj,
                                               uint32_t light_prim, float &tmax, OnHit on_hit) {
    TraversalState t;
    traversal_begin(t, s, ray, visibility, src_obj, src_prim, light_obj, light_prim);
    t.tmax = tmax;
    while (!traversal_steps(t, s, 1 << 30, [&](uint32_t ii, uint32_t local, uint32_t cp, float th, float u, float v) {
        const bool stop = on_hit(ii, local, cp, th, u, v);
        t.tmax = tmax;
        return stop;
    })) {
    }
}

// Closest hit of the whole scene under the Cycles predicate
// (UnifiedSceneTraversalComponent::trace, src/luisa/path_kernel_scene_traversal.cpp:301-490):
// closed [tmin, tmax], exclusion of the source and light identities, and
// equal distances resolved to the greatest (object, primitive).
__device__ __forceinline__ bool trace_closest(const SceneView &s, const Ray &ray, uint32_t visibility,
                                              uint32_t src_obj, uint32_t src_prim, uint32_t light_obj,
                                              uint32_t light_prim, Hit &best) {
    bool has = false;
    best.t = ray.tmax;
    best.u = best.v = 0.0f;
    best.instance = best.prim = best.object = best.cycles_prim = kInvalid;
    float tmax = ray.tmax;
    traverse_scene(s, ray, visibility, src_obj, src_prim, light_obj, light_prim, tmax,
                   [&](uint32_t ii, uint32_t local, uint32_t cp, float t, float u, float v) {
                       const bool later = ii > best.object || (ii == best.object && cp > best.cycles_prim);
                       if (has && !(t < best.t || (t == best.t && later))) return false;
                       has = true;
                       best.t = t;
                       best.u = u;
                       best.v = v;
                       best.instance = ii;
                       best.prim = local;
                       best.object = ii;
                       best.cycles_prim = cp;
                       tmax = t;
                       return false;
                   });
    return has;
}

// ---------------------------------------------------------- hit geometry

struct SurfacePoint {
    f3 position, object_position, ng, n;
    f3 p0, p1, p2, wp0, wp1, wp2;
    bool back_facing;
    uint32_t instance, material, object, cycles_prim;
};

__device__ __forceinline__ f3 tri_interp(float u, float v, f3 a, f3 b, f3 c) {
    return a * (1.0f - u - v) + b * u + c * v;
}

// FinalSupportTriangleSurfaceComponent::resolve (src/luisa/cycles_triangle_surface_component.cpp:9-95)
// for instanced meshes.
__device__ __forceinline__ SurfacePoint surface_point(const SceneView &s, const Hit &h, f3 ray_d) {
    SurfacePoint sp;
    const InstanceGpu &inst = s.instances[h.instance];
    const MeshGpu mesh = s.meshes[inst.mesh];
    const uint32_t *idx = s.indices + mesh.index_offset + 3u * h.prim;
    const uint32_t i0 = idx[0], i1 = idx[1], i2 = idx[2];
    const float *P = s.positions + 3u * mesh.vertex_offset;
    sp.p0 = ld3(P + 3u * i0);
    sp.p1 = ld3(P + 3u * i1);
    sp.p2 = ld3(P + 3u * i2);
    const Xform o2w = load_xform(inst.o2w);
    const Xform nrm = load_xform(inst.nrm);
    sp.wp0 = xform_point(o2w, sp.p0);
    sp.wp1 = xform_point(o2w, sp.p1);
    sp.wp2 = xform_point(o2w, sp.p2);
    const f3 ogn = safe_normalize(cross(sp.p1 - sp.p0, sp.p2 - sp.p0), mk3(0.0f, 0.0f, 1.0f));
    f3 ng = safe_normalize(xform_direction(nrm, ogn), -ray_d);
    f3 osn = ogn;
    if (mesh.smooth) {
        const float *N = s.normals + 3u * mesh.vertex_offset;
        osn = tri_interp(h.u, h.v, ld3(N + 3u * i0), ld3(N + 3u * i1), ld3(N + 3u * i2));
    }
    f3 n = safe_normalize(xform_direction(nrm, osn), ng);
    sp.back_facing = dot(ng, -ray_d) < 0.0f;
    if (sp.back_facing) {
        ng = -ng;
        n = -n;
    }
    if (dot(n, ng) < 0.0f) n = -n;
    sp.ng = ng;
    sp.n = n;
    sp.object_position = sp.p0 + (sp.p1 - sp.p0) * h.u + (sp.p2 - sp.p0) * h.v;
    sp.position = xform_point(o2w, sp.object_position);
    sp.instance = h.instance;
    sp.material = mesh.material_offset == kInvalid ? inst.material : s.tri_materials[mesh.material_offset + h.prim];
    sp.object = h.object;
    sp.cycles_prim = h.cycles_prim;
    return sp;
}

// Wachter & Binder robust offset (Ray Tracing Gems ch. 6), the published
// method behind Luisa's offset_ray_origin.
__device__ __forceinline__ float offset_component(float p, float n) {
    const float origin = 1.0f / 32.0f, float_scale = 1.0f / 65536.0f, int_scale = 256.0f;
    const int of_i = static_cast<int>(int_scale * n);
    const float p_i = __int_as_float(__float_as_int(p) + (p < 0.0f ? -of_i : of_i));
    return fabsf(p) < origin ? p + float_scale * n : p_i;
}

// origin_with_explicit_self_exclusion (include/psycles/luisa/surface_ray.h:49-100).
__device__ __forceinline__ f3 origin_with_self_exclusion(const SurfacePoint &sp, f3 oo, f3 od) {
    const f3 v0 = sp.p0 - oo, v1 = sp.p1 - oo, v2 = sp.p2 - oo;
    const f3 e0 = v2 - v0, e1 = v0 - v1, e2 = v1 - v2;
    const float u = dot(cross(v2 + v0, e0), od);
    const float v = dot(cross(v0 + v1, e1), od);
    const float w = dot(cross(v1 + v2, e2), od);
    const float eps = 1.1920928955078125e-07f * fabsf(u + v + w);
    const float mn = minf_(u, minf_(v, w)), mx = maxf_(u, maxf_(v, w));
    if ((mn >= eps) || (mx <= -eps)) return sp.position;
    return mk3(offset_component(sp.position.x, sp.ng.x), offset_component(sp.position.y, sp.ng.y),
               offset_component(sp.position.z, sp.ng.z));
}

// ------------------------------------------------------- light sampling

// The flat light distribution's pick (src/luisa/path_tracer_light_distribution.cpp:12-55):
// the search for the first entry whose cumulative value exceeds u, then the
// entry before it.
__device__ __forceinline__ DistEntryGpu distribution_sample(const SceneView &s, float u) {
    if (s.emitter_count == 0u) return {0.0f, 0.0f, 3u, 0u};
    uint32_t first = 0u, length = s.emitter_count + 1u;
    while (length > 0u) {
        const uint32_t half = length >> 1u;
        const uint32_t middle = first + half;
        if (u < s.distribution[middle].cumulative) {
            length = half;
        } else {
            first = middle + 1u;
            length = length - half - 1u;
        }
    }
    uint32_t selected = first > 0u ? first - 1u : 0u;
    selected = min(selected, s.emitter_count - 1u);
    return s.distribution[selected];
}

__device__ __forceinline__ float triangle_solid_angle(f3 r, f3 p0, f3 p1, f3 p2) {
    const f3 a = normalize_or(p0 - r, mk3(1.0f, 0.0f, 0.0f));
    const f3 b = normalize_or(p1 - r, mk3(0.0f, 1.0f, 0.0f));
    const f3 c = normalize_or(p2 - r, mk3(0.0f, 0.0f, 1.0f));
    const float num = fabsf(dot(a, cross(b, c)));
    const float den = 1.0f + dot(a, b) + dot(b, c) + dot(c, a);
    return 2.0f * atan2_(num, den);
}
__device__ __forceinline__ bool use_solid_angle(f3 r, f3 p0, f3 p1, f3 p2) {
    const f3 e0 = p1 - p0, e1 = p2 - p0, e2 = p2 - p1;
    const float longest = maxf_(dot(e0, e0), maxf_(dot(e1, e1), dot(e2, e2)));
    const f3 un = cross(e0, e1);
    const float nl2 = dot(un, un);
    const float dist = dot(un, p0 - r) / maxf_(nl2, 1.0e-20f);
    return nl2 > 1.0e-20f && longest > dist * dist;
}
struct TriPdf {
    float value;
    bool valid;
};
// triangle_directional_pdf (include/psycles/luisa/spherical_geometry.h:161-203).
__device__ __forceinline__ TriPdf triangle_directional_pdf(f3 r, f3 lp, f3 p0, f3 p1, f3 p2) {
    const f3 e0 = p1 - p0, e1 = p2 - p0;
    const f3 un = cross(e0, e1);
    const float da = sqrtf(maxf_(dot(un, un), 0.0f));
    const float area = 0.5f * da;
    const f3 nrm = un / maxf_(da, 1.0e-20f);
    const f3 off = lp - r;
    const float d2 = dot(off, off);
    const f3 dir = off / sqrtf(maxf_(d2, 1.0e-20f));
    const float cosine = fabsf(dot(nrm, -dir));
    const bool sa = use_solid_angle(r, p0, p1, p2);
    const float solid = triangle_solid_angle(r, p0, p1, p2);
    const float area_pdf = d2 / maxf_(cosine * area, 1.0e-20f);
    const float sa_pdf = 1.0f / maxf_(solid, 1.0e-20f);
    const bool valid_area = area > 0.0f && d2 > 1.0e-12f && cosine > 0.0f;
    return {sa ? sa_pdf : area_pdf, sa ? (valid_area && solid > 0.0f) : valid_area};
}
struct TriSample {
    f3 position, direction;
    float distance, pdf;
    bool valid;
};
// sample_triangle (spherical_geometry.h:207-283).
__device__ __forceinline__ TriSample sample_triangle(f3 r, f3 p0, f3 p1, f3 p2, f2 rnd) {
    const float x = clampf_(rnd.x, 0.0f, 1.0f), y = clampf_(rnd.y, 0.0f, 1.0f);
    f2 ab;
    if (y > x) {
        ab.x = 0.5f * x;
        ab.y = y - ab.x;
    } else {
        ab.y = 0.5f * y;
        ab.x = x - ab.y;
    }
    const f3 area_position = p0 * (1.0f - ab.x - ab.y) + p1 * ab.x + p2 * ab.y;
    const f3 area_offset = area_position - r;
    const float area_d2 = dot(area_offset, area_offset);
    const float area_distance = sqrtf(maxf_(area_d2, 1.0e-20f));
    const f3 area_direction = area_offset / area_distance;
    TriSample out;
    const bool sa = use_solid_angle(r, p0, p1, p2);
    if (!sa) {
        const TriPdf pdf = triangle_directional_pdf(r, area_position, p0, p1, p2);
        out.position = area_position;
        out.direction = area_direction;
        out.distance = area_distance;
        out.pdf = pdf.value;
        out.valid = pdf.valid && area_d2 > 1.0e-12f;
        return out;
    }
    const f3 a = normalize_or(p0 - r, mk3(1.0f, 0.0f, 0.0f));
    const f3 b = normalize_or(p1 - r, mk3(0.0f, 1.0f, 0.0f));
    const f3 c = normalize_or(p2 - r, mk3(0.0f, 0.0f, 1.0f));
    const float cos_b = clampf_(dot(a, c), -1.0f, 1.0f);
    const float cos_c = clampf_(dot(a, b), -1.0f, 1.0f);
    const float solid = triangle_solid_angle(r, p0, p1, p2);
    const f3 ab_n = normalize_or(cross(a, b), mk3(1.0f, 0.0f, 0.0f));
    const f3 ac_n = normalize_or(cross(a, c), mk3(0.0f, 1.0f, 0.0f));
    const float cos_alpha = clampf_(dot(ab_n, ac_n), -1.0f, 1.0f);
    const float sin_alpha = sqrtf(maxf_(1.0f - cos_alpha * cos_alpha, 0.0f));
    const float alpha = acos_(cos_alpha);
    const float phi = x * solid - alpha;
    const float sin_phi = sin_(phi), cos_phi = cos_(phi);
    const float u = cos_phi - cos_alpha;
    const float v = sin_phi + sin_alpha * cos_c;
    const float num = (v * cos_phi - u * sin_phi) * cos_alpha - v;
    const float den = (v * sin_phi + u * cos_phi) * sin_alpha;
    const float safe_den = fabsf(den) > 1.0e-20f ? den : (den >= 0.0f ? 1.0e-20f : -1.0e-20f);
    const float q = fabsf(den) <= 1.0e-20f ? 1.0f : num / safe_den;
    const f3 tangent = normalize_or(c - a * cos_b, mk3(0.0f, 1.0f, 0.0f));
    const f3 c_prime = normalize_or(a * clampf_(q, -1.0f, 1.0f) + tangent * sqrtf(maxf_(1.0f - q * q, 0.0f)), a);
    const float z = 1.0f - y * (1.0f - dot(c_prime, b));
    const f3 edge_dir = normalize_or(c_prime - b * dot(c_prime, b), a);
    const f3 solid_dir = normalize_or(b * z + edge_dir * sqrtf(maxf_(1.0f - z * z, 0.0f)), b);
    const f3 e01 = p1 - p0, e02 = p2 - p0;
    const f3 pv = cross(solid_dir, e02);
    const float det = dot(e01, pv);
    const float safe_det = fabsf(det) > 1.0e-20f ? det : (det >= 0.0f ? 1.0e-20f : -1.0e-20f);
    const float inv_det = 1.0f / safe_det;
    const f3 tv = r - p0;
    const float su = dot(tv, pv) * inv_det;
    const f3 qv = cross(tv, e01);
    const float sv = dot(solid_dir, qv) * inv_det;
    const float sd = dot(e02, qv) * inv_det;
    const f3 solid_position = r + solid_dir * sd;
    const bool solid_valid = fabsf(det) > 1.0e-20f && sd > 0.0f && su >= -1.0e-5f && sv >= -1.0e-5f &&
                             su + sv <= 1.0f + 1.0e-5f && solid > 0.0f;
    const TriPdf pdf = triangle_directional_pdf(r, solid_position, p0, p1, p2);
    out.position = solid_position;
    out.direction = solid_dir;
    out.distance = sd;
    out.pdf = pdf.value;
    out.valid = pdf.valid && solid_valid;
    return out;
}

__device__ __forceinline__ bool samples_front(uint32_t m) { return m == 1u || m == 2u || m == 4u; }
__device__ __forceinline__ bool samples_back(uint32_t m) { return m == 1u || m == 3u || m == 4u; }
__device__ __forceinline__ bool sampled_side(uint32_t m, f3 ng, f3 dir) {
    return dot(ng, -dir) < 0.0f ? samples_back(m) : samples_front(m);
}

__device__ __forceinline__ float emissive_forward_pdf(float selection_pdf, uint32_t sampling, f3 reference, f3 lp,
                                                      f3 p0, f3 p1, f3 p2, f3 oriented_ng) {
    const TriPdf pdf = triangle_directional_pdf(reference, lp, p0, p1, p2);
    const f3 dir = normalize_or(lp - reference, mk3(0.0f, 0.0f, 1.0f));
    const bool side = sampled_side(sampling, oriented_ng, dir);
    const float area = 0.5f * length(cross(p1 - p0, p2 - p0));
    const float value = pdf.value * selection_pdf;
    return (sampling != 0u && side && pdf.valid && area > 0.0f && value > 0.0f) ? value : 0.0f;
}

struct AnalyticSample {
    bool valid;
    f3 direction, position;
    float distance, pdf, eval_factor;
};

// ---------------------------------------------------------- sphere lamps
// sin_squared_to_one_minus_cosine (include/psycles/luisa/cycles_sample_mapping.h).
__device__ __forceinline__ float sin2_to_one_minus_cos(float s2) {
    return s2 > 0.0004f ? 1.0f - sqrtf(maxf_(1.0f - s2, 0.0f)) : 0.5f * s2;
}

// spot_one_minus_cosine_larger_spread (analytic_light_sampling.h:355-376),
// a per-lamp constant.
__device__ __forceinline__ float spot_spread_cap(const LampConstGpu &c) { return c.spot_rz.w; }

struct SphereHit {
    bool valid;
    float distance;
    f3 position;
};

// intersect_sphere (analytic_light_sampling.h:192-239): open interval, the
// far side only from inside.
__device__ __forceinline__ SphereHit intersect_sphere(f3 o, f3 d, float tmin, float tmax, f3 c, float r) {
    const f3 co = c - o;
    const float r2 = r * r;
    const float cd2 = dot(co, co);
    const float pd = dot(co, d);
    const f3 perp = co - d * pd;
    const float pp2 = dot(perp, perp);
    const float dist = pd - copysignf(sqrtf(maxf_(r2 - pp2, 0.0f)), cd2 - r2);
    const bool valid = !(cd2 > r2 && pd < 0.0f) && pp2 <= r2 && dist > tmin && dist < tmax;
    return {valid, dist, o + d * dist};
}

// sample_uniform_sphere (cycles_sample_mapping.h:380-387).
__device__ __forceinline__ f3 sample_uniform_sphere(f2 u) {
    const float z = 1.0f - 2.0f * u.x;
    const float r = sqrtf(maxf_(1.0f - z * z, 0.0f));
    const float phi = 2.0f * kPi * u.y;
    return mk3(r * cos_(phi), r * sin_(phi), z);
}

// sample_sphere_geometry (analytic_light_sampling.h:430-548): a cone towards
// the sphere from outside (optionally around another axis, then intersected),
// the shading hemisphere or the whole sphere from inside.
__device__ __forceinline__ AnalyticSample sample_sphere(f3 reference, f3 n, bool transmission, f3 center, float r,
                                                        f3 outside_axis, float outside_omc, bool intersect_sampled,
                                                        f2 rnd) {
    AnalyticSample out;
    const float r2 = r * r;
    f3 ln = reference - center;
    const float cd2 = dot(ln, ln);
    const float cd = sqrtf(maxf_(cd2, 1.0e-30f));
    ln = ln / cd;
    const bool outside = cd2 > r2;
    f3 dir = mk3(0.0f);
    float cosine = 1.0f, pdf = 0.0f, dist = 0.0f;
    f3 pos = reference;
    bool known = false;
    bool valid = r > 0.0f && cd2 > 0.0f;
    if (outside) {
        const ConeSample c = sample_uniform_cone(outside_axis, outside_omc, rnd);
        dir = c.direction;
        cosine = c.cosine;
        pdf = c.pdf;
        if (intersect_sampled) {
            const SphereHit h = intersect_sphere(reference, dir, 0.0f, 1.0e30f, center, r);
            valid = valid && h.valid;
            dist = h.distance;
            pos = h.position;
            known = h.valid;
        }
    } else {
        if (transmission) {
            dir = sample_uniform_sphere(rnd);
            pdf = 0.5f * kInvTwoPi;
        } else {
            dir = sample_cosine_hemisphere(n, rnd, &pdf);
        }
        cosine = -dot(dir, ln);
    }
    if (!known) {
        dist = cd * cosine - copysignf(sqrtf(maxf_(r2 - cd2 + cd2 * cosine * cosine, 0.0f)), cd2 - r2);
        pos = reference + dir * dist;
    }
    const f3 normal = light_safe_normalize(pos - center, -dir);
    out.valid = valid;
    out.direction = dir;
    out.position = normal * r + center;
    out.distance = dist;
    out.pdf = pdf;
    out.eval_factor = 0.0f;
    return out;
}

// rectangle_solid_angle_context (include/psycles/luisa/analytic_light_sampling.h:
// Ureña et al. spherical rectangle seen from `reference`, with the planar pdf
// limit for tiny or grazing rectangles).
struct RectContext {
    f3 z;
    float z0, x0, x1, y0, y1;
    float e[4], g[4];
    float solid, pdf;
};

__device__ __forceinline__ RectContext rect_context(f3 reference, f3 center, f3 au, float lu, f3 av, float lv) {
    RectContext c;
    c.z = cross(au, av);
    const f3 co = center - reference;
    c.z0 = dot(co, c.z);
    if (c.z0 > 0.0f) {
        c.z = -c.z;
        c.z0 = -c.z0;
    }
    const float cu = dot(co, au), cv = dot(co, av);
    c.x0 = cu - 0.5f * lu;
    c.x1 = cu + 0.5f * lu;
    c.y0 = cv - 0.5f * lv;
    c.y1 = cv + 0.5f * lv;
    c.e[0] = -c.y0;
    c.e[1] = c.x1;
    c.e[2] = c.y1;
    c.e[3] = -c.x0;
#pragma unroll
    for (int k = 0; k < 4; ++k) c.e[k] = c.e[k] / sqrtf(c.e[k] * c.e[k] + c.z0 * c.z0);
#pragma unroll
    for (int k = 0; k < 4; ++k) c.g[k] = asin_(clampf_(-c.e[k] * c.e[(k + 1) & 3], -1.0f, 1.0f));
    c.solid = -(c.g[0] + c.g[1] + c.g[2] + c.g[3]);
    const float min_e2 =
        minf_(minf_(c.e[0] * c.e[0], c.e[1] * c.e[1]), minf_(c.e[2] * c.e[2], c.e[3] * c.e[3]));
    const float cd = length(co);
    const float pden = c.z0 * lu * lv;
    const float planar = pden != 0.0f ? -(cd * cd * cd) / pden : 0.0f;
    c.pdf = (c.solid < 1.0e-5f || min_e2 > 0.99999f) ? planar : 1.0f / c.solid;
    return c;
}

// point_eval_factor (analytic_light_sampling.h:880-896), a per-lamp constant.
__device__ __forceinline__ float point_eval_factor(const LampConstGpu &c) { return c.factors.x; }

// spot_light_to_local + spot_light_attenuation (analytic_light_sampling.h:309-345)
// for the direction `from_light` leaving the lamp; the inverse axes and the
// cone constants are the lamp's.
__device__ __forceinline__ float spot_attenuation(const LampConstGpu &c, f3 from_light) {
    const f3 rx = mk3(c.spot_rx.x, c.spot_rx.y, c.spot_rx.z);
    const f3 ry = mk3(c.spot_ry.x, c.spot_ry.y, c.spot_ry.z);
    const f3 rz = mk3(c.spot_rz.x, c.spot_rz.y, c.spot_rz.z);
    f3 local = light_safe_normalize(mk3(dot(rx, from_light), dot(ry, from_light), dot(rz, from_light)),
                                    mk3(0.0f, 0.0f, -1.0f));
    local.z = -local.z;
    const float cos_half = c.spot_rx.w;
    const float blend = c.spot_ry.w;
    const float ratio = blend != 0.0f ? (local.z - cos_half) / blend : 0.0f;
    const float lin = clampf_(ratio, 0.0f, 1.0f);
    const float smooth = lin * lin * (3.0f - 2.0f * lin);
    const float hard = local.z >= cos_half ? 1.0f : 0.0f;
    return blend > 0.0f ? smooth : hard;
}

// include/psycles/luisa/analytic_light_sampling.h:84-108 (distant),
// :549-603 (disk), :856-896 (pdf / eval factor), :309-345 (spot profile).
__device__ __noinline__ AnalyticSample sample_analytic(const psy_light_desc &l, const LampConstGpu &lc, f3 reference,
                                                       f3 shading_n, bool transmission, f2 rnd) {
    AnalyticSample out;
    const bool normalize_power = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    if (l.type == PSY_LIGHT_DISTANT) {
        const f3 az = ld3(l.axis_z);
        const ConeSample c = sample_uniform_cone(-az, lc.factors.y, rnd);
        out.eval_factor = lc.factors.z;
        out.direction = -c.direction;
        out.position = c.direction;
        out.distance = 1.0e30f;
        out.pdf = c.pdf;
        out.valid = true;
        return out;
    }
    if (l.type == PSY_LIGHT_AREA) {
        // AreaLightSampling::from_position, full spread
        // (src/luisa/area_light_sampling.cpp:494-642; analytic_light_sampling.h:605-793)
        out.valid = false;
        out.eval_factor = 0.0f;
        const f3 center = ld3(l.position), au = ld3(l.axis_x), av = ld3(l.axis_y), az = ld3(l.axis_z);
        const float lu = l.size_u, lv = l.size_v;
        const bool ellipse = (l.flags & PSY_LIGHT_FLAG_ELLIPSE) != 0u;
        const f3 normal = -az;
        out.position = center;
        out.direction = mk3(0.0f);
        out.distance = 0.0f;
        out.pdf = 0.0f;
        if (!(dot(center - reference, normal) <= 0.0f)) return out;
        f3 position;
        float pdf;
        if (!ellipse) {
            const RectContext c = rect_context(reference, center, au, lu, av, lv);
            const f3 z = c.z;
            const float z0 = c.z0, x0 = c.x0, x1 = c.x1, y0 = c.y0, y1 = c.y1;
            pdf = c.pdf;
            const float solid = c.solid;
            const float b0 = c.e[0], b1 = c.e[2];
            const float alpha = rnd.x * solid + c.g[2] + c.g[3];
            const float sa = sin_(alpha);
            const float fu = sa != 0.0f ? (cos_(alpha) * b0 + b1) / sa : 0.0f;
            float cos_u = copysignf(1.0f / sqrtf(fu * fu + b0 * b0), fu);
            cos_u = clampf_(cos_u, -1.0f, 1.0f);
            float su = -(cos_u * z0) / maxf_(sqrtf(maxf_(1.0f - cos_u * cos_u, 0.0f)), 1.0e-7f);
            su = clampf_(su, x0, x1);
            const float du2 = su * su + z0 * z0;
            const float h0 = y0 / sqrtf(du2 + y0 * y0);
            const float h1 = y1 / sqrtf(du2 + y1 * y1);
            const float hv = h0 + rnd.y * (h1 - h0);
            const float hv2 = hv * hv;
            const float sv = hv2 < 1.0f - 1.0e-6f ? hv * sqrtf(du2 / (1.0f - hv2)) : y1;
            position = reference + au * su + av * sv + z * z0;
        } else {
            const f2 disk = sample_uniform_disk(rnd);
            position = center + au * (0.5f * lu * disk.x) + av * (0.5f * lv * disk.y);
            pdf = 4.0f * kInvPi / (lu * lv);
        }
        const f3 off = position - reference;
        const float d2 = dot(off, off);
        const float dist = sqrtf(maxf_(d2, 0.0f));
        const f3 dir = off / maxf_(dist, 1.0e-30f);
        if (ellipse) {
            const float cosine = dot(normal, -dir);
            pdf *= cosine > 0.0f ? d2 / cosine : 0.0f;
        }
        float area = lu * lv;
        if (ellipse) area *= 0.25f * kPi;
        const float inv_area = (normalize_power && area != 0.0f) ? 1.0f / area : 1.0f;
        const float factor = kInvPi * inv_area * 1.0f;
        const f3 inplane = position - center;
        const float u = dot(inplane, au), v = dot(inplane, av);
        const float eu = (0.5f + 1.0e-7f) * lu + 1.0e-6f, ev = (0.5f + 1.0e-7f) * lv + 1.0e-6f;
        const bool inside = ellipse ? (u * u / (eu * eu) + v * v / (ev * ev) <= 1.0f)
                                    : (fabsf(u) <= eu && fabsf(v) <= ev);
        out.valid = inside && factor > 0.0f;
        out.direction = dir;
        out.position = position;
        out.distance = dist;
        out.pdf = pdf;
        out.eval_factor = factor;
        return out;
    }
    if ((l.flags & PSY_LIGHT_FLAG_SPHERE) != 0u && l.radius > 0.0f) {
        // sample_point_light / sample_spot_light, sphere geometry
        // (analytic_light_sampling.h:898-1105)
        const f3 center = ld3(l.position);
        const f3 off = reference - center;
        const float cd2 = dot(off, off);
        const float r2 = l.radius * l.radius;
        const f3 ln = light_safe_normalize(off, mk3(0.0f, 0.0f, -1.0f));
        const float sphere_cap = sin2_to_one_minus_cos(r2 / maxf_(cd2, 1.0e-30f));
        f3 axis = -ln;
        float cap = sphere_cap;
        bool spread = false;
        if (l.type == PSY_LIGHT_SPOT) {
            const float spot_cap = spot_spread_cap(lc);
            spread = cd2 > r2 && !(sphere_cap < spot_cap);
            if (spread) {
                axis = ld3(l.axis_z);
                cap = spot_cap;
            }
        }
        out = sample_sphere(reference, shading_n, transmission, center, l.radius, axis, cap, spread, rnd);
        float eval = point_eval_factor(lc);
        if (l.type == PSY_LIGHT_SPOT && cd2 > r2) eval *= spot_attenuation(lc, -out.direction);
        out.eval_factor = eval;
        if (l.type == PSY_LIGHT_SPOT) out.valid = out.valid && eval != 0.0f;
        return out;
    }
    const f3 center = ld3(l.position);
    f3 ln = reference - center;
    const float cd2 = dot(ln, ln);
    const float cd = sqrtf(maxf_(cd2, 1.0e-30f));
    ln = ln / cd;
    const Basis b = make_orthonormals(ln);
    const f2 disk = sample_uniform_disk(rnd);
    const f3 position = center + (b.tangent * disk.x + b.bitangent * disk.y) * l.radius;
    const f3 off = position - reference;
    const float d2 = dot(off, off);
    const float dist = sqrtf(maxf_(d2, 1.0e-30f));
    const f3 dir = off / dist;
    const float cosine = dot(ln, -dir);
    const float r2 = l.radius * l.radius;
    const float inv_area = r2 > 0.0f ? 1.0f / maxf_(r2 * kPi, 1.0e-20f) : 1.0f;
    out.pdf = cosine > 0.0f ? inv_area * d2 / cosine : 0.0f;
    float eval = point_eval_factor(lc);
    if (l.type == PSY_LIGHT_SPOT) eval *= spot_attenuation(lc, -dir);
    out.eval_factor = eval;
    out.direction = dir;
    out.position = position;
    out.distance = dist;
    out.valid = cd2 > 0.0f && cosine > 0.0f && eval != 0.0f;
    return out;
}


// ------------------------------------------------- forward lamp events

// A lamp in front of the committed mesh event: ClosestEventStageImpl's lamp
// loop (src/luisa/path_kernel_closest_event.cpp:56-230) over the
// intersections of include/psycles/luisa/analytic_light_intersection.h.
struct LampHit {
    bool valid;
    uint32_t index;
    float distance, pdf, eval_factor;
};

// intersect_area (analytic_light_intersection.h:268-353) at full spread:
// strictly inside (tmin, tmax), front side only; the directional pdf of
// AreaLightSampling::from_intersection (src/luisa/area_light_sampling.cpp:644-727).
__device__ __forceinline__ bool intersect_area_lamp(const psy_light_desc &l, f3 o, f3 d, float tmin, float tmax,
                                                    float &distance, float &pdf, float &eval) {
    const f3 center = ld3(l.position), au = ld3(l.axis_x), av = ld3(l.axis_y);
    const f3 normal = -ld3(l.axis_z);
    const float lu = l.size_u, lv = l.size_v;
    const bool ellipse = (l.flags & PSY_LIGHT_FLAG_ELLIPSE) != 0u;
    const float dn = dot(d, normal);
    const float num = dot(center - o, normal);
    distance = dn != 0.0f ? num / dn : 0.0f;
    const f3 inplane = (o + d * distance) - center;
    const float u = lu != 0.0f ? dot(inplane, au) / lu : 0.0f;
    const float v = lv != 0.0f ? dot(inplane, av) / lv : 0.0f;
    const bool inside = u >= -0.5f && u <= 0.5f && v >= -0.5f && v <= 0.5f && (!ellipse || u * u + v * v <= 0.25f);
    if (!(dn < 0.0f && distance > tmin && distance < tmax && inside)) return false;
    if (!ellipse) {
        pdf = rect_context(o, center, au, lu, av, lv).pdf;
    } else {
        const float cosine = dot(normal, -d);
        pdf = 4.0f * kInvPi / (lu * lv) * (cosine > 0.0f ? (distance * distance) / cosine : 0.0f);
    }
    float area = lu * lv;
    if (ellipse) area *= 0.25f * kPi;
    const float inv_area = ((l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u && area != 0.0f) ? 1.0f / area : 1.0f;
    eval = kInvPi * inv_area * 1.0f;
    return area > 0.0f && eval > 0.0f;
}

// intersect_point / intersect_spot (analytic_light_intersection.h:33-266)
// for the oriented-disk geometry (radius > 0, not a sphere): the disk faces
// the ray origin.
__device__ __forceinline__ bool intersect_disk_lamp(const psy_light_desc &l, const LampConstGpu &lc, f3 o, f3 d,
                                                    float tmin, float tmax, f3 mis_n, bool had_transmission,
                                                    float &distance, float &pdf, float &eval) {
    const f3 center = ld3(l.position);
    const f3 offset = o - center;
    if ((l.flags & PSY_LIGHT_FLAG_SPHERE) != 0u) {
        // intersect_point / intersect_spot, sphere geometry, with
        // sphere_light_pdf (analytic_light_intersection.h:33-266,
        // analytic_light_sampling.h:282-307)
        if (!(l.radius > 0.0f)) return false;
        const float cd2 = dot(offset, offset);
        const float r2 = l.radius * l.radius;
        float cap = sin2_to_one_minus_cos(r2 / maxf_(cd2, 1.0e-30f));
        if (l.type == PSY_LIGHT_SPOT) cap = minf_(cap, spot_spread_cap(lc));
        const SphereHit h = intersect_sphere(o, d, tmin, tmax, center, l.radius);
        if (!h.valid) return false;
        distance = h.distance;
        if (cd2 > r2) {
            pdf = kInvTwoPi / maxf_(cap, 1.0e-30f);
        } else if (had_transmission) {
            pdf = 0.5f * kInvTwoPi;
        } else {
            const float c = dot(mis_n, d);
            pdf = c > 0.0f ? c * kInvPi : 0.0f;
        }
        eval = point_eval_factor(lc);
        if (l.type == PSY_LIGHT_SPOT) {
            if (cd2 > r2) eval *= spot_attenuation(lc, -d);
            if (!(dot(d, offset) < 0.0f)) return false;
        }
        return eval > 0.0f;
    }
    const f3 ln = light_safe_normalize(offset, -d);
    const float plane = dot(offset, ln);
    const float cosine = dot(ln, -d);
    distance = cosine != 0.0f ? plane / cosine : 0.0f;
    const f3 radial = (o + d * distance) - center;
    const float r2 = l.radius * l.radius;
    const bool hit = plane * cosine > 0.0f && distance >= 0.0f && dot(radial, radial) < r2 && distance > tmin &&
                     distance < tmax;
    if (!(hit && l.radius > 0.0f)) return false;
    const float inv_area = r2 > 0.0f ? 1.0f / maxf_(r2 * kPi, 1.0e-20f) : 1.0f;
    pdf = cosine > 0.0f ? inv_area * (distance * distance) / cosine : 0.0f;
    eval = point_eval_factor(lc);
    if (l.type == PSY_LIGHT_SPOT) {
        eval *= spot_attenuation(lc, -d);
        if (!(dot(d, offset) < 0.0f)) return false;
    }
    return eval > 0.0f;
}

// Nearest eligible lamp strictly inside (tmin, event_distance); ties keep the
// lower index.  Eligibility: the lamp's visibility covers the ray, the ray
// is a camera ray or the lamp takes part in MIS, and it is not the lamp the
// previous event hit.
__device__ __noinline__ LampHit closest_lamp(const SceneView &s, f3 o, f3 d, float tmin, float event_distance,
                                             uint32_t ray_visibility, uint32_t excluded, f3 mis_n,
                                             bool had_transmission) {
    LampHit best{false, kInvalid, event_distance, 0.0f, 0.0f};
    const bool camera_path = (ray_visibility & PSY_VISIBILITY_CAMERA) != 0u;
    for (uint32_t k = 0; k < s.lamp_count; ++k) {
        // Bounding-sphere rejection with a margin well above the float
        // error of the test, so no lamp the exact test accepts is skipped.
        const float4 bound = s.lamp_bounds[k];
        const f3 oc = mk3(bound.x, bound.y, bound.z) - o;
        const float tca = dot(oc, d);
        const float oc2 = dot(oc, oc);
        const float miss2 = oc2 - tca * tca;
        if (miss2 > bound.w * 1.0625f + oc2 * 1.0e-5f) continue;
        if (tca < 0.0f && oc2 > bound.w * 1.0625f + 1.0e-6f) continue;
        const uint32_t li = s.lamp_ids[k];
        const psy_light_desc &l = s.lights[li];
        const bool use_mis = (l.flags & kLightFlagUseMis) != 0u;
        if (!((l.visibility & ray_visibility) != 0u && (camera_path || use_mis) && li != excluded)) continue;
        float distance = 0.0f, pdf = 0.0f, eval = 0.0f;
        const bool hit = l.type == PSY_LIGHT_AREA ? intersect_area_lamp(l, o, d, tmin, best.distance, distance, pdf, eval)
                                                  : intersect_disk_lamp(l, s.lamp_consts[li], o, d, tmin, best.distance, mis_n,
                                                                        had_transmission, distance, pdf, eval);
        if (hit) best = LampHit{true, li, distance, pdf, eval};
    }
    return best;
}

}  // namespace psy
