// TEST INFRASTRUCTURE ONLY -- CPU oracle (see oracle_math.h).
//
// Host tables and the per-sample Sobol lookup of the reference:
//   * tabulated-Sobol LUT      src/sampling/tabulated_sobol.cpp:40-200
//   * pixel-filter inverse CDF src/sampling/pixel_filter.cpp:30-85
//   * device Sobol lookup      include/psycles/luisa/cycles_sampler.h:36-339
//   * sample mappings          include/psycles/luisa/cycles_sample_mapping.h:49-118
// The 4-D xor table and the direction constants are the published Cycles
// constants (Blender intern/cycles, Apache-2.0) that the reference also
// carries; they are data of the algorithm, not code.
#pragma once

#include "oracle_math.h"

#include <algorithm>
#include <array>
#include <vector>

namespace oracle {

// Cycles' xor table that picks the previously placed point of each
// stratum (tabulated_sobol.cpp:23-73), one row per component.
inline const uint32_t kSobolXors[4][32] = {
    {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u,
     0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u},
    {0x00000000u, 0x00000001u, 0x00000001u, 0x00000007u, 0x00000001u, 0x00000013u, 0x00000015u, 0x0000007fu,
     0x00000001u, 0x00000103u, 0x00000105u, 0x0000070fu, 0x00000111u, 0x00001333u, 0x00001555u, 0x00007fffu,
     0x00000001u, 0x00010003u, 0x00010005u, 0x0007000fu, 0x00010011u, 0x00130033u, 0x00150055u, 0x007f00ffu,
     0x00010101u, 0x01030303u, 0x01050505u, 0x070f0f0fu, 0x01111111u, 0x13333333u, 0x15555555u, 0x7fffffffu},
    {0x00000000u, 0x00000001u, 0x00000003u, 0x00000001u, 0x00000005u, 0x0000001fu, 0x0000002bu, 0x0000003du,
     0x00000011u, 0x00000133u, 0x00000377u, 0x00000199u, 0x00000445u, 0x00001ccfu, 0x00002ddbu, 0x0000366du,
     0x00000101u, 0x00010303u, 0x00030707u, 0x00010909u, 0x00051515u, 0x001f3f3fu, 0x002b6b6bu, 0x003dbdbdu,
     0x00101011u, 0x01303033u, 0x03707077u, 0x01909099u, 0x04515145u, 0x1cf3f3cfu, 0x2db6b6dbu, 0x36dbdb6du},
    {0x00000000u, 0x00000001u, 0x00000000u, 0x00000003u, 0x0000000du, 0x0000000cu, 0x00000005u, 0x0000004fu,
     0x00000014u, 0x000000e7u, 0x00000329u, 0x0000039cu, 0x00000011u, 0x00001033u, 0x00000044u, 0x000030bbu,
     0x0000d1cdu, 0x0000c2ecu, 0x00005415u, 0x0004fc3fu, 0x00015054u, 0x000e5c97u, 0x0032e5b9u, 0x0039725cu,
     0x00000101u, 0x01000303u, 0x00000404u, 0x03000b0bu, 0x0d001d1du, 0x0c002c2cu, 0x05004545u, 0x4f00cfcfu},
};

// Hash Prospector (tabulated_sobol.cpp:75-90, cycles_sampler.h:91-104).
inline uint32_t hash_hp_uint(uint32_t v) {
    v ^= v >> 16u;
    v *= 0x21f0aaadu;
    v ^= v >> 15u;
    v *= 0xd35a2d97u;
    v ^= v >> 15u;
    return v ^ 0xe6fe3bebu;
}
inline uint32_t hash_hp_seeded_uint(uint32_t v, uint32_t seed) {
    seed ^= seed << 19u;
    return hash_hp_uint(v ^ seed);
}
inline float hash_hp_float(uint32_t v) {
    return static_cast<float>(hash_hp_uint(v)) * (1.0f / 4294967808.0f);
}

// generate_sequence (tabulated_sobol.cpp:97-148): progressive
// multi-jittered 4-D points, one pattern per seed.
inline void generate_sequence(float4 *points, uint32_t size, uint32_t rng_seed) {
    uint32_t rng_index = hash_hp_seeded_uint(rng_seed, 0x44605a73u);
    points[0].x = hash_hp_float(rng_index++);
    points[0].y = hash_hp_float(rng_index++);
    points[0].z = hash_hp_float(rng_index++);
    points[0].w = hash_hp_float(rng_index++);
    uint32_t log_n = 0u;
    for (uint32_t n = 1u; n < size; ++log_n, n *= 2u) {
        const float strata = static_cast<float>(n * 2u);
        for (uint32_t i = 0u; i < n && n + i < size; ++i) {
            const uint32_t ox = static_cast<uint32_t>(points[i ^ kSobolXors[0][log_n]].x * strata);
            const uint32_t oy = static_cast<uint32_t>(points[i ^ kSobolXors[1][log_n]].y * strata);
            const uint32_t oz = static_cast<uint32_t>(points[i ^ kSobolXors[2][log_n]].z * strata);
            const uint32_t ow = static_cast<uint32_t>(points[i ^ kSobolXors[3][log_n]].w * strata);
            float4 &p = points[n + i];
            p.x = (static_cast<float>(ox ^ 1u) + hash_hp_float(rng_index++)) / strata;
            p.y = (static_cast<float>(oy ^ 1u) + hash_hp_float(rng_index++)) / strata;
            p.z = (static_cast<float>(oz ^ 1u) + hash_hp_float(rng_index++)) / strata;
            p.w = (static_cast<float>(ow ^ 1u) + hash_hp_float(rng_index++)) / strata;
        }
    }
}

inline bool sobol_valid_size(uint32_t s) {
    return s >= 256u && s <= 8192u && (s & (s - 1u)) == 0u;
}

// sequence_size_for_samples (tabulated_sobol.cpp:156-173).
inline uint32_t sobol_sequence_size_for_samples(uint32_t samples) {
    const uint32_t c = std::clamp(samples, 1u, 8192u);
    uint32_t unbounded = 1u;
    if (c != 1u) {
        unbounded = 1u << (32u - static_cast<uint32_t>(__builtin_clz(c - 1u)));
    }
    return std::clamp(unbounded, 256u, 8192u);
}

// generate_table (tabulated_sobol.cpp:175-200): 256 patterns.
inline std::vector<float4> sobol_generate_table(uint32_t size) {
    std::vector<float4> table(static_cast<size_t>(size) * 256u);
    for (uint32_t pattern = 0u; pattern < 256u; ++pattern) {
        generate_sequence(table.data() + static_cast<size_t>(pattern) * size, size, pattern);
    }
    return table;
}

// FNV-1a over the IEEE-754 bits of every component, the fingerprint that
// tests/test_tabulated_sobol.cpp:93-100 checks.
inline uint64_t sobol_table_fingerprint(const std::vector<float4> &table) {
    uint64_t h = 14695981039346656037ull;
    auto mix = [&](float v) {
        uint32_t b = float_bits(v);
        for (int i = 0; i < 4; ++i) {
            h ^= (b >> (8 * i)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    for (const auto &s : table) {
        mix(s.x); mix(s.y); mix(s.z); mix(s.w);
    }
    return h;
}

// ---------------------------------------------------------------- sampler

inline uint32_t reverse_bits(uint32_t v) {
    v = ((v >> 1u) & 0x55555555u) | ((v & 0x55555555u) << 1u);
    v = ((v >> 2u) & 0x33333333u) | ((v & 0x33333333u) << 2u);
    v = ((v >> 4u) & 0x0f0f0f0fu) | ((v & 0x0f0f0f0fu) << 4u);
    v = ((v >> 8u) & 0x00ff00ffu) | ((v & 0x00ff00ffu) << 8u);
    return (v >> 16u) | (v << 16u);
}

// cycles_sampler.h:52-68.
inline uint32_t reversed_bit_owen(uint32_t v, uint32_t seed) {
    v ^= v * 0x3d20adeau;
    v += seed;
    v *= (seed >> 16u) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return v;
}
inline uint32_t nested_uniform_scramble(uint32_t v, uint32_t seed) {
    return reverse_bits(reversed_bit_owen(reverse_bits(v), seed));
}

// cycles_sampler.h:70-79.
inline uint32_t hash_wang_seeded_uint(uint32_t v, uint32_t seed) {
    v = (v ^ 61u) ^ seed;
    v += v << 3u;
    v ^= v >> 4u;
    v *= 0x27d4eb2du;
    return v;
}

// cycles_sampler.h:184-210 (256 patterns: the rejection loop runs once).
inline uint32_t shuffled_pattern_index(uint32_t dimension, uint32_t seed) {
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

// cycles_sampler.h:212-219.
inline uint32_t pixel_hash(uint32_t x, uint32_t y, uint32_t seed) {
    const uint32_t qx = 1103515245u * ((x >> 1u) ^ y);
    const uint32_t qy = 1103515245u * ((y >> 1u) ^ x);
    const uint32_t h = 1103515245u * (qx ^ (qy >> 3u));
    return h ^ seed;
}

// cycles_sampler.h:241-258.
inline uint32_t shuffled_sample_index(uint32_t sample, uint32_t dimension, uint32_t seed,
                                      uint32_t sequence_size) {
    const uint32_t pattern = shuffled_pattern_index(dimension, seed);
    const uint32_t mask = sequence_size - 1u;
    const uint32_t shuffled = nested_uniform_scramble(sample, hash_wang_seeded_uint(dimension, seed));
    sample = (sample & ~mask) | (shuffled & mask);
    return ((pattern * sequence_size) + sample) % (sequence_size * 256u);
}

struct SobolTable {
    std::vector<float4> rows;
    uint32_t sequence_size{256u};
    float4 sample_4d(uint32_t sample, uint32_t rng_hash, uint32_t dimension) const {
        return rows[shuffled_sample_index(sample, dimension, rng_hash, sequence_size)];
    }
};

// Sobol dimension constants (include/psycles/sampling/tabulated_sobol.h:15-44).
constexpr uint32_t kDimFilter = 0u;
constexpr uint32_t kDimLensTime = 1u;
constexpr uint32_t kDimTerminate = 0u;
constexpr uint32_t kDimLight = 1u;
constexpr uint32_t kDimLightTerminate = 2u;
constexpr uint32_t kDimBsdf = 3u;
constexpr uint32_t kBounceDimensions = 16u;

// ----------------------------------------------------------- pixel filter

// make_pixel_filter_table (src/sampling/pixel_filter.cpp:30-85).
inline std::array<float, 1024> pixel_filter_table(uint32_t filter, float width) {
    width = std::max(width, 1.0e-5f);
    auto box = [](float, float) { return 1.0f; };
    auto gaussian = [](float v, float w) {
        v *= 6.0f / w;
        return std::exp(-2.0f * v * v);
    };
    auto blackman_harris = [](float v, float w) {
        constexpr float two_pi = 6.28318530717958647692f;
        v = two_pi * (v / w + 0.5f);
        return 0.35875f - 0.48829f * std::cos(v) + 0.14128f * std::cos(2.0f * v) -
               0.01168f * std::cos(3.0f * v);
    };
    float (*function)(float, float) = box;
    if (filter == 1u) {
        function = gaussian;
        width *= 3.0f;
    } else if (filter == 2u) {
        function = blackman_harris;
        width *= 2.0f;
    }
    constexpr size_t size = 1024u;
    constexpr size_t resolution = size - 1u;
    std::array<float, size> cdf{};
    const float range = width * 0.5f;
    for (size_t i = 0u; i < resolution; ++i) {
        const float value = range * static_cast<float>(i) / static_cast<float>(resolution - 1u);
        cdf[i + 1u] = cdf[i] + std::fabs(function(value, width));
    }
    const float normalization = cdf[resolution] == 0.0f ? 0.0f : 1.0f / cdf[resolution];
    for (auto &v : cdf) v *= normalization;
    cdf[resolution] = 1.0f;
    std::array<float, size> inverse{};
    constexpr size_t half = (size - 1u) / 2u;
    for (size_t i = 0u; i <= half; ++i) {
        const float x = static_cast<float>(i) / static_cast<float>(half);
        auto it = std::upper_bound(cdf.begin(), cdf.end(), x);
        size_t index = static_cast<size_t>(it - cdf.begin());
        float t = 0.0f;
        if (index < resolution) {
            t = (x - cdf[index]) / (cdf[index + 1u] - cdf[index]);
        } else {
            index = resolution;
        }
        const float y = (static_cast<float>(index) + t) / static_cast<float>(size - 1u) * (2.0f * range);
        inverse[half + i] = 0.5f * (1.0f + y);
        inverse[half - i] = 0.5f * (1.0f - y);
    }
    return inverse;
}

// pixel_filter::sample (include/psycles/luisa/pixel_filter.h:17-29).
inline float pixel_filter_sample(const std::array<float, 1024> &table, float random) {
    const uint32_t last = 1023u;
    const float coordinate = clampf(random, 0.0f, 1.0f) * static_cast<float>(last);
    const uint32_t index = std::min(static_cast<uint32_t>(coordinate), last);
    const uint32_t next = std::min(index + 1u, last);
    const float t = coordinate - static_cast<float>(index);
    return lerp(table[index], table[next], t);
}

// ---------------------------------------------------------- sample maps

// cycles_sample_mapping::sample_uniform_disk (cycles_sample_mapping.h:49-63).
inline float2 sample_uniform_disk(float2 r) {
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
    float3 tangent, bitangent;
};

// make_orthonormals (cycles_sample_mapping.h:70-81).
inline Basis make_orthonormals(float3 n) {
    const float3 general = f3(n.z - n.y, n.x - n.z, n.y - n.x);
    const float3 equal = f3(n.z - n.y, n.x + n.z, -n.y - n.x);
    const bool use_general = (n.x != n.y) || (n.x != n.z);
    const float3 t = normalize(use_general ? general : equal);
    return {t, cross(n, t)};
}

struct HemisphereSample {
    float3 direction;
    float pdf;
};

// sample_cosine_hemisphere (cycles_sample_mapping.h:111-121).
inline HemisphereSample sample_cosine_hemisphere(float3 n, float2 r) {
    const float2 d = sample_uniform_disk(r);
    const float c = std::sqrt(maxf(1.0f - dot(d, d), 0.0f));
    const Basis b = make_orthonormals(n);
    return {b.tangent * d.x + b.bitangent * d.y + n * c, c * kInvPi};
}

// sample_ggx_visible_normal (cycles_sample_mapping.h:131-183): Heitz 2018,
// "Sampling the GGX Distribution of Visible Normals", in the frame of
// make_orthonormals(normal) with the concentric disk map; the half vector
// is not renormalised in world space.
inline float3 sample_ggx_visible_normal(float3 normal, float3 incoming, float alpha, float2 random) {
    const Basis w = make_orthonormals(normal);
    const float3 li = f3(dot(w.tangent, incoming), dot(w.bitangent, incoming), dot(normal, incoming));
    const float3 si = normalize(f3(alpha * li.x, alpha * li.y, li.z));
    const float pl2 = si.x * si.x + si.y * si.y;
    const float3 pt = f3(-si.y, si.x, 0.0f) / std::sqrt(maxf(pl2, 1.0e-20f));
    const float3 bx = pl2 > 1.0e-7f ? pt : f3(1.0f, 0.0f, 0.0f);
    const float3 by = cross(si, bx);
    float2 disk = sample_uniform_disk(random);
    const float projected_area = 0.5f * (1.0f + si.z);
    disk.y = lerp(std::sqrt(maxf(1.0f - disk.x * disk.x, 0.0f)), disk.y, projected_area);
    const float hz = std::sqrt(maxf(1.0f - disk.x * disk.x - disk.y * disk.y, 0.0f));
    const float3 sh = bx * disk.x + by * disk.y + si * hz;
    const float3 lh = normalize(f3(alpha * sh.x, alpha * sh.y, maxf(sh.z, 0.0f)));
    return w.tangent * lh.x + w.bitangent * lh.y + normal * lh.z;
}

// erf of Abramowitz & Stegun 7.1.28 (1 - 1 / (1 + a1 x + ... + a6 x^6)^16,
// |error| <= 3e-7) as Cycles evaluates it (cycles_sample_mapping.h:188-208):
// Horner steps as fused multiply-adds, +-1 beyond |x| = 12.3.
inline float fast_erf(float value) {
    const float magnitude = std::fabs(value);
    const float crushed = 1.0f - (1.0f - magnitude);
    float p = std::fmaf(0.0000430638f, crushed, 0.0002765672f);
    p = std::fmaf(p, crushed, 0.0001520143f);
    p = std::fmaf(p, crushed, 0.0092705272f);
    p = std::fmaf(p, crushed, 0.0422820123f);
    p = std::fmaf(p, crushed, 0.0705230784f);
    p = std::fmaf(p, crushed, 1.0f);
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
inline float fast_inverse_erf(float value) {
    const float magnitude = minf(std::fabs(value), 0.99999994f);
    const float base = -log_((1.0f - magnitude) * (1.0f + magnitude));
    const float cx = base - 2.5f;
    float central = std::fmaf(2.81022636e-08f, cx, 3.43273939e-07f);
    central = std::fmaf(central, cx, -3.5233877e-06f);
    central = std::fmaf(central, cx, -4.39150654e-06f);
    central = std::fmaf(central, cx, 0.00021858087f);
    central = std::fmaf(central, cx, -0.00125372503f);
    central = std::fmaf(central, cx, -0.00417768164f);
    central = std::fmaf(central, cx, 0.246640727f);
    central = std::fmaf(central, cx, 1.50140941f);
    const float tx = std::sqrt(base) - 3.0f;
    float tail = std::fmaf(-0.000200214257f, tx, 0.000100950558f);
    tail = std::fmaf(tail, tx, 0.00134934322f);
    tail = std::fmaf(tail, tx, -0.00367342844f);
    tail = std::fmaf(tail, tx, 0.00573950773f);
    tail = std::fmaf(tail, tx, -0.0076224613f);
    tail = std::fmaf(tail, tx, 0.00943887047f);
    tail = std::fmaf(tail, tx, 1.00167406f);
    tail = std::fmaf(tail, tx, 2.83297682f);
    return (base < 5.0f ? central : tail) * value;
}

// sample_beckmann_visible_normal (cycles_sample_mapping.h:239-310): the
// visible-slope sampler of Heitz and d'Eon (2014) with Cycles' root solve
// -- a quadratic first guess, at most three Newton steps kept inside the
// bracket (bisection otherwise) -- in the frame of make_orthonormals(normal).
inline float3 sample_beckmann_visible_normal(float3 normal, float3 incoming, float alpha, float2 random) {
    const Basis w = make_orthonormals(normal);
    const float3 li = f3(dot(w.tangent, incoming), dot(w.bitangent, incoming), dot(normal, incoming));
    const float3 si = normalize(f3(alpha * li.x, alpha * li.y, li.z));
    const float normal_radius = std::sqrt(-log_(random.x));
    const float normal_phi = 2.0f * kPi * random.y;
    const float2 normal_slope = f2(normal_radius * cos_(normal_phi), normal_radius * sin_(normal_phi));
    const float cosine = si.z;
    const float sine = std::sqrt(maxf(1.0f - cosine * cosine, 0.0f));
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
    const float quadratic_b = (0.5f - std::sqrt(maxf(k * (k - approximate_y + 1.0f) + 0.25f, 0.0f))) / safe_k;
    const float b = k > 0.0f ? quadratic_b : approximate_y - 1.0f;
    float inverse_erf = fast_inverse_erf(b);
    float2 begin = f2(-1.0f, -exact_y);
    float2 end = f2(erf_a, 1.0f + erf_a + k * exponential - exact_y);
    float2 current = f2(b, 1.0f + b + k * exp_(-inverse_erf * inverse_erf) - exact_y);
    for (uint32_t iteration = 0; std::fabs(current.y) > 1.0e-6f && iteration < 3u; ++iteration) {
        const bool same_sign = (begin.y < 0.0f) == (current.y < 0.0f);
        if (same_sign) begin = current;
        else end.x = current.x;
        const float newton = current.x - current.y / (1.0f - inverse_erf * tangent);
        const bool inside = newton >= begin.x && newton <= end.x;
        current.x = inside ? newton : 0.5f * (begin.x + end.x);
        inverse_erf = fast_inverse_erf(current.x);
        current.y = 1.0f + current.x + k * exp_(-inverse_erf * inverse_erf) - exact_y;
    }
    const float2 general_slope = f2(inverse_erf, fast_inverse_erf(2.0f * random.y - 1.0f));
    const float2 slope = si.z >= 0.99999f ? normal_slope : general_slope;
    const float2 rotated = f2(cosine_phi * slope.x - sine_phi * slope.y, sine_phi * slope.x + cosine_phi * slope.y) *
                           alpha;
    const float3 lh = normalize(f3(-rotated.x, -rotated.y, 1.0f));
    return w.tangent * lh.x + w.bitangent * lh.y + normal * lh.z;
}

// sin_squared_to_one_minus_cosine (cycles_sample_mapping.h:302-309).
inline float sin_squared_to_one_minus_cosine(float s2) {
    return s2 > 0.0004f ? 1.0f - std::sqrt(maxf(1.0f - s2, 0.0f)) : 0.5f * s2;
}

struct ConeSample {
    float3 direction;
    float cosine;
    float pdf;
};

// sample_uniform_cone (cycles_sample_mapping.h:315-339).
inline ConeSample sample_uniform_cone(float3 axis, float one_minus_cosine, float2 r) {
    const float2 disk = sample_uniform_disk(r);
    const float r2 = dot(disk, disk);
    const float cosine = 1.0f - r2 * one_minus_cosine;
    const float scale = std::sqrt(maxf(one_minus_cosine * (2.0f - one_minus_cosine * r2), 0.0f));
    const float2 mapped = disk * scale;
    const Basis b = make_orthonormals(axis);
    const float3 finite_dir = b.tangent * mapped.x + b.bitangent * mapped.y + axis * cosine;
    const float finite_pdf = kInvTwoPi / one_minus_cosine;
    if (one_minus_cosine > 0.0f) return {finite_dir, cosine, finite_pdf};
    return {axis, 1.0f, 1.0f};
}

}  // namespace oracle
