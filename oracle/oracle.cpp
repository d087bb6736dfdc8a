// TEST INFRASTRUCTURE ONLY -- CPU oracle of the Psycles path-trace
// integrator (the checker for the CUDA kernels; nothing in the product loads
// it).  A scalar restatement of the reference's Luisa render kernel for the
// in-scope feature set: tabulated-Sobol camera rays, closest hit with the
// Cycles Pluecker test and identity tie order, diffuse / emission /
// transparent / add / mix closures, emissive-mesh and point / spot / sun NEE
// through the flat light distribution, Russian roulette, the Cycles path
// state transition and film accumulation.  Each function cites the
// reference file:line it follows.  Threads split the image by rows; every
// pixel accumulates its samples in sample order.
#include "../include/psycles_cuda.h"
#include "oracle_math.h"
#include "oracle_sampling.h"
#include "oracle_light_tree.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <memory>
#include <thread>
#include <vector>

namespace oracle {

// ------------------------------------------------------------------ scene

struct BvhNode {
    float lo[3], hi[3];
    uint32_t left_or_first;  // inner: left child; leaf: first triangle slot
    uint32_t count;          // 0 for inner nodes (right child = left + 1)
};

struct Mesh {
    std::vector<float3> p, n;
    std::vector<uint32_t> idx, mat;
    bool smooth{false};
    uint32_t prim_offset{0};
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> order;  // leaf triangle slots -> local primitive
};

struct Instance {
    mat4 o2w, w2o, nrm;
    uint32_t mesh, material, visibility;
};

struct Material {
    std::vector<psy_closure_instruction> code;
    std::vector<psy_value_instruction> values;
    uint32_t root{0};
    std::vector<float> scalars;
    std::vector<float3> vectors;
    uint32_t emission_sampling{0};
    bool has_emission{false};
    bool has_transparent{false};
    bool bump_correction{true};  // contract::Material::use_bump_map_correction
    const float *ggx_e{nullptr};     // the scene's GGX albedo tables (MULTI_GGX glossy closures)
    const float *ggx_eavg{nullptr};
};

struct Emitter {
    uint32_t instance, prim, material, object, cycles_prim, emission_sampling;
    float3 p0, p1, p2, ng;
    float area;
};

// sampling::LightDistributionEntry (include/psycles/sampling/light_distribution.h:17).
struct DistEntry {
    float cumulative, selection_pdf;
    uint32_t kind, index;
};
constexpr uint32_t kKindTriangle = 0u, kKindAnalytic = 1u, kKindEnvironment = 2u, kKindSentinel = 3u;

struct Scene {
    std::vector<Mesh> meshes;
    std::vector<Instance> instances;
    std::vector<Material> materials;
    std::vector<psy_light_desc> lights;
    std::vector<Emitter> emitters;
    std::vector<DistEntry> distribution;  // emitter_count + 1 entries
    uint32_t emitter_count{0};
    float triangle_area_pdf{0.0f};
    float light_selection_pdf{0.0f};
    psy_camera_desc camera{};
    float3 background{};
    uint32_t world_visibility{PSY_VISIBILITY_ALL};
    bool brute_force{false};
    // many-light tree over the same emitters (triangles, then lights) and
    // the (object, primitive) -> emitter lookup of forward hits
    lt::LightTree tree;
    bool tree_usable{false};
    std::vector<std::array<uint32_t, 3>> tree_lookup;
};

// Median-split binary BVH over one mesh (object space).  The oracle's BVH
// only has to be conservative: boxes are widened and tested in double
// precision, and the closest-hit reduction is exact, so the result equals a
// brute-force scan (tests compare both).
static void build_mesh_bvh(Mesh &m) {
    const uint32_t n = static_cast<uint32_t>(m.idx.size() / 3u);
    m.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) m.order[i] = i;
    std::vector<float3> centroid(n), lo(n), hi(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float3 a = m.p[m.idx[3 * i]], b = m.p[m.idx[3 * i + 1]], c = m.p[m.idx[3 * i + 2]];
        lo[i] = {minf(a.x, minf(b.x, c.x)), minf(a.y, minf(b.y, c.y)), minf(a.z, minf(b.z, c.z))};
        hi[i] = {maxf(a.x, maxf(b.x, c.x)), maxf(a.y, maxf(b.y, c.y)), maxf(a.z, maxf(b.z, c.z))};
        centroid[i] = (lo[i] + hi[i]) * 0.5f;
    }
    m.nodes.clear();
    m.nodes.reserve(2 * n + 1);
    struct Item { uint32_t node, begin, end; };
    std::vector<Item> stack;
    m.nodes.push_back({});
    stack.push_back({0u, 0u, n});
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        double blo[3] = {1e300, 1e300, 1e300}, bhi[3] = {-1e300, -1e300, -1e300};
        double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
        for (uint32_t k = it.begin; k < it.end; ++k) {
            const uint32_t t = m.order[k];
            const float l[3] = {lo[t].x, lo[t].y, lo[t].z}, h[3] = {hi[t].x, hi[t].y, hi[t].z};
            const float c[3] = {centroid[t].x, centroid[t].y, centroid[t].z};
            for (int a = 0; a < 3; ++a) {
                blo[a] = std::min(blo[a], double(l[a]));
                bhi[a] = std::max(bhi[a], double(h[a]));
                clo[a] = std::min(clo[a], double(c[a]));
                chi[a] = std::max(chi[a], double(c[a]));
            }
        }
        BvhNode &node = m.nodes[it.node];
        for (int a = 0; a < 3; ++a) {
            const double pad = 1e-5 * (bhi[a] - blo[a]) + 1e-6 * std::max(std::fabs(blo[a]), std::fabs(bhi[a])) + 1e-30;
            node.lo[a] = float(blo[a] - pad);
            node.hi[a] = float(bhi[a] + pad);
        }
        const uint32_t count = it.end - it.begin;
        if (count <= 4u) {
            node.left_or_first = it.begin;
            node.count = count;
            continue;
        }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        const uint32_t mid = it.begin + count / 2u;
        auto key = [&](uint32_t t) {
            return axis == 0 ? centroid[t].x : axis == 1 ? centroid[t].y : centroid[t].z;
        };
        std::nth_element(m.order.begin() + it.begin, m.order.begin() + mid, m.order.begin() + it.end,
                         [&](uint32_t a, uint32_t b) { return key(a) < key(b) || (key(a) == key(b) && a < b); });
        const uint32_t left = static_cast<uint32_t>(m.nodes.size());
        m.nodes[it.node].left_or_first = left;
        m.nodes[it.node].count = 0u;
        m.nodes.push_back({});
        m.nodes.push_back({});
        stack.push_back({left, it.begin, mid});
        stack.push_back({left + 1u, mid, it.end});
    }
}

// ------------------------------------------------------ closure programs

// The value stream (GraphSurfaceImplementation::trace_value_stage,
// src/luisa/graph_surface_values.cpp:70-100): instructions 0..id in order,
// scalars held in x.  Operations as src/luisa/graph_surface_value_math.cpp:
// 54-880 (parameter, conversions, float math, mixes, colour blends),
// graph_surface_value_context.cpp:80-108 (multiply_color, invert) and
// graph_surface_value_procedural.cpp:568-600 (separate / combine RGB).
// cast<int>(x) of scalar_to_boolean truncates toward zero, NaN giving 0.
static bool truncates_nonzero(float x) {
    if (std::isnan(x)) return false;
    return std::trunc(x) != 0.0f;
}
static float3 lerp3(float3 a, float3 b, float3 t) {
    return f3(lerp(a.x, b.x, t.x), lerp(a.y, b.y, t.y), lerp(a.z, b.z, t.z));
}
static float3 eval_value(const Material &mat, uint32_t id) {
    std::vector<float3> v;
    const uint32_t n = std::min<uint32_t>(id + 1u, uint32_t(mat.values.size()));
    v.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        const psy_value_instruction &in = mat.values[i];
        const float3 a = in.a < i ? v[in.a] : f3(0.0f);
        const float3 b = in.b < i ? v[in.b] : f3(0.0f);
        const float3 c = in.c < i ? v[in.c] : f3(0.0f);
        auto clamp01 = [](float x) { return std::fmin(std::fmax(x, 0.0f), 1.0f); };
        float3 r = f3(0.0f);
        switch (in.op) {
        case PSY_VALUE_PARAMETER:
            r = in.type == PSY_VALUE_TYPE_SCALAR ? f3(mat.scalars[in.parameter], 0.0f, 0.0f) : mat.vectors[in.parameter];
            break;
        case PSY_VALUE_PASSTHROUGH: r = a; break;
        case PSY_VALUE_SCALAR_TO_COLOR: r = f3(a.x); break;
        case PSY_VALUE_SCALAR_TO_BOOLEAN: r.x = truncates_nonzero(a.x) ? 1.0f : 0.0f; break;
        case PSY_VALUE_COLOR_TO_SCALAR: r.x = a.x * 0.21267404f + a.y * 0.7151516f + a.z * 0.07217542f; break;
        case PSY_VALUE_VECTOR_TO_SCALAR: r.x = (a.x + a.y + a.z) / 3.0f; break;
        case PSY_VALUE_ADD: r.x = a.x + b.x; break;
        case PSY_VALUE_SUBTRACT: r.x = a.x - b.x; break;
        case PSY_VALUE_MULTIPLY: r.x = a.x * b.x; break;
        case PSY_VALUE_DIVIDE: r.x = std::fabs(b.x) > 1.0e-20f ? a.x / b.x : 0.0f; break;
        case PSY_VALUE_MINIMUM: r.x = std::fmin(a.x, b.x); break;
        case PSY_VALUE_MAXIMUM: r.x = std::fmax(a.x, b.x); break;
        case PSY_VALUE_POWER: r.x = pow_(std::fmax(a.x, 0.0f), b.x); break;
        case PSY_VALUE_ABSOLUTE: r.x = std::fabs(a.x); break;
        case PSY_VALUE_CLAMP01: r.x = clamp01(a.x); break;
        case PSY_VALUE_CLAMP_RANGE: {
            float lo = b.x, hi = c.x;
            if (in.static_u0 == 1u && lo > hi) std::swap(lo, hi);
            r.x = std::fmin(std::fmax(a.x, lo), hi);
            break;
        }
        case PSY_VALUE_MIX_FLOAT: r.x = lerp(a.x, b.x, in.static_u0 != 0u ? clamp01(c.x) : c.x); break;
        case PSY_VALUE_MIX_VECTOR: {
            float3 t = in.static_u0 != 0u ? c : f3(c.x);
            if (in.static_u1 != 0u) t = f3(clamp01(t.x), clamp01(t.y), clamp01(t.z));
            r = lerp3(a, b, t);
            break;
        }
        case PSY_VALUE_MIX: {
            const float t = (in.static_u1 & 1u) != 0u ? clamp01(c.x) : c.x;
            const float3 tt = f3(t);
            switch (in.static_u0) {
            case PSY_BLEND_DARKEN: r = lerp3(a, f3(std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)), tt); break;
            case PSY_BLEND_MULTIPLY: r = lerp3(a, a * b, tt); break;
            case PSY_BLEND_LIGHTEN: r = lerp3(a, f3(std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)), tt); break;
            case PSY_BLEND_SCREEN: {
                const float k = 1.0f - t;
                r = f3(1.0f - (k + t * (1.0f - b.x)) * (1.0f - a.x), 1.0f - (k + t * (1.0f - b.y)) * (1.0f - a.y),
                       1.0f - (k + t * (1.0f - b.z)) * (1.0f - a.z));
                break;
            }
            case PSY_BLEND_ADD: r = lerp3(a, a + b, tt); break;
            case PSY_BLEND_DIFFERENCE:
                r = lerp3(a, f3(std::fabs(a.x - b.x), std::fabs(a.y - b.y), std::fabs(a.z - b.z)), tt);
                break;
            case PSY_BLEND_SUBTRACT: r = lerp3(a, a - b, tt); break;
            default: r = lerp3(a, b, tt); break;
            }
            break;
        }
        case PSY_VALUE_MULTIPLY_COLOR: r = lerp3(a, a * b, f3(clamp01(c.x))); break;
        case PSY_VALUE_INVERT: r = lerp3(a, f3(1.0f) - a, f3(b.x)); break;
        case PSY_VALUE_SEPARATE_R: r.x = a.x; break;
        case PSY_VALUE_SEPARATE_G: r.x = a.y; break;
        case PSY_VALUE_SEPARATE_B: r.x = a.z; break;
        case PSY_VALUE_COMBINE_COLOR: r = f3(a.x, b.x, c.x); break;
        default: break;
        }
        v.push_back(r);
    }
    return n > id ? v[id] : f3(0.0f);
}

// A closure input: the closure node's own parameter slot (an unlinked
// socket), or a value of the stream (PSY_INPUT_VALUE: a linked socket).
static float3 input_vector(const Material &mat, uint32_t ref) {
    if ((ref & PSY_INPUT_VALUE) == 0u) return mat.vectors[ref];
    return eval_value(mat, ref & ~PSY_INPUT_VALUE);
}
static float input_scalar(const Material &mat, uint32_t ref) {
    if (ref == PSY_INPUT_NONE) return 0.0f;
    if ((ref & PSY_INPUT_VALUE) == 0u) return mat.scalars[ref];
    return eval_value(mat, ref & ~PSY_INPUT_VALUE).x;
}

// compiler::ClosureOperation walk of GraphSurfaceImplementation::
// for_each_closure (src/luisa/graph_surface_closures.cpp:5-356): add visits
// both children with the same weight, mix splits clamp(fac, 0, 1).  A
// diffuse leaf keeps its authored colour and roughness, a glossy leaf its
// roughness; a glossy op carries kBeckmann for the Beckmann distribution.
constexpr uint32_t kBeckmann = 0x100u;
constexpr uint32_t kMultiscatter = 0x200u;  // a MULTI_GGX glossy op; its closure keeps 1 / E in f0
inline bool is_glossy(uint32_t op) { return (op & 0xffu) == PSY_CLOSURE_GLOSSY; }
inline bool is_glass(uint32_t op) { return (op & 0xffu) == PSY_CLOSURE_GLASS; }
inline bool is_refraction(uint32_t op) { return (op & 0xffu) == PSY_CLOSURE_REFRACTION; }
inline bool is_dielectric(uint32_t op) { return is_glass(op) || is_refraction(op); }

struct TracedClosure {
    uint32_t op;
    float3 weight;
    float3 color;
    float roughness;
    float ior{1.0f};
};

static void walk_closures(const Material &mat, uint32_t id, float mix_weight, std::vector<TracedClosure> &out,
                          int depth) {
    if (id >= mat.code.size() || depth > 32) return;
    const psy_closure_instruction &c = mat.code[id];
    switch (c.op) {
    case PSY_CLOSURE_ADD:
        walk_closures(mat, c.a, mix_weight, out, depth + 1);
        walk_closures(mat, c.b, mix_weight, out, depth + 1);
        return;
    case PSY_CLOSURE_MIX: {
        const float factor = clampf(input_scalar(mat, c.scalar), 0.0f, 1.0f);
        walk_closures(mat, c.a, mix_weight * (1.0f - factor), out, depth + 1);
        walk_closures(mat, c.b, mix_weight * factor, out, depth + 1);
        return;
    }
    case PSY_CLOSURE_DIFFUSE:
    case PSY_CLOSURE_TRANSPARENT: {
        const float3 color = input_vector(mat, c.color);
        const float roughness = c.op == PSY_CLOSURE_DIFFUSE ? input_scalar(mat, c.roughness) : 0.0f;
        out.push_back({c.op, color * mix_weight, color, roughness});
        return;
    }
    case PSY_CLOSURE_EMISSION: {
        const float3 color = input_vector(mat, c.color) * input_scalar(mat, c.scalar);
        out.push_back({c.op, color * mix_weight, color, 0.0f});
        return;
    }
    case PSY_CLOSURE_GLOSSY: {
        const float3 color = input_vector(mat, c.color);
        const uint32_t op = c.a == PSY_GLOSSY_BECKMANN    ? (uint32_t(PSY_CLOSURE_GLOSSY) | kBeckmann)
                            : c.a == PSY_GLOSSY_MULTI_GGX ? (uint32_t(PSY_CLOSURE_GLOSSY) | kMultiscatter)
                                                          : uint32_t(PSY_CLOSURE_GLOSSY);
        out.push_back({op, color * mix_weight, color, input_scalar(mat, c.roughness)});
        return;
    }
    case PSY_CLOSURE_GLASS:
    case PSY_CLOSURE_REFRACTION: {
        // graph_surface_closures.cpp:290-320: Glass is allocated with the mix
        // weight and takes Color as its Fresnel tint; Refraction's weight is
        // Color x mix weight
        const float3 color = max3(input_vector(mat, c.color), f3(0.0f));
        const bool glass = c.op == PSY_CLOSURE_GLASS;
        const uint32_t op = uint32_t(c.op) | (c.a == PSY_GLOSSY_BECKMANN ? kBeckmann : 0u);
        out.push_back({op, glass ? f3(mix_weight) : color * mix_weight, color, input_scalar(mat, c.roughness),
                       maxf(input_scalar(mat, c.scalar), 1.0e-5f)});
        return;
    }
    default:
        return;
    }
}

// sample_weight (src/luisa/graph_surface_state.cpp:19-24).
static float closure_sample_weight(float3 w) { return std::fabs((w.x + w.y + w.z) / 3.0f); }

// bsdf_allocated_weight (graph_surface_state.cpp:39-48).
static float3 bsdf_allocated_weight(float3 v) {
    v = max3(v, f3(0.0f));
    const float average = (v.x + v.y + v.z) / 3.0f;
    return average >= 1.0e-5f ? v : f3(0.0f);
}

constexpr uint32_t kMaxClosures = 16u;

// One retained physical closure: Cycles' ShaderClosure after allocation.
struct PhysicalClosure {
    uint32_t op;  // DIFFUSE, TRANSPARENT, GLOSSY, GLASS or REFRACTION (| kBeckmann)
    float3 weight;
    float sample_weight;
    float3 normal;    // diffuse: the shading normal; glossy / glass / refraction: after setup's
                      // specular-reflection correction
    float3 color;     // authored colour (Oren-Nayar albedo); glass: the Fresnel tint
    float roughness;  // diffuse roughness (Lambert below 1e-5); microfacet roughness (alpha = roughness^2)
    float ior{1.0f};  // glass / refraction: the relative IOR (inverted on a back-facing hit)
    float f0{0.0f};   // glass: F0 of the authored IOR (the Fresnel interpolation's lower end)
};

struct SurfaceClosures {
    PhysicalClosure c[kMaxClosures];
    uint32_t count{0};
    float3 emission{};
};

// The surface point's inputs to closure setup, evaluation and sampling.
struct ClosurePoint {
    float3 shading_normal;   // SurfacePoint::shading_normal
    float3 geometric_normal; // SurfacePoint::geometric_normal (facing the incoming ray)
    float3 incoming;         // SurfacePoint::incoming (-ray direction)
    bool bump_correction;    // SurfacePoint::use_bump_map_correction
    bool back_facing;        // SurfacePoint::back_facing
};

// ensure_valid_specular_reflection (src/luisa/graph_surface_scattering.cpp:119-155):
// a shading normal whose mirror direction of `incoming` would dip below the
// geometric surface is tilted toward the geometric normal until the
// reflection clears it by min(0.9 cos_i, 0.01).
static float3 ensure_valid_specular_reflection(float3 ng, float3 incoming, float3 n) {
    const float3 reflected = 2.0f * dot(n, incoming) * n - incoming;
    const float ig = maxf(dot(incoming, ng), 0.0f);
    const float threshold = minf(0.9f * ig, 0.01f);
    const bool valid = dot(ng, reflected) >= threshold;
    const float3 tangent = safe_normalize(n - dot(n, ng) * ng, n);
    const float it = dot(incoming, tangent);
    const float a = it * it + ig * ig;
    const float b = 2.0f * (a + ig * threshold);
    const float c = (threshold + ig) * (threshold + ig);
    const float disc = maxf(b * b - 4.0f * a * c, 0.0f);
    const float signed_root = it < 0.0f ? b + std::sqrt(disc) : b - std::sqrt(disc);
    const float nz2 = clampf(0.25f * signed_root / maxf(a, 1.0e-20f), 0.0f, 1.0f);
    const float3 corrected =
        safe_normalize(std::sqrt(maxf(1.0f - nz2, 0.0f)) * tangent + std::sqrt(nz2) * ng, ng);
    return (!valid && a > 1.0e-20f) ? corrected : n;
}

// maybe_ensure_valid_specular_reflection (graph_surface_scattering.cpp:157-168).
static float3 specular_normal(bool correction, float3 ng, float3 incoming, float3 n) {
    const bool equal = ng.x == n.x && ng.y == n.y && ng.z == n.z;
    return correction && !equal ? ensure_valid_specular_reflection(ng, incoming, n) : n;
}

// fresnel_dielectric_cos / f0_from_ior (graph_surface_scattering.cpp:42-58).
static float fresnel_dielectric_cos(float cosine, float eta) {
    const float c = std::fabs(cosine);
    const float g2 = eta * eta - 1.0f + c * c;
    const float g = std::sqrt(maxf(g2, 0.0f));
    const float a = (g - c) / maxf(g + c, 1.0e-20f);
    const float den = c * (g - c) + 1.0f;
    const float b = (c * (g + c) - 1.0f) / (std::fabs(den) > 1.0e-20f ? den : 1.0e-20f);
    const float regular = 0.5f * a * a * (1.0f + b * b);
    return g2 > 0.0f ? regular : 1.0f;
}
static float f0_from_ior(float ior) {
    const float r = (ior - 1.0f) / maxf(ior + 1.0f, 1.0e-20f);
    return r * r;
}

// cycles_table_1d / cycles_table_2d (src/luisa/graph_surface_state.cpp:84-130):
// coordinates clamped to [0, 1], linear between the two nearest entries; a
// 2-D table is y_size rows of x_size entries.
static float cycles_table_1d(const float *table, float x, uint32_t size) {
    const float coordinate = clampf(x, 0.0f, 1.0f) * float(size - 1u);
    const uint32_t index = std::min(uint32_t(coordinate), size - 1u);
    const uint32_t next = std::min(index + 1u, size - 1u);
    const float t = coordinate - float(index);
    return lerp(table[index], table[next], t);
}
static float cycles_table_2d(const float *table, float x, float y, uint32_t x_size, uint32_t y_size) {
    const float coordinate = clampf(y, 0.0f, 1.0f) * float(y_size - 1u);
    const uint32_t index = std::min(uint32_t(coordinate), y_size - 1u);
    const uint32_t next = std::min(index + 1u, y_size - 1u);
    const float t = coordinate - float(index);
    const float d0 = cycles_table_1d(table + x_size * index, x, x_size);
    const float d1 = cycles_table_1d(table + x_size * next, x, x_size);
    return lerp(d0, d1, t);
}

// ggx_energy (src/luisa/graph_surface_scattering.cpp:170-198): MULTI_GGX's
// darkening of the weight, (1 + Fms (1 - E) / E) E, and evaluation scale 1 / E.
struct GgxEnergy {
    float3 darkening;
    float energy_scale;
};
static GgxEnergy ggx_energy(const Material &mat, float roughness, float incoming_cosine, float3 fss) {
    const float energy = maxf(cycles_table_2d(mat.ggx_e, roughness, incoming_cosine, 32u, 32u), 1.0e-20f);
    const float average = cycles_table_1d(mat.ggx_eavg, roughness, 32u);
    const float missing = (1.0f - energy) / energy;
    const float scale = 1.0f / energy;
    const float3 fms(fss.x * average / maxf(1.0f - fss.x * (1.0f - average), 1.0e-20f),
                     fss.y * average / maxf(1.0f - fss.y * (1.0f - average), 1.0e-20f),
                     fss.z * average / maxf(1.0f - fss.z * (1.0f - average), 1.0e-20f));
    GgxEnergy r;
    r.darkening = float3((1.0f + fms.x * missing) / scale, (1.0f + fms.y * missing) / scale,
                         (1.0f + fms.z * missing) / scale);
    r.energy_scale = scale;
    return r;
}

// Closure allocation (graph_surface_state.cpp:26-48,
// graph_surface_physical_closures.cpp:158-520): diffuse goes through
// bsdf_alloc (negative weight clamped, average cutoff 1e-5); glossy is
// allocated the same way (reflective caustics on), its normal corrected
// for a valid specular reflection and its weight kept (GGX / Beckmann
// without energy preservation: darkening and evaluation scale one);
// transparent keeps its signed weight, uses the cutoff on |average|, and
// every allocated transparent contribution merges into the first one
// (bsdf_transparent_setup, :483-518: summed weights and sample weights).
static SurfaceClosures collect_surface(const Material &mat, const ClosurePoint &pt) {
    std::vector<TracedClosure> traced;
    walk_closures(mat, mat.root, 1.0f, traced, 0);
    SurfaceClosures s;
    const float3 closure_normal = safe_normalize(pt.shading_normal, pt.shading_normal);
    const float3 incoming = safe_normalize(pt.incoming, pt.shading_normal);
    int transparent_slot = -1;
    for (const auto &t : traced) {
        if (t.op == PSY_CLOSURE_EMISSION) {
            s.emission += t.weight;
            continue;
        }
        PhysicalClosure p;
        p.op = t.op;
        p.color = t.color;
        p.roughness = t.roughness;
        if (t.op == PSY_CLOSURE_DIFFUSE) {
            p.weight = bsdf_allocated_weight(t.weight);
            p.sample_weight = closure_sample_weight(p.weight);
            p.normal = closure_normal;
            if (!(p.weight.x != 0.0f || p.weight.y != 0.0f || p.weight.z != 0.0f)) continue;
        } else if (is_glossy(t.op)) {
            const float3 allocated = max3(t.weight, f3(0.0f));
            const float allocation = closure_sample_weight(allocated);
            if (!(allocation >= 1.0e-5f)) continue;
            p.weight = allocated;
            p.sample_weight = allocation * closure_sample_weight(f3(1.0f));
            p.normal = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, closure_normal);
            if ((t.op & kMultiscatter) != 0u) {
                // MULTI_GGX (graph_surface_physical_closures.cpp:379-391): the Fresnel
                // single-scattering albedo is max(colour, 0)
                const GgxEnergy e = ggx_energy(mat, clampf(t.roughness, 0.0f, 1.0f),
                                               clampf(dot(p.normal, incoming), 0.0f, 1.0f), max3(t.color, f3(0.0f)));
                p.weight = allocated * e.darkening;
                p.sample_weight = allocation * closure_sample_weight(e.darkening);
                p.f0 = e.energy_scale;
            }
        } else if (is_dielectric(t.op)) {
            // MicrofacetGlassComponent::setup (microfacet_glass_component.cpp:180-232): the
            // corrected normal, roughness sqrt(clamp(r^2)), the IOR inverted on a
            // back face; weight = max(weight, 0) (no energy preservation: darkening
            // one).  A glass closure's selection weight would scale this by Cycles'
            // tabulated Fresnel albedo; a glass closure is the only BSDF closure of
            // its material (compile refuses other mixes), so that factor only
            // rescales weighted_pdf / total and is taken as one.
            const float3 allocated = max3(t.weight, f3(0.0f));
            const float allocation = closure_sample_weight(allocated);
            if (!(allocation >= 1.0e-5f)) continue;
            p.weight = allocated;
            p.sample_weight = allocation * 1.0f * closure_sample_weight(f3(1.0f));
            p.normal = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, closure_normal);
            p.roughness = std::sqrt(clampf(t.roughness * t.roughness, 0.0f, 1.0f));
            p.ior = pt.back_facing ? 1.0f / t.ior : t.ior;
            p.f0 = clampf(f0_from_ior(t.ior), 0.0f, 1.0f);
        } else {
            const float sw = closure_sample_weight(t.weight);
            if (!(sw >= 1.0e-5f)) continue;
            if (transparent_slot >= 0) {
                s.c[transparent_slot].weight += t.weight;
                s.c[transparent_slot].sample_weight += sw;
                continue;
            }
            p.weight = t.weight;
            p.sample_weight = sw;
            p.normal = pt.shading_normal;
        }
        if (s.count >= kMaxClosures) continue;
        if (t.op == PSY_CLOSURE_TRANSPARENT) transparent_slot = int(s.count);
        s.c[s.count++] = p;
    }
    return s;
}

// Cycles ClosureLabel / runtime-flag constants
// (include/psycles/luisa/cycles_closure.h:39-66) and contract surface
// events (include/psycles/contract/surface.h).
constexpr uint32_t kEventReflection = 1u, kEventTransmission = 2u, kEventDiffuse = 4u, kEventGlossy = 8u,
                   kEventSingular = 16u, kEventTransparent = 32u;
constexpr uint32_t kLabelTransmit = 1u, kLabelReflect = 2u, kLabelDiffuse = 4u, kLabelGlossy = 8u,
                   kLabelSingular = 16u, kLabelTransparent = 32u;
constexpr uint32_t kRuntimeBackfacing = 1u, kRuntimeEmission = 4u, kRuntimeBsdf = 8u, kRuntimeBsdfHasEval = 16u,
                   kRuntimeTransparent = 1024u, kRuntimeBsdfHasTransmission = 2048u;
constexpr float kMicrofacetSingularAlphaProduct = 2.0e-10f;

// cycles_closure::label_from_events (cycles_closure.h:67-112).
static uint32_t label_from_events(uint32_t e) {
    uint32_t l = 0u;
    if (e & kEventTransmission) l |= kLabelTransmit;
    if (e & kEventReflection) l |= kLabelReflect;
    if (e & kEventDiffuse) l |= kLabelDiffuse;
    if (e & kEventGlossy) l |= kLabelGlossy;
    if (e & kEventSingular) l |= kLabelSingular;
    if (e & kEventTransparent) l |= kLabelTransparent;
    return l;
}

// microfacet_alpha / microfacet_is_singular (graph_surface_scattering.cpp:549-568)
// without the glossy filter (its roughness is zero: Filter Glossy off).
static float microfacet_alpha(float roughness) {
    const float a = clampf(roughness, 0.0f, 1.0f);
    return a * a;
}
static bool microfacet_singular(float roughness) {
    const float a = microfacet_alpha(roughness);
    return a * a <= kMicrofacetSingularAlphaProduct;
}

// cycles_runtime_flags (src/luisa/graph_surface_scattering.cpp:292-365)
// for the in-scope closures, plus the back-facing bit.
static uint32_t runtime_flags(const SurfaceClosures &s, bool back_facing) {
    uint32_t f = back_facing ? kRuntimeBackfacing : 0u;
    for (uint32_t i = 0; i < s.count; ++i) {
        const PhysicalClosure &c = s.c[i];
        if (c.op == PSY_CLOSURE_DIFFUSE) f |= kRuntimeBsdf | kRuntimeBsdfHasEval;
        else if (is_glossy(c.op)) f |= kRuntimeBsdf | (microfacet_singular(c.roughness) ? 0u : kRuntimeBsdfHasEval);
        else if (is_dielectric(c.op))
            f |= kRuntimeBsdf | (microfacet_singular(c.roughness) ? 0u : kRuntimeBsdfHasEval) | kRuntimeBsdfHasTransmission;
        else f |= kRuntimeBsdf | kRuntimeTransparent;
    }
    return f;
}

// bump_shadowing_term (graph_surface_scattering.cpp:219-281) of a diffuse
// or glossy closure: one when the closure normal is the shading normal;
// otherwise a direction on the wrong side of the smooth surface is rejected
// during evaluation (and, for diffuse closures, also when sampling), and
// a diffuse closure under bump correction gets the smoothed shadowing
// factor.
static float bump_shadowing(float3 smooth_normal, float3 closure_normal, float3 direction, bool is_evaluation,
                            bool diffuse, bool bump_correction) {
    if (closure_normal.x == smooth_normal.x && closure_normal.y == smooth_normal.y &&
        closure_normal.z == smooth_normal.z)
        return 1.0f;
    const float csd = dot(smooth_normal, direction);
    const float csc = dot(smooth_normal, closure_normal);
    const float ccd = dot(closure_normal, direction);
    const bool reject = csd * csc * ccd < 0.0f && (is_evaluation || diffuse);
    const float cos_i = std::fabs(csd);
    const float cos_d = std::fabs(csc);
    const float tan_d2 = maxf(1.0f / maxf(cos_d * cos_d, 1.0e-20f) - 1.0f, 0.0f);
    const float bump_alpha2 = clampf(0.125f * tan_d2, 0.0f, 1.0f);
    const float tan_i2 = maxf(1.0f / maxf(cos_i * cos_i, 1.0e-20f) - 1.0f, 0.0f);
    const float lambda = 0.5f * (std::sqrt(1.0f + bump_alpha2 * tan_i2) - 1.0f);
    const float smoothed = 1.0f / (1.0f + lambda);
    const bool domain = diffuse && bump_correction && cos_d < 1.0f && cos_i < 1.0f;
    const bool grazing = domain && cos_i < 1.0e-6f;
    float result = domain && !grazing ? smoothed : 1.0f;
    if (reject || grazing) result = 0.0f;
    return result;
}

// microfacet_distribution / microfacet_lambda (graph_surface_scattering.cpp:508-547).
static float microfacet_distribution(bool beckmann, float n_dot_h, float alpha) {
    const float alpha2 = alpha * alpha;
    const float cosine2 = minf(n_dot_h * n_dot_h, 1.0f);
    const float one_minus = 1.0f - cosine2;
    if (!beckmann) {
        const float den = one_minus + alpha2 * cosine2;
        return alpha2 / maxf(kPi * den * den, 1.0e-20f);
    }
    const float exponent = one_minus / (cosine2 * alpha2);
    return 1.0f / (exp_(exponent) * kPi * alpha2 * cosine2 * cosine2);
}
static float microfacet_lambda(bool beckmann, float n_dot_v, float alpha) {
    const float cosine2 = n_dot_v * n_dot_v;
    const float sat = alpha * alpha * maxf(1.0f / cosine2 - 1.0f, 0.0f);
    if (!beckmann) return 0.5f * (std::sqrt(1.0f + sat) - 1.0f);
    const float a = 1.0f / std::sqrt(sat);
    const float approximation = ((0.396f * a - 1.259f) * a + 1.0f) / ((2.181f * a + 3.535f) * a);
    return sat < 0.39f ? 0.0f : approximation;
}

// microfacet_intensity and microfacet_pdf (graph_surface_scattering.cpp:665-728)
// of a standalone glossy closure (Fresnel constant one: its colour is in
// the closure weight).
static float microfacet_intensity(const PhysicalClosure &c, float3 incoming, float3 outgoing, float3 gn) {
    const bool beckmann = (c.op & kBeckmann) != 0u;
    const float ndv = maxf(dot(gn, incoming), 0.0f);
    const float ndl = maxf(dot(gn, outgoing), 0.0f);
    const float3 h = safe_normalize(incoming + outgoing, gn);
    const float ndh = maxf(dot(gn, h), 0.0f);
    const float vdh = maxf(dot(incoming, h), 0.0f);
    const bool singular = microfacet_singular(c.roughness);
    const float alpha = maxf(microfacet_alpha(c.roughness), 1.0e-10f);
    const float d = microfacet_distribution(beckmann, ndh, alpha);
    const float g = 1.0f / (1.0f + microfacet_lambda(beckmann, ndv, alpha) + microfacet_lambda(beckmann, ndl, alpha));
    // the glossy Fresnel factor: one, or MULTI_GGX's scale 1 / E (microfacet_reflection_fresnel,
    // graph_surface_scattering.cpp:632-662)
    const float fresnel = (c.op & kMultiscatter) != 0u ? c.f0 : 1.0f;
    const float intensity = fresnel * d * g / maxf(4.0f * ndv, 1.0e-20f);
    return (ndv > 0.0f && ndl > 0.0f && ndh > 0.0f && vdh > 0.0f && !singular) ? intensity : 0.0f;
}
static float microfacet_pdf(const PhysicalClosure &c, float3 incoming, float3 outgoing, float3 gn) {
    const bool beckmann = (c.op & kBeckmann) != 0u;
    const float3 h = safe_normalize(incoming + outgoing, gn);
    const float ndh = maxf(dot(gn, h), 0.0f);
    const float vdh = maxf(dot(incoming, h), 0.0f);
    const bool singular = microfacet_singular(c.roughness);
    const float alpha = maxf(microfacet_alpha(c.roughness), 1.0e-10f);
    const float ndv = maxf(dot(gn, incoming), 0.0f);
    const float ndl = maxf(dot(gn, outgoing), 0.0f);
    const float pdf = microfacet_distribution(beckmann, ndh, alpha) / maxf(4.0f * ndv, 1.0e-20f) /
                      (1.0f + microfacet_lambda(beckmann, ndv, alpha));
    return (ndv > 0.0f && ndl > 0.0f && ndh > 0.0f && vdh > 0.0f && !singular) ? pdf : 0.0f;
}

struct GlassFresnel {
    float3 reflection, transmission;
};

// glass_fresnel / masked_fresnel (microfacet_glass_component.cpp:32-77) of a
// standalone Glass closure (F0 of its IOR, F90 one, both tints its colour:
// caustics on) or Refraction closure (no reflection; transmission one unless
// totally reflected).
static GlassFresnel glass_fresnel(const PhysicalClosure &c, float cos_hi, bool reflection_allowed,
                                  bool transmission_allowed) {
    const float real = fresnel_dielectric_cos(cos_hi, c.ior);
    GlassFresnel r;
    if (is_refraction(c.op)) {
        r.reflection = f3(0.0f);
        r.transmission = real == 1.0f ? f3(0.0f) : f3(1.0f);
    } else {
        const float real_f0 = f0_from_ior(c.ior);
        const float t = clampf((real - real_f0) / (1.0f - real_f0), 0.0f, 1.0f);
        const float3 fresnel = f3(lerp(c.f0, 1.0f, t));
        r.reflection = fresnel * c.color;
        r.transmission = (f3(1.0f) - fresnel) * c.color;
    }
    if (!reflection_allowed) r.reflection = f3(0.0f);
    if (!transmission_allowed) r.transmission = f3(0.0f);
    return r;
}

static float reflection_probability(const GlassFresnel &f) {
    const float r = closure_sample_weight(f.reflection);
    const float t = closure_sample_weight(f.transmission);
    return r / maxf(r + t, 1.0e-20f);
}

struct GlassGeometry {
    float3 half;
    float inverse_half_length, cos_i, cos_o, cos_hi, cos_nh, cos_ho;
    bool transmission;
};

// glass_geometry (microfacet_glass_component.cpp:79-109).
static GlassGeometry glass_geometry(const PhysicalClosure &c, float3 incoming, float3 outgoing, float3 n) {
    GlassGeometry g;
    g.cos_o = dot(n, outgoing);
    g.transmission = g.cos_o < 0.0f;
    const float3 uh = g.transmission ? -(c.ior * outgoing + incoming) : incoming + outgoing;
    const float hl = std::sqrt(dot(uh, uh));
    const bool unit_ior_transmission = g.transmission && c.ior == 1.0f;
    const bool finite = hl != 0.0f && !unit_ior_transmission;
    g.inverse_half_length = finite ? 1.0f / hl : 0.0f;
    g.half = uh * g.inverse_half_length;
    g.cos_i = dot(n, incoming);
    g.cos_hi = dot(g.half, incoming);
    g.cos_nh = dot(n, g.half);
    g.cos_ho = dot(g.half, outgoing);
    return g;
}

// MicrofacetGlassComponent::intensity and ::pdf (microfacet_glass_component.cpp:234-320).
static float3 glass_intensity(const PhysicalClosure &c, float3 incoming, float3 outgoing, float3 gn) {
    const bool beckmann = (c.op & kBeckmann) != 0u;
    const GlassGeometry g = glass_geometry(c, incoming, outgoing, gn);
    const float setup_alpha = microfacet_alpha(c.roughness);
    const float alpha = maxf(setup_alpha, 1.0e-7f);
    const float d = microfacet_distribution(beckmann, g.cos_nh, alpha);
    const float li = microfacet_lambda(beckmann, g.cos_i, alpha);
    const float lo = microfacet_lambda(beckmann, g.cos_o, alpha);
    const GlassFresnel f = glass_fresnel(c, g.cos_hi, true, true);
    const float3 lobe = g.transmission ? f.transmission : f.reflection;
    const float jacobian = c.ior * c.ior * g.inverse_half_length * g.inverse_half_length * std::fabs(g.cos_hi * g.cos_ho);
    const float common = d / g.cos_i * (g.transmission ? jacobian : 0.25f);
    const float3 value = lobe * common / (1.0f + li + lo) * 1.0f;
    const bool valid = g.cos_i > 0.0f && setup_alpha * setup_alpha > kMicrofacetSingularAlphaProduct;
    return valid ? value : f3(0.0f);
}
static float glass_pdf(const PhysicalClosure &c, float3 incoming, float3 outgoing, float3 gn, bool reflection_allowed,
                       bool transmission_allowed) {
    const bool beckmann = (c.op & kBeckmann) != 0u;
    const GlassGeometry g = glass_geometry(c, incoming, outgoing, gn);
    const float setup_alpha = microfacet_alpha(c.roughness);
    const float alpha = maxf(setup_alpha, 1.0e-7f);
    const float d = microfacet_distribution(beckmann, g.cos_nh, alpha);
    const GlassFresnel f = glass_fresnel(c, g.cos_hi, reflection_allowed, transmission_allowed);
    const float probability = reflection_probability(f);
    const float lobe_probability = g.transmission ? 1.0f - probability : probability;
    const float li = microfacet_lambda(beckmann, g.cos_i, alpha);
    const float jacobian = c.ior * c.ior * g.inverse_half_length * g.inverse_half_length * std::fabs(g.cos_hi * g.cos_ho);
    const float common = d / g.cos_i * (g.transmission ? jacobian : 0.25f);
    const float directional = common / (1.0f + li);
    const float lobe_energy = g.transmission ? closure_sample_weight(f.transmission) : closure_sample_weight(f.reflection);
    const bool valid = g.cos_i > 0.0f && lobe_energy > 0.0f && setup_alpha * setup_alpha > kMicrofacetSingularAlphaProduct;
    return valid ? directional * lobe_probability : 0.0f;
}

struct GlassSample {
    float3 direction, singular_evaluation;
    float singular_pdf;
    bool transmission, singular, valid;
};

// MicrofacetGlassComponent::sample (microfacet_glass_component.cpp:322-395).
static GlassSample glass_sample(const PhysicalClosure &c, float3 incoming, float3 gn, float3 ng, float2 random,
                                float random_lobe, bool reflection_allowed, bool transmission_allowed) {
    const float alpha = microfacet_alpha(c.roughness);
    bool singular = alpha * alpha <= kMicrofacetSingularAlphaProduct;
    const float sampling_alpha = maxf(alpha, 1.0e-7f);
    const float3 sampled = (c.op & kBeckmann) != 0u ? sample_beckmann_visible_normal(gn, incoming, sampling_alpha, random)
                                                    : sample_ggx_visible_normal(gn, incoming, sampling_alpha, random);
    const float3 h = singular ? gn : sampled;
    const float cos_hi = dot(h, incoming);
    const GlassFresnel f = glass_fresnel(c, cos_hi, reflection_allowed, transmission_allowed);
    const float probability = reflection_probability(f);
    GlassSample r;
    r.transmission = random_lobe >= probability;
    const float3 reflected = 2.0f * cos_hi * h - incoming;
    const float e2 = c.ior * c.ior - (1.0f - cos_hi * cos_hi);
    const float cos_ho = -std::sqrt(maxf(e2, 0.0f)) / c.ior;
    const float inverse_eta = 1.0f / c.ior;
    const float3 transmitted = (inverse_eta * cos_hi + cos_ho) * h - inverse_eta * incoming;
    r.direction = r.transmission ? transmitted : reflected;
    const float3 selected = r.transmission ? f.transmission : f.reflection;
    const float lobe_probability = r.transmission ? 1.0f - probability : probability;
    const bool shading_negative = dot(gn, r.direction) < 0.0f;
    const bool geometric_negative = dot(ng, r.direction) < 0.0f;
    const bool shading_ok = r.transmission ? shading_negative : !shading_negative;
    const bool geometric_ok = r.transmission ? geometric_negative : !geometric_negative;
    const bool has_energy = closure_sample_weight(f.reflection + f.transmission) > 0.0f;
    r.valid = has_energy && cos_hi > 0.0f && shading_ok && geometric_ok;
    singular = singular || (r.transmission && std::fabs(c.ior - 1.0f) < 1.0e-4f);
    r.singular = singular;
    r.singular_evaluation = c.weight * selected * 1.0f * 1.0e6f;
    r.singular_pdf = lobe_probability * 1.0e6f;
    return r;
}

struct Evaluation {
    float3 f{};
    float3 diffuse_f{};
    float pdf{0.0f};
    uint32_t events{0u};
};

// oren_nayar_g (src/luisa/graph_surface_scattering.cpp:463-473).
static float oren_nayar_g(float cosine) {
    const float c = clampf(cosine, 0.0f, 1.0f);
    const float sine = std::sqrt(maxf(1.0f - c * c, 0.0f));
    const float theta = acos_(c);
    const float safe_cosine = maxf(c, 1.0e-6f);
    const float regular = sine * (theta - 2.0f / 3.0f - sine * c) +
                          2.0f / 3.0f * (sine / safe_cosine) * (1.0f - sine * sine * sine);
    const float taylor = (kPi * 0.5f - 2.0f / 3.0f) - c;
    return c < 1.0e-6f ? taylor : regular;
}

// diffuse_intensity (src/luisa/graph_surface_scattering.cpp:475-506): Lambert
// below roughness 1e-5, else Cycles' energy-compensated Oren-Nayar (single
// scattering a + b t plus the multiple-scattering term of the clamped
// albedo).  `incoming` points to the viewer, `outgoing` to the light.
static float3 diffuse_intensity(const PhysicalClosure &c, float3 incoming, float3 outgoing) {
    const float nl = maxf(dot(c.normal, outgoing), 0.0f);
    const float sigma = clampf(c.roughness, 0.0f, 1.0f);
    if (sigma < 1.0e-5f) return f3(nl * kInvPi);
    const float a = 1.0f / (kPi + sigma * (kPi * 0.5f - 2.0f / 3.0f));
    const float b = sigma * a;
    const float nv = maxf(dot(c.normal, incoming), 0.0f);
    float t = dot(outgoing, incoming) - nl * nv;
    if (t > 0.0f) t = t / (maxf(nl, nv) + 1.17549435e-38f);
    const float single_scatter = a + b * t;
    const float3 albedo = clamp3(c.color, 0.0f, 1.0f);
    const float e_average = a * kPi + ((2.0f * kPi - 5.6f) / 3.0f) * b;
    const float ratio = e_average / (1.0f - e_average);
    const float keep = 1.0f - e_average;
    const float3 e_ms = f3(kInvPi * (albedo.x * albedo.x) * ratio / (1.0f - albedo.x * keep),
                           kInvPi * (albedo.y * albedo.y) * ratio / (1.0f - albedo.y * keep),
                           kInvPi * (albedo.z * albedo.z) * ratio / (1.0f - albedo.z * keep));
    const float e_incoming = a * kPi + b * oren_nayar_g(nv);
    const float3 multiscatter = e_ms * (1.0f - e_incoming);
    const float e_outgoing = a * kPi + b * oren_nayar_g(nl);
    return (f3(single_scatter) + multiscatter * (1.0f - e_outgoing)) * nl;
}

// Mixture evaluation of every retained closure in a direction
// (surface_closure_evaluation_contribution, src/luisa/surface_closure_evaluation.cpp:61-394,
// and SurfaceClosureEvaluationAccumulator::finish :410-438).  `selected`
// marks the closure that produced the direction (its pdf survives a zero
// bump term, and a glossy closure is not rejected for it).
static Evaluation evaluate_mixture(const SurfaceClosures &s, const ClosurePoint &pt, float3 outgoing_raw,
                                   uint32_t lobe_mask, int selected) {
    const float3 outgoing = safe_normalize(outgoing_raw, pt.shading_normal);
    const float3 incoming = safe_normalize(pt.incoming, -outgoing);
    Evaluation e;
    float total = 0.0f, weighted_pdf = 0.0f;
    const bool diffuse_enabled = (lobe_mask & kEventDiffuse) != 0u;
    const bool glossy_enabled = (lobe_mask & kEventGlossy) != 0u;
    const bool transparent_enabled = (lobe_mask & kEventTransparent) != 0u;
    const bool transmission_enabled = (lobe_mask & kEventTransmission) != 0u;
    for (uint32_t i = 0; i < s.count; ++i) {
        const PhysicalClosure &c = s.c[i];
        if (c.op == PSY_CLOSURE_TRANSPARENT) {
            if (transparent_enabled) total += c.sample_weight;
            continue;
        }
        const bool is_selected = int(i) == selected;
        if (is_dielectric(c.op)) {
            // glass / refraction (surface_closure_evaluation.cpp:134-394): the side of
            // `outgoing` picks reflection or transmission; a selected transmission
            // keeps its bump term, and a selected unit-IOR transmission is a delta
            const float3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, c.normal);
            const bool transmission = dot(gn, outgoing) < 0.0f;
            const bool unit_ior_delta = is_selected && transmission && std::fabs(c.ior - 1.0f) < 1.0e-4f;
            float bump = bump_shadowing(pt.shading_normal, c.normal, outgoing, !is_selected, false,
                                        pt.bump_correction);
            if (is_selected && transmission) bump = 1.0f;
            const bool pdf_valid = bump != 0.0f || is_selected;
            const bool allowed = is_glass(c.op) ? (transmission ? transmission_enabled : glossy_enabled)
                                                : (glossy_enabled && transmission_enabled);
            if (!allowed) continue;  // any_allowed false: no weight, no pdf
            float pdf = glass_pdf(c, incoming, outgoing, gn, glossy_enabled, transmission_enabled);
            if (!pdf_valid || unit_ior_delta) pdf = 0.0f;
            float3 value = c.weight * glass_intensity(c, incoming, outgoing, gn) * bump;
            if (unit_ior_delta) value = f3(0.0f);
            e.f += value;
            total += c.sample_weight;
            weighted_pdf += c.sample_weight * pdf;
            if (closure_sample_weight(value) > 0.0f)
                e.events |= kEventGlossy | (transmission ? kEventTransmission : kEventReflection);
            continue;
        }
        const bool glossy = is_glossy(c.op);
        const float bump = bump_shadowing(pt.shading_normal, c.normal, outgoing, !is_selected, !glossy,
                                          pt.bump_correction);
        const bool pdf_valid = bump != 0.0f || is_selected;
        if (glossy) {
            if (!glossy_enabled) continue;  // any_allowed false: no weight, no pdf
            const float3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, c.normal);
            const float pdf = pdf_valid ? microfacet_pdf(c, incoming, outgoing, gn) : 0.0f;
            const float3 value = c.weight * microfacet_intensity(c, incoming, outgoing, gn) * bump;
            e.f += value;
            total += c.sample_weight;
            weighted_pdf += c.sample_weight * pdf;
            if (closure_sample_weight(value) > 0.0f) e.events |= kEventGlossy | kEventReflection;
            continue;
        }
        float pdf = maxf(dot(c.normal, outgoing), 0.0f) * kInvPi;
        if (!pdf_valid) pdf = 0.0f;
        if (!diffuse_enabled) continue;
        const float3 value = c.weight * diffuse_intensity(c, incoming, outgoing) * bump;
        e.f += value;
        e.diffuse_f += value;
        total += c.sample_weight;
        weighted_pdf += c.sample_weight * pdf;
        if (closure_sample_weight(value) > 0.0f) e.events |= kEventDiffuse | kEventReflection;
    }
    e.pdf = total > 0.0f ? weighted_pdf / maxf(total, 1.0e-20f) : 0.0f;
    if (!(weighted_pdf > 0.0f)) e.events = 0u;
    return e;
}

struct SurfaceSample {
    bool valid{false};
    float3 wi{};
    Evaluation eval{};
    uint32_t closure_index{kInvalid};
};

// Closure selection + conditional sample + mixture (SurfaceClosureSamplingVisitor::visit,
// src/luisa/surface_closure_sampling_core.cpp:744-812; selection :97-214;
// categorical inversion :420-437; conditional sample :216-337, glossy
// sample_microfacet_reflection graph_surface_scattering.cpp:730-770;
// finish :490-660).
static SurfaceSample sample_surface(const SurfaceClosures &s, const ClosurePoint &pt, float u_lobe, float2 u_dir,
                                    uint32_t lobe_mask) {
    SurfaceSample out;
    const bool diffuse_enabled = (lobe_mask & kEventDiffuse) != 0u;
    const bool glossy_enabled = (lobe_mask & kEventGlossy) != 0u;
    const bool transparent_enabled = (lobe_mask & kEventTransparent) != 0u;
    const bool transmission_enabled = (lobe_mask & kEventTransmission) != 0u;
    const float3 incoming = safe_normalize(pt.incoming, pt.shading_normal);
    float weights[kMaxClosures];
    float total = 0.0f;
    for (uint32_t i = 0; i < s.count; ++i) {
        const uint32_t op = s.c[i].op;
        const bool eligible = op == PSY_CLOSURE_DIFFUSE ? diffuse_enabled
                              : is_glossy(op)           ? glossy_enabled
                              : is_glass(op)            ? (glossy_enabled || transmission_enabled)
                              : is_refraction(op)       ? (glossy_enabled && transmission_enabled)
                                                        : transparent_enabled;
        weights[i] = eligible ? s.c[i].sample_weight : 0.0f;
        total += weights[i];
    }
    const float random_lobe = clampf(u_lobe, 0.0f, 0.99999994f);
    const float target = random_lobe * total;
    float accumulated = 0.0f;
    int chosen = -1;
    float rescaled = random_lobe;
    for (uint32_t i = 0; i < s.count; ++i) {
        const float next = accumulated + weights[i];
        if (chosen < 0 && weights[i] > 0.0f && target < next) {
            chosen = int(i);
            // SurfaceClosureCategoricalInversion::consider (:420-437): the lobe
            // number rescaled into the chosen closure's interval
            if (s.count > 1u) rescaled = (target - accumulated) / maxf(weights[i], 1.0e-20f);
        }
        accumulated = next;
    }
    if (chosen < 0) return out;
    const PhysicalClosure &c = s.c[chosen];
    float3 direction;
    const bool transparent = c.op == PSY_CLOSURE_TRANSPARENT;
    const bool glossy = is_glossy(c.op);
    const bool dielectric = is_dielectric(c.op);
    bool candidate_valid = true, singular = false, transmission = false;
    GlassSample gs{};
    if (transparent) {
        direction = pt.incoming * -1.0f;
    } else if (dielectric) {
        const float3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, c.normal);
        gs = glass_sample(c, incoming, gn, pt.geometric_normal, u_dir, rescaled, glossy_enabled, transmission_enabled);
        direction = gs.direction;
        candidate_valid = gs.valid;
        singular = gs.singular;
        transmission = gs.transmission;
    } else if (glossy) {
        const float3 gn = specular_normal(pt.bump_correction, pt.geometric_normal, incoming, c.normal);
        const float alpha = microfacet_alpha(c.roughness);
        const float sampling_alpha = maxf(alpha, 1.0e-10f);
        const float3 h = (c.op & kBeckmann) != 0u ? sample_beckmann_visible_normal(gn, incoming, sampling_alpha, u_dir)
                                                  : sample_ggx_visible_normal(gn, incoming, sampling_alpha, u_dir);
        singular = alpha * alpha <= kMicrofacetSingularAlphaProduct;
        direction = singular ? 2.0f * dot(gn, incoming) * gn - incoming : 2.0f * dot(incoming, h) * h - incoming;
        candidate_valid = dot(gn, incoming) > 0.0f && dot(gn, direction) > 0.0f &&
                          dot(pt.geometric_normal, direction) > 0.0f;
    } else {
        direction = sample_cosine_hemisphere(c.normal, u_dir).direction;
    }
    const bool geometric_valid =
        transmission ? dot(pt.geometric_normal, direction) < 0.0f : dot(pt.geometric_normal, direction) > 0.0f;
    const bool sample_valid = candidate_valid && (transparent || geometric_valid);
    out.closure_index = uint32_t(chosen);
    out.wi = direction;
    if (!sample_valid) return out;
    Evaluation mixture = evaluate_mixture(s, pt, direction, lobe_mask, chosen);
    Evaluation r;
    r.f = mixture.f;
    r.diffuse_f = mixture.diffuse_f;
    float delta_pdf_numerator = 0.0f;
    if (transparent) {
        r.f += c.weight * 1.0e6f;
        delta_pdf_numerator = 1.0e6f * weights[chosen];
    } else if (glossy && singular) {
        // singular_evaluation = weight x Fresnel (one, or MULTI_GGX's scale)
        // x bump term (one when sampling a glossy closure) x 1e6, singular pdf 1e6
        r.f += (c.op & kMultiscatter) != 0u ? c.weight * c.f0 * 1.0e6f : c.weight * 1.0e6f;
        delta_pdf_numerator = 1.0e6f * weights[chosen];
    } else if (dielectric && singular) {
        r.f += gs.singular_evaluation;
        delta_pdf_numerator = gs.singular_pdf * weights[chosen];
    }
    r.pdf = mixture.pdf + delta_pdf_numerator / maxf(total, 1.0e-20f);
    if (transparent) r.events = kEventTransmission | kEventTransparent;
    else if (dielectric)
        r.events = (singular ? kEventSingular : kEventGlossy) | (transmission ? kEventTransmission : kEventReflection);
    else if (glossy) r.events = singular ? (kEventSingular | kEventReflection) : (kEventGlossy | kEventReflection);
    else r.events = kEventDiffuse | kEventReflection;
    out.eval = r;
    out.valid = true;
    return out;
}

// AOV visitor (src/luisa/surface_closure_operations.cpp:402-462, contribution :40-161).
struct Aov {
    float3 albedo, normal, transparency;
};
static Aov surface_aov(const SurfaceClosures &s, const ClosurePoint &pt) {
    Aov a{f3(0.0f), pt.shading_normal, f3(0.0f)};
    const float3 incoming = safe_normalize(pt.incoming, pt.shading_normal);
    float total = 0.0f;
    float3 normal = f3(0.0f);
    for (uint32_t i = 0; i < s.count; ++i) {
        const PhysicalClosure &c = s.c[i];
        if (c.op == PSY_CLOSURE_DIFFUSE) {
            a.albedo += c.weight;
            const float w = closure_sample_weight(c.weight);
            normal += c.normal * w;
            total += w;
        } else if (is_glossy(c.op) || is_dielectric(c.op)) {
            // glossy and glass colour are not in the Albedo pass; their
            // corrected normal is in the Normal pass
            const float w = closure_sample_weight(c.weight);
            normal += specular_normal(pt.bump_correction, pt.geometric_normal, incoming, c.normal) * w;
            total += w;
        } else {
            a.transparency += c.weight;
        }
    }
    a.normal = safe_normalize(total > 0.0f ? normal : pt.shading_normal, pt.shading_normal);
    return a;
}

// transparent_extinction (src/luisa/graph_surface_implementation.cpp:354-372).
static float3 transparent_extinction(const Material &mat) {
    std::vector<TracedClosure> traced;
    walk_closures(mat, mat.root, 1.0f, traced, 0);
    float3 r = f3(0.0f);
    for (const auto &t : traced) {
        if (t.op != PSY_CLOSURE_TRANSPARENT) continue;
        if (closure_sample_weight(t.weight) >= 1.0e-5f) r += t.weight;
    }
    return r;
}

static float3 material_emission(const Material &mat) {
    std::vector<TracedClosure> traced;
    walk_closures(mat, mat.root, 1.0f, traced, 0);
    float3 r = f3(0.0f);
    for (const auto &t : traced)
        if (t.op == PSY_CLOSURE_EMISSION) r += t.weight;
    return r;
}

// estimate_surface_emission (src/compiler/surface_program.cpp:244-330):
// bottom-up over the instructions; emission colour x strength, add a + b,
// mix a (1 - f) + b f with the factor as authored; a forward or missing
// operand counts as one.
// Only an unlinked socket of the closure node itself is a literal
// (direct_parameter_value, surface_program.cpp:170-186): a linked colour or
// strength counts as one, and a mix with a linked factor sums its branches.
static float3 emission_estimate(const Material &mat) {
    std::vector<float3> e;
    auto literal = [](uint32_t ref) { return (ref & PSY_INPUT_VALUE) == 0u; };
    for (const psy_closure_instruction &c : mat.code) {
        auto operand = [&](uint32_t id) { return id < e.size() ? e[id] : f3(1.0f); };
        float3 v = f3(0.0f);
        if (c.op == PSY_CLOSURE_EMISSION) {
            const float strength = literal(c.scalar) ? mat.scalars[c.scalar] : 1.0f;
            v = (literal(c.color) ? mat.vectors[c.color] : f3(1.0f)) * strength;
        } else if (c.op == PSY_CLOSURE_ADD) {
            v = operand(c.a) + operand(c.b);
        } else if (c.op == PSY_CLOSURE_MIX) {
            if (literal(c.scalar))
                v = operand(c.a) * (1.0f - mat.scalars[c.scalar]) + operand(c.b) * mat.scalars[c.scalar];
            else
                v = operand(c.a) + operand(c.b);
        }
        e.push_back(v);
    }
    return mat.root < e.size() ? e[mat.root] : f3(0.0f);
}

static bool program_has(const Material &mat, uint32_t op) {
    for (const auto &c : mat.code)
        if (c.op == op) return true;
    return false;
}

// ---------------------------------------------------------- intersection

struct Ray {
    float3 o, d;
    float tmin, tmax;
};

struct Hit {
    bool valid{false};
    float t{0.0f};
    float u{0.0f}, v{0.0f};
    uint32_t instance{kInvalid}, prim{kInvalid}, object{kInvalid}, cycles_prim{kInvalid};
};

struct Identity {
    uint32_t object{kInvalid}, primitive{kInvalid};
};

// clamp_bvh_direction (src/luisa/cycles_triangle_intersection_component.cpp:31-37).
static float clamp_bvh_direction(float v) {
    const float m = 8.271806e-25f;
    return std::fabs(v) > m ? v : std::copysign(m, v);
}

// Pluecker products with the explicit FMA tree
// (cycles_triangle_intersection_component.cpp:13-29).
static float3 pl_cross(float3 a, float3 b) {
    return {std::fma(a.y, b.z, -(a.z * b.y)), std::fma(a.z, b.x, -(a.x * b.z)), std::fma(a.x, b.y, -(a.y * b.x))};
}
static float pl_dot(float3 a, float3 b) { return std::fma(a.x, b.x, std::fma(a.y, b.y, a.z * b.z)); }

struct TriHit {
    bool valid;
    float t, u, v;
};

// PlueckerTriangleIntersectionComponent::intersect
// (cycles_triangle_intersection_component.cpp:39-105); `o`/`d` already in
// the triangle's space with d clamped.
static TriHit intersect_triangle(float3 o, float3 d, float tmin, float tmax, float3 p0, float3 p1, float3 p2) {
    const float3 v0 = p0 - o, v1 = p1 - o, v2 = p2 - o;
    const float3 e0 = v2 - v0, e1 = v0 - v1, e2 = v1 - v2;
    const float u = pl_dot(pl_cross(e0, v2 + v0), d);
    const float v = pl_dot(pl_cross(e1, v0 + v1), d);
    const float w = pl_dot(pl_cross(e2, v1 + v2), d);
    const float sum = u + v + w;
    const float tol = std::numeric_limits<float>::epsilon() * std::fabs(sum);
    const float mn = minf(u, minf(v, w));
    const float mx = maxf(u, maxf(v, w));
    const bool inside = (mn >= -tol) || (mx <= tol);
    const float3 n2 = pl_cross(e1, e0) * 2.0f;
    const float den = pl_dot(n2, d);
    const float safe_den = den != 0.0f ? den : 1.0f;
    const float t = pl_dot(v0, n2) / safe_den;
    const bool in_range = (t >= tmin) && (t <= tmax);
    const float rs = std::fabs(sum) >= 1.0e-18f ? 1.0f / sum : 0.0f;
    return {inside && den != 0.0f && in_range, t, minf(u * rs, 1.0f), minf(v * rs, 1.0f)};
}

// CyclesClosestHitOrder (src/luisa/path_kernel_scene_traversal.cpp:34-66):
// nearest distance, ties to the greatest (object, primitive).
struct ClosestOrder {
    bool has{false};
    float t{0.0f};
    uint32_t object{0}, prim{0};
    bool accepts(float dist, uint32_t obj, uint32_t pr) const {
        const bool later = obj > object || (obj == object && pr > prim);
        return !has || dist < t || (dist == t && later);
    }
};

static bool box_hit(const BvhNode &n, const double o[3], const double inv[3], double tmin, double tmax) {
    double t0 = tmin, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        double ta = (double(n.lo[a]) - o[a]) * inv[a];
        double tb = (double(n.hi[a]) - o[a]) * inv[a];
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
    }
    return t0 <= t1 * (1.0 + 1e-9) + 1e-30;
}

// UnifiedSceneTraversalComponent::trace (path_kernel_scene_traversal.cpp:301-490)
// restated as an exact reduction over every candidate triangle of every
// visible instance; the Luisa Accel only supplied candidates.
static Hit closest_hit(const Scene &s, const Ray &ray, uint32_t visibility, Identity source, Identity light) {
    ClosestOrder order;
    Hit best;
    for (uint32_t i = 0; i < s.instances.size(); ++i) {
        const Instance &inst = s.instances[i];
        if ((inst.visibility & visibility) == 0u) continue;
        const Mesh &m = s.meshes[inst.mesh];
        const float3 o = transform_point(inst.w2o, ray.o);
        const float3 rd = transform_direction(inst.w2o, ray.d);
        const float3 d = {clamp_bvh_direction(rd.x), clamp_bvh_direction(rd.y), clamp_bvh_direction(rd.z)};
        auto test = [&](uint32_t k) {
            const uint32_t cp = m.prim_offset + k;
            const bool excluded = (source.object == i && source.primitive == cp) ||
                                  (light.object == i && light.primitive == cp);
            if (excluded) return;
            const TriHit h = intersect_triangle(o, d, ray.tmin, ray.tmax, m.p[m.idx[3 * k]], m.p[m.idx[3 * k + 1]],
                                                m.p[m.idx[3 * k + 2]]);
            if (!h.valid || !order.accepts(h.t, i, cp)) return;
            order = {true, h.t, i, cp};
            best = {true, h.t, h.u, h.v, i, k, i, cp};
        };
        const uint32_t tri_count = static_cast<uint32_t>(m.idx.size() / 3u);
        if (s.brute_force || m.nodes.empty()) {
            for (uint32_t k = 0; k < tri_count; ++k) test(k);
            continue;
        }
        const double od[3] = {o.x, o.y, o.z};
        const double inv[3] = {1.0 / double(d.x), 1.0 / double(d.y), 1.0 / double(d.z)};
        uint32_t stack[128];
        int sp = 0;
        stack[sp++] = 0u;
        while (sp > 0) {
            const BvhNode &n = m.nodes[stack[--sp]];
            const double tmax = order.has ? double(order.t) : double(ray.tmax);
            if (!box_hit(n, od, inv, double(ray.tmin) - 1e-6 * std::fabs(double(ray.tmin)), tmax * (1.0 + 1e-6) + 1e-30))
                continue;
            if (n.count > 0u) {
                for (uint32_t k = 0; k < n.count; ++k) test(m.order[n.left_or_first + k]);
            } else {
                stack[sp++] = n.left_or_first;
                stack[sp++] = n.left_or_first + 1u;
            }
        }
    }
    return best;
}

// ----------------------------------------------------- surface geometry

struct SurfacePoint {
    float3 position, object_position;
    float3 ng, n;  // world geometric / shading normal, facing the ray
    bool back_facing;
    float3 p0, p1, p2;     // object-space vertices
    float3 wp0, wp1, wp2;  // world-space vertices
    uint32_t instance, material, object, cycles_prim;
};

// triangle_interpolate: (1 - u - v) a + u b + v c.
static float3 tri_interp(float u, float v, float3 a, float3 b, float3 c) {
    return a * (1.0f - u - v) + b * u + c * v;
}

// FinalSupportTriangleSurfaceComponent::resolve for an instanced (not
// transform-applied) mesh (src/luisa/cycles_triangle_surface_component.cpp:9-95).
static SurfacePoint surface_point(const Scene &s, const Hit &h, const Ray &ray) {
    const Instance &inst = s.instances[h.instance];
    const Mesh &m = s.meshes[inst.mesh];
    SurfacePoint sp;
    const uint32_t i0 = m.idx[3 * h.prim], i1 = m.idx[3 * h.prim + 1], i2 = m.idx[3 * h.prim + 2];
    sp.p0 = m.p[i0];
    sp.p1 = m.p[i1];
    sp.p2 = m.p[i2];
    sp.wp0 = transform_point(inst.o2w, sp.p0);
    sp.wp1 = transform_point(inst.o2w, sp.p1);
    sp.wp2 = transform_point(inst.o2w, sp.p2);
    const float3 ogn = safe_normalize(cross(sp.p1 - sp.p0, sp.p2 - sp.p0), f3(0.0f, 0.0f, 1.0f));
    float3 ng = safe_normalize(transform_direction(inst.nrm, ogn), -ray.d);
    const float3 osn = m.smooth ? tri_interp(h.u, h.v, m.n[i0], m.n[i1], m.n[i2]) : ogn;
    float3 n = safe_normalize(transform_direction(inst.nrm, osn), ng);
    sp.back_facing = dot(ng, -ray.d) < 0.0f;
    if (sp.back_facing) {
        ng = -ng;
        n = -n;
    }
    if (dot(n, ng) < 0.0f) n = -n;
    sp.ng = ng;
    sp.n = n;
    sp.object_position = sp.p0 + (sp.p1 - sp.p0) * h.u + (sp.p2 - sp.p0) * h.v;
    sp.position = transform_point(inst.o2w, sp.object_position);
    sp.instance = h.instance;
    sp.material = m.mat.empty() ? inst.material : m.mat[h.prim];
    sp.object = h.object;
    sp.cycles_prim = h.cycles_prim;
    return sp;
}

// Wachter & Binder robust origin offset (Ray Tracing Gems, ch. 6), the
// published method behind Luisa's offset_ray_origin builtin.
static float offset_component(float p, float n) {
    const float origin = 1.0f / 32.0f, float_scale = 1.0f / 65536.0f, int_scale = 256.0f;
    const int32_t of_i = static_cast<int32_t>(int_scale * n);
    int32_t bits;
    std::memcpy(&bits, &p, 4);
    bits += p < 0.0f ? -of_i : of_i;
    float p_i;
    std::memcpy(&p_i, &bits, 4);
    return std::fabs(p) < origin ? p + float_scale * n : p_i;
}
static float3 offset_ray_origin(float3 p, float3 n) {
    return {offset_component(p.x, n.x), offset_component(p.y, n.y), offset_component(p.z, n.z)};
}

// source_triangle_covers_ray_origin / origin_with_explicit_self_exclusion
// (include/psycles/luisa/surface_ray.h:49-100).
static float3 origin_with_self_exclusion(const SurfacePoint &sp, float3 object_origin, float3 object_direction) {
    const float3 v0 = sp.p0 - object_origin, v1 = sp.p1 - object_origin, v2 = sp.p2 - object_origin;
    const float3 e0 = v2 - v0, e1 = v0 - v1, e2 = v1 - v2;
    const float u = dot(cross(v2 + v0, e0), object_direction);
    const float v = dot(cross(v0 + v1, e1), object_direction);
    const float w = dot(cross(v1 + v2, e2), object_direction);
    const float eps = std::numeric_limits<float>::epsilon() * std::fabs(u + v + w);
    const float mn = minf(u, minf(v, w)), mx = maxf(u, maxf(v, w));
    const bool exact = (mn >= eps) || (mx <= -eps);
    return exact ? sp.position : offset_ray_origin(sp.position, sp.ng);
}

// SurfaceGeometryContext::make_ray_origin (src/luisa/path_kernel_surface_geometry.cpp:151-166)
// and make_shadow_origin with a zero shadow-terminator offset (:168-185).
static float3 surface_ray_origin(const Scene &s, const SurfacePoint &sp, float3 direction) {
    const Instance &inst = s.instances[sp.instance];
    return origin_with_self_exclusion(sp, sp.object_position, transform_direction(inst.w2o, direction));
}
static float3 surface_shadow_origin(const Scene &s, const SurfacePoint &sp, float3 direction) {
    const Instance &inst = s.instances[sp.instance];
    const float3 oo = transform_point(inst.w2o, sp.position);
    const float3 od = transform_direction(inst.w2o, direction);
    return origin_with_self_exclusion(sp, oo, od);
}

// ------------------------------------------------------- light sampling

// make_light_distribution_sample_callable (src/luisa/path_tracer_light_distribution.cpp:8-52).
static DistEntry distribution_sample(const Scene &s, float u) {
    if (s.emitter_count == 0u) return {0.0f, 0.0f, kKindSentinel, 0u};
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
    selected = std::min(selected, s.emitter_count - 1u);
    return s.distribution[selected];
}

// spherical_geometry.h:96-205 (solid angle, strategy predicate, low
// distortion map, directional pdf) and sample_triangle :207-283.
static float triangle_solid_angle(float3 r, float3 p0, float3 p1, float3 p2) {
    const float3 a = normalize_or(p0 - r, f3(1.0f, 0.0f, 0.0f));
    const float3 b = normalize_or(p1 - r, f3(0.0f, 1.0f, 0.0f));
    const float3 c = normalize_or(p2 - r, f3(0.0f, 0.0f, 1.0f));
    const float num = std::fabs(dot(a, cross(b, c)));
    const float den = 1.0f + dot(a, b) + dot(b, c) + dot(c, a);
    return 2.0f * atan2_(num, den);
}
static bool use_solid_angle(float3 r, float3 p0, float3 p1, float3 p2) {
    const float3 e0 = p1 - p0, e1 = p2 - p0, e2 = p2 - p1;
    const float longest = maxf(dot(e0, e0), maxf(dot(e1, e1), dot(e2, e2)));
    const float3 un = cross(e0, e1);
    const float nl2 = dot(un, un);
    const float safe = maxf(nl2, 1.0e-20f);
    const float dist = dot(un, p0 - r) / safe;
    return nl2 > 1.0e-20f && longest > dist * dist;
}
static float2 low_distortion_barycentric(float2 r) {
    const float x = clampf(r.x, 0.0f, 1.0f), y = clampf(r.y, 0.0f, 1.0f);
    if (y > x) {
        const float u = 0.5f * x;
        return {u, y - u};
    }
    const float v = 0.5f * y;
    return {x - v, v};
}
struct TriPdf {
    float value;
    bool valid;
};
static TriPdf triangle_directional_pdf(float3 r, float3 lp, float3 p0, float3 p1, float3 p2) {
    const float3 e0 = p1 - p0, e1 = p2 - p0;
    const float3 un = cross(e0, e1);
    const float da = std::sqrt(maxf(dot(un, un), 0.0f));
    const float area = 0.5f * da;
    const float3 nrm = un / maxf(da, 1.0e-20f);
    const float3 off = lp - r;
    const float d2 = dot(off, off);
    const float3 dir = off / std::sqrt(maxf(d2, 1.0e-20f));
    const float cosine = std::fabs(dot(nrm, -dir));
    const bool sa = use_solid_angle(r, p0, p1, p2);
    const float solid = triangle_solid_angle(r, p0, p1, p2);
    const float area_pdf = d2 / maxf(cosine * area, 1.0e-20f);
    const float sa_pdf = 1.0f / maxf(solid, 1.0e-20f);
    const bool valid_area = area > 0.0f && d2 > 1.0e-12f && cosine > 0.0f;
    const bool valid_sa = valid_area && solid > 0.0f;
    return {sa ? sa_pdf : area_pdf, sa ? valid_sa : valid_area};
}
struct TriSample {
    float3 position, direction;
    float distance, pdf;
    bool valid;
};
static TriSample sample_triangle(float3 r, float3 p0, float3 p1, float3 p2, float2 rnd) {
    const float2 ab = low_distortion_barycentric(rnd);
    const float3 area_position = p0 * (1.0f - ab.x - ab.y) + p1 * ab.x + p2 * ab.y;
    const float3 area_offset = area_position - r;
    const float area_d2 = dot(area_offset, area_offset);
    const float area_distance = std::sqrt(maxf(area_d2, 1.0e-20f));
    const float3 area_direction = area_offset / area_distance;
    const float3 a = normalize_or(p0 - r, f3(1.0f, 0.0f, 0.0f));
    const float3 b = normalize_or(p1 - r, f3(0.0f, 1.0f, 0.0f));
    const float3 c = normalize_or(p2 - r, f3(0.0f, 0.0f, 1.0f));
    const float cos_b = clampf(dot(a, c), -1.0f, 1.0f);
    const float cos_c = clampf(dot(a, b), -1.0f, 1.0f);
    const float solid = triangle_solid_angle(r, p0, p1, p2);
    const float3 ab_n = normalize_or(cross(a, b), f3(1.0f, 0.0f, 0.0f));
    const float3 ac_n = normalize_or(cross(a, c), f3(0.0f, 1.0f, 0.0f));
    const float cos_alpha = clampf(dot(ab_n, ac_n), -1.0f, 1.0f);
    const float sin_alpha = std::sqrt(maxf(1.0f - cos_alpha * cos_alpha, 0.0f));
    const float alpha = acos_(cos_alpha);
    const float phi = clampf(rnd.x, 0.0f, 1.0f) * solid - alpha;
    const float sin_phi = sin_(phi), cos_phi = cos_(phi);
    const float u = cos_phi - cos_alpha;
    const float v = sin_phi + sin_alpha * cos_c;
    const float num = (v * cos_phi - u * sin_phi) * cos_alpha - v;
    const float den = (v * sin_phi + u * cos_phi) * sin_alpha;
    const float safe_den = std::fabs(den) > 1.0e-20f ? den : (den >= 0.0f ? 1.0e-20f : -1.0e-20f);
    const float q = std::fabs(den) <= 1.0e-20f ? 1.0f : num / safe_den;
    const float3 tangent = normalize_or(c - a * cos_b, f3(0.0f, 1.0f, 0.0f));
    const float3 c_prime = normalize_or(a * clampf(q, -1.0f, 1.0f) + tangent * std::sqrt(maxf(1.0f - q * q, 0.0f)), a);
    const float z = 1.0f - clampf(rnd.y, 0.0f, 1.0f) * (1.0f - dot(c_prime, b));
    const float3 edge_dir = normalize_or(c_prime - b * dot(c_prime, b), a);
    const float3 solid_dir = normalize_or(b * z + edge_dir * std::sqrt(maxf(1.0f - z * z, 0.0f)), b);
    const float3 e01 = p1 - p0, e02 = p2 - p0;
    const float3 pv = cross(solid_dir, e02);
    const float det = dot(e01, pv);
    const float safe_det = std::fabs(det) > 1.0e-20f ? det : (det >= 0.0f ? 1.0e-20f : -1.0e-20f);
    const float inv_det = 1.0f / safe_det;
    const float3 tv = r - p0;
    const float su = dot(tv, pv) * inv_det;
    const float3 qv = cross(tv, e01);
    const float sv = dot(solid_dir, qv) * inv_det;
    const float sd = dot(e02, qv) * inv_det;
    const float3 solid_position = r + solid_dir * sd;
    const bool solid_valid = std::fabs(det) > 1.0e-20f && sd > 0.0f && su >= -1.0e-5f && sv >= -1.0e-5f &&
                             su + sv <= 1.0f + 1.0e-5f && solid > 0.0f;
    const bool sa = use_solid_angle(r, p0, p1, p2);
    const float3 position = sa ? solid_position : area_position;
    const TriPdf pdf = triangle_directional_pdf(r, position, p0, p1, p2);
    TriSample out;
    out.position = position;
    out.direction = sa ? solid_dir : area_direction;
    out.distance = sa ? sd : area_distance;
    out.pdf = pdf.value;
    out.valid = pdf.valid && (sa ? solid_valid : area_d2 > 1.0e-12f);
    return out;
}

// samples_front / samples_back / sampled_side
// (src/luisa/path_kernel_emissive_triangle.cpp:26-70).
static bool samples_front(uint32_t m) { return m == 1u || m == 2u || m == 4u; }
static bool samples_back(uint32_t m) { return m == 1u || m == 3u || m == 4u; }
static bool sampled_side(uint32_t m, float3 ng, float3 dir) {
    const bool back = dot(ng, -dir) < 0.0f;
    return back ? samples_back(m) : samples_front(m);
}

// Forward-hit pdf of an emissive triangle (from_intersection,
// path_kernel_emissive_triangle.cpp:589-646).
static float emissive_forward_pdf(float selection_pdf, uint32_t sampling, float3 reference, float3 lp, float3 p0,
                                  float3 p1, float3 p2, float3 oriented_ng) {
    const TriPdf pdf = triangle_directional_pdf(reference, lp, p0, p1, p2);
    const float3 dir = normalize_or(lp - reference, f3(0.0f, 0.0f, 1.0f));
    const bool side = sampled_side(sampling, oriented_ng, dir);
    const float area = 0.5f * length(cross(p1 - p0, p2 - p0));
    const float value = pdf.value * selection_pdf;
    const bool valid = sampling != 0u && side && pdf.valid && area > 0.0f && value > 0.0f;
    return valid ? value : 0.0f;
}

// Analytic light sampling, include/psycles/luisa/analytic_light_sampling.h.
struct AnalyticSample {
    bool valid;
    float3 direction, position;
    float distance, pdf, eval_factor;
};

static float point_eval_factor(float radius, bool normalize_power) {  // :880-896
    const float r2 = radius * radius;
    const float area = r2 > 0.0f ? 4.0f * kPi * r2 : 4.0f;
    const float inv = normalize_power ? 1.0f / maxf(area, 1.0e-20f) : 1.0f;
    return inv * kInvPi;
}
static float point_disk_pdf(float d2, float cosine, float radius) {  // :856-873
    const float r2 = radius * radius;
    const float inv_area = r2 > 0.0f ? 1.0f / maxf(r2 * kPi, 1.0e-20f) : 1.0f;
    return cosine > 0.0f ? inv_area * d2 / cosine : 0.0f;
}
// sample_disk_geometry (:549-603).
static AnalyticSample sample_disk(float3 r, float3 center, float radius, float2 rnd) {
    float3 ln = r - center;
    const float cd2 = dot(ln, ln);
    const float cd = std::sqrt(maxf(cd2, 1.0e-30f));
    ln = ln / cd;
    const Basis b = make_orthonormals(ln);
    const float2 disk = sample_uniform_disk(rnd);
    const float3 position = center + (b.tangent * disk.x + b.bitangent * disk.y) * radius;
    const float3 off = position - r;
    const float d2 = dot(off, off);
    const float dist = std::sqrt(maxf(d2, 1.0e-30f));
    const float3 dir = off / dist;
    const float cosine = dot(ln, -dir);
    return {cd2 > 0.0f && cosine > 0.0f, dir, position, dist, point_disk_pdf(d2, cosine, radius), 0.0f};
}
// spot_light_attenuation and light_linear_transform (:137-166, :309-345).
static float spot_attenuation(const psy_light_desc &l, float3 dir_from_light) {
    const float3 ax = f3(l.axis_x[0], l.axis_x[1], l.axis_x[2]) * l.axis_scale[0];
    const float3 ay = f3(l.axis_y[0], l.axis_y[1], l.axis_y[2]) * l.axis_scale[1];
    const float3 az = f3(l.axis_z[0], l.axis_z[1], l.axis_z[2]) * l.axis_scale[2];
    const float3 adj_x = cross(ay, az);
    const float det = dot(ax, adj_x);
    const bool valid = std::fabs(det) > 1.0e-20f;
    const float inv_det = 1.0f / (valid ? det : 1.0f);
    const float3 rx = adj_x * inv_det, ry = cross(az, ax) * inv_det, rz = cross(ax, ay) * inv_det;
    float3 local = light_safe_normalize(f3(dot(rx, dir_from_light), dot(ry, dir_from_light), dot(rz, dir_from_light)),
                                        f3(0.0f, 0.0f, -1.0f));
    local.z = -local.z;
    const float cos_half = cos_(0.5f * l.spot_angle);
    const float blend = (1.0f - cos_half) * l.spot_smooth;
    const float ratio = blend != 0.0f ? (local.z - cos_half) / blend : 0.0f;
    const float lin = clampf(ratio, 0.0f, 1.0f);
    const float smooth = lin * lin * (3.0f - 2.0f * lin);
    const float hard = local.z >= cos_half ? 1.0f : 0.0f;
    return blend > 0.0f ? smooth : hard;
}
// sample_distant_light (:84-108).
static AnalyticSample sample_distant(const psy_light_desc &l, float2 rnd) {
    const float3 az = f3(l.axis_z[0], l.axis_z[1], l.axis_z[2]);
    const float half_angle = 0.5f * maxf(l.angle, 0.0f);
    const float sq = sin_(0.5f * half_angle);
    const float omc = 2.0f * sq * sq;
    const ConeSample c = sample_uniform_cone(-az, omc, rnd);
    const bool finite = half_angle > 0.0f;
    const float sh = sin_(half_angle);
    const float disk_area = kPi * sh * sh;
    const bool normalize_power = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    const float eval = (normalize_power && finite) ? 1.0f / maxf(disk_area, 1.0e-20f) : 1.0f;
    const float3 dir = -c.direction;
    return {true, dir, -dir, 1.0e30f, c.pdf, eval};
}
// spot_one_minus_cosine_larger_spread (:355-376), with 1/sqrt for rsqrt.
static float spot_spread_cap(const psy_light_desc &l) {
    const float t = tan_(0.5f * l.spot_angle);
    const float ts2 = maxf(l.axis_scale[0] * l.axis_scale[0], l.axis_scale[1] * l.axis_scale[1]);
    const float as2 = l.axis_scale[2] * l.axis_scale[2];
    return 1.0f - 1.0f / std::sqrt(1.0f + t * t * ts2 / maxf(as2, 1.0e-30f));
}

struct SphereHit {
    bool valid;
    float distance;
    float3 position;
};

// intersect_sphere (:192-239).
static SphereHit intersect_sphere(float3 o, float3 d, float tmin, float tmax, float3 c, float r) {
    const float3 co = c - o;
    const float r2 = r * r;
    const float cd2 = dot(co, co);
    const float pd = dot(co, d);
    const float3 perp = co - d * pd;
    const float pp2 = dot(perp, perp);
    const float dist = pd - std::copysign(std::sqrt(maxf(r2 - pp2, 0.0f)), cd2 - r2);
    const bool valid = !(cd2 > r2 && pd < 0.0f) && pp2 <= r2 && dist > tmin && dist < tmax;
    return {valid, dist, o + d * dist};
}

// sample_uniform_sphere (cycles_sample_mapping.h:380-387).
static float3 sample_uniform_sphere(float2 u) {
    const float z = 1.0f - 2.0f * u.x;
    const float r = std::sqrt(maxf(1.0f - z * z, 0.0f));
    const float phi = 2.0f * kPi * u.y;
    return f3(r * cos_(phi), r * sin_(phi), z);
}

// sample_sphere_geometry (:430-548).
static AnalyticSample sample_sphere(float3 reference, float3 n, bool transmission, float3 center, float r,
                                    float3 outside_axis, float outside_omc, bool intersect_sampled, float2 rnd) {
    const float r2 = r * r;
    float3 ln = reference - center;
    const float cd2 = dot(ln, ln);
    const float cd = std::sqrt(maxf(cd2, 1.0e-30f));
    ln = ln / cd;
    float3 dir = f3(0.0f);
    float cosine = 1.0f, pdf = 0.0f, dist = 0.0f;
    float3 pos = reference;
    bool known = false;
    bool valid = r > 0.0f && cd2 > 0.0f;
    if (cd2 > r2) {
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
            const HemisphereSample hs = sample_cosine_hemisphere(n, rnd);
            dir = hs.direction;
            pdf = hs.pdf;
        }
        cosine = -dot(dir, ln);
    }
    if (!known) {
        dist = cd * cosine - std::copysign(std::sqrt(maxf(r2 - cd2 + cd2 * cosine * cosine, 0.0f)), cd2 - r2);
        pos = reference + dir * dist;
    }
    const float3 normal = light_safe_normalize(pos - center, -dir);
    return {valid, dir, normal * r + center, dist, pdf, 0.0f};
}

// sample_point_light / sample_spot_light (:898-1105): delta, disk and
// sphere sources.
static AnalyticSample sample_point_or_spot(const psy_light_desc &l, float3 reference, float3 shading_n,
                                           bool transmission, float2 rnd) {
    const float3 center = f3(l.position[0], l.position[1], l.position[2]);
    const bool normalize_power = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    if ((l.flags & PSY_LIGHT_FLAG_SPHERE) != 0u && l.radius > 0.0f) {
        const float3 off = reference - center;
        const float cd2 = dot(off, off);
        const float r2 = l.radius * l.radius;
        const float3 ln = light_safe_normalize(off, f3(0.0f, 0.0f, -1.0f));
        const float sphere_cap = sin_squared_to_one_minus_cosine(r2 / maxf(cd2, 1.0e-30f));
        float3 axis = -ln;
        float cap = sphere_cap;
        bool spread = false;
        if (l.type == PSY_LIGHT_SPOT) {
            const float spot_cap = spot_spread_cap(l);
            spread = cd2 > r2 && !(sphere_cap < spot_cap);
            if (spread) {
                axis = f3(l.axis_z[0], l.axis_z[1], l.axis_z[2]);
                cap = spot_cap;
            }
        }
        AnalyticSample g = sample_sphere(reference, shading_n, transmission, center, l.radius, axis, cap, spread, rnd);
        float eval = point_eval_factor(l.radius, normalize_power);
        if (l.type == PSY_LIGHT_SPOT && cd2 > r2) eval *= spot_attenuation(l, -g.direction);
        g.eval_factor = eval;
        if (l.type == PSY_LIGHT_SPOT) g.valid = g.valid && eval != 0.0f;
        return g;
    }
    AnalyticSample g = sample_disk(reference, center, l.radius, rnd);
    float eval = point_eval_factor(l.radius, normalize_power);
    if (l.type == PSY_LIGHT_SPOT) eval *= spot_attenuation(l, -g.direction);
    g.eval_factor = eval;
    g.valid = g.valid && eval != 0.0f;
    return g;
}

// Area lights with full spread: rectangle_solid_angle_context /
// sample_rectangle_solid_angle (analytic_light_sampling.h:605-793) and
// AreaLightSampling::from_position (src/luisa/area_light_sampling.cpp:494-642).
static float safe_div(float a, float b) { return b != 0.0f ? a / b : 0.0f; }
static AnalyticSample sample_area(const psy_light_desc &l, float3 reference, float2 rnd) {
    AnalyticSample out{false, f3(0.0f), f3(l.position[0], l.position[1], l.position[2]), 0.0f, 0.0f, 0.0f};
    const float3 center = f3(l.position[0], l.position[1], l.position[2]);
    const float3 au = f3(l.axis_x[0], l.axis_x[1], l.axis_x[2]);
    const float3 av = f3(l.axis_y[0], l.axis_y[1], l.axis_y[2]);
    const float3 az = f3(l.axis_z[0], l.axis_z[1], l.axis_z[2]);
    const float lu = l.size_u, lv = l.size_v;
    const bool ellipse = (l.flags & PSY_LIGHT_FLAG_ELLIPSE) != 0u;
    const float3 normal = -az;
    if (!(dot(center - reference, normal) <= 0.0f)) return out;
    float3 position = center;
    float pdf = 0.0f;
    if (!ellipse) {
        float3 z = cross(au, av);
        const float3 co = center - reference;
        float z0 = dot(co, z);
        if (z0 > 0.0f) {
            z = -z;
            z0 = -z0;
        }
        const float cu = dot(co, au), cv = dot(co, av);
        const float x0 = cu - 0.5f * lu, x1 = cu + 0.5f * lu, y0 = cv - 0.5f * lv, y1 = cv + 0.5f * lv;
        float e[4] = {-y0, x1, y1, -x0};
        for (float &v : e) v = v / std::sqrt(v * v + z0 * z0);
        float g[4];
        for (int k = 0; k < 4; ++k) g[k] = asin_(clampf(-e[k] * e[(k + 1) & 3], -1.0f, 1.0f));
        const float solid = -(g[0] + g[1] + g[2] + g[3]);
        const float min_e2 = minf(minf(e[0] * e[0], e[1] * e[1]), minf(e[2] * e[2], e[3] * e[3]));
        const float cd = length(co);
        const float planar = safe_div(-(cd * cd * cd), z0 * lu * lv);
        pdf = (solid < 1.0e-5f || min_e2 > 0.99999f) ? planar : 1.0f / solid;
        const float b0 = e[0], b1 = e[2];
        const float alpha = rnd.x * solid + g[2] + g[3];
        const float fu = safe_div(cos_(alpha) * b0 + b1, sin_(alpha));
        float cos_u = std::copysign(1.0f / std::sqrt(fu * fu + b0 * b0), fu);
        cos_u = clampf(cos_u, -1.0f, 1.0f);
        float su = -(cos_u * z0) / maxf(std::sqrt(maxf(1.0f - cos_u * cos_u, 0.0f)), 1.0e-7f);
        su = clampf(su, x0, x1);
        const float du2 = su * su + z0 * z0;
        const float h0 = y0 / std::sqrt(du2 + y0 * y0);
        const float h1 = y1 / std::sqrt(du2 + y1 * y1);
        const float hv = h0 + rnd.y * (h1 - h0);
        const float hv2 = hv * hv;
        const float sv = hv2 < 1.0f - 1.0e-6f ? hv * std::sqrt(du2 / (1.0f - hv2)) : y1;
        position = reference + au * su + av * sv + z * z0;
    } else {
        const float2 disk = sample_uniform_disk(rnd);
        position = center + au * (0.5f * lu * disk.x) + av * (0.5f * lv * disk.y);
        pdf = 4.0f * kInvPi / (lu * lv);
    }
    const float3 off = position - reference;
    const float d2 = dot(off, off);
    const float dist = std::sqrt(maxf(d2, 0.0f));
    const float3 dir = off / maxf(dist, 1.0e-30f);
    if (ellipse) {
        const float cosine = dot(normal, -dir);
        pdf *= cosine > 0.0f ? d2 / cosine : 0.0f;
    }
    float area = lu * lv;
    if (ellipse) area *= 0.25f * kPi;
    const bool normalize_power = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    const float inv_area = (normalize_power && area != 0.0f) ? safe_div(1.0f, area) : 1.0f;
    const float factor = kInvPi * inv_area * 1.0f;
    const float3 inplane = position - center;
    const float u = dot(inplane, au), v = dot(inplane, av);
    const float eu = (0.5f + 1.0e-7f) * lu + 1.0e-6f, ev = (0.5f + 1.0e-7f) * lv + 1.0e-6f;
    const bool inside = ellipse ? (u * u / (eu * eu) + v * v / (ev * ev) <= 1.0f)
                                : (std::fabs(u) <= eu && std::fabs(v) <= ev);
    out.valid = inside && factor > 0.0f;
    out.direction = dir;
    out.position = position;
    out.distance = dist;
    out.pdf = pdf;
    out.eval_factor = factor;
    return out;
}

// Derived light flags (path_tracer_scene.cpp:1787-1830): effective use_mis
// (lamps with a finite extent) and forward intersectability.
constexpr uint32_t kLightUseMis = 1u << 30, kLightForward = 1u << 31;

// rectangle_solid_angle_context(...).pdf (analytic_light_sampling.h): the
// directional pdf of the spherical rectangle, planar limit for tiny or
// grazing rectangles.
static float rectangle_pdf(float3 reference, float3 center, float3 au, float lu, float3 av, float lv) {
    const float3 co = center - reference;
    float z0 = dot(co, cross(au, av));
    if (z0 > 0.0f) z0 = -z0;
    const float cu = dot(co, au), cv = dot(co, av);
    const float x0 = cu - 0.5f * lu, x1 = cu + 0.5f * lu, y0 = cv - 0.5f * lv, y1 = cv + 0.5f * lv;
    float e[4] = {-y0, x1, y1, -x0};
    for (float &v : e) v = v / std::sqrt(v * v + z0 * z0);
    float angles[4];
    for (int k = 0; k < 4; ++k) angles[k] = asin_(clampf(-e[k] * e[(k + 1) & 3], -1.0f, 1.0f));
    const float solid = -(angles[0] + angles[1] + angles[2] + angles[3]);
    const float min_e2 = minf(minf(e[0] * e[0], e[1] * e[1]), minf(e[2] * e[2], e[3] * e[3]));
    const float cd = length(co);
    const float planar = safe_div(-(cd * cd * cd), z0 * lu * lv);
    return (solid < 1.0e-5f || min_e2 > 0.99999f) ? planar : 1.0f / solid;
}

struct LampHit {
    bool valid;
    uint32_t index;
    float distance, pdf, eval_factor;
};

// intersect_area (analytic_light_intersection.h:268-353) with the pdf and
// factor of AreaLightSampling::from_intersection (area_light_sampling.cpp:644-727)
// at full spread: front side, strictly inside (tmin, tmax).
static bool lamp_area(const psy_light_desc &l, const Ray &ray, float tmin, float tmax, LampHit &out) {
    const float3 center = f3(l.position[0], l.position[1], l.position[2]);
    const float3 au = f3(l.axis_x[0], l.axis_x[1], l.axis_x[2]);
    const float3 av = f3(l.axis_y[0], l.axis_y[1], l.axis_y[2]);
    const float3 normal = -f3(l.axis_z[0], l.axis_z[1], l.axis_z[2]);
    const bool ellipse = (l.flags & PSY_LIGHT_FLAG_ELLIPSE) != 0u;
    const float denom = dot(ray.d, normal);
    const float t = safe_div(dot(center - ray.o, normal), denom);
    const float3 inplane = (ray.o + ray.d * t) - center;
    const float u = safe_div(dot(inplane, au), l.size_u);
    const float v = safe_div(dot(inplane, av), l.size_v);
    bool inside = u >= -0.5f && u <= 0.5f && v >= -0.5f && v <= 0.5f;
    if (ellipse) inside = inside && u * u + v * v <= 0.25f;
    if (!(denom < 0.0f && t > tmin && t < tmax && inside)) return false;
    float pdf;
    if (ellipse) {
        const float cosine = dot(normal, -ray.d);
        pdf = 4.0f * kInvPi / (l.size_u * l.size_v) * (cosine > 0.0f ? t * t / cosine : 0.0f);
    } else {
        pdf = rectangle_pdf(ray.o, center, au, l.size_u, av, l.size_v);
    }
    float area = l.size_u * l.size_v;
    if (ellipse) area *= 0.25f * kPi;
    const bool normalize_power = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    const float eval = kInvPi * ((normalize_power && area != 0.0f) ? safe_div(1.0f, area) : 1.0f) * 1.0f;
    if (!(area > 0.0f && eval > 0.0f)) return false;
    out = {true, 0u, t, pdf, eval};
    return true;
}

// intersect_point / intersect_spot, oriented-disk case (analytic_light_intersection.h:33-266):
// the disk of `radius` faces the ray origin.
static bool lamp_disk(const psy_light_desc &l, const Ray &ray, float tmin, float tmax, float3 mis_n,
                      bool had_transmission, LampHit &out) {
    const float3 center = f3(l.position[0], l.position[1], l.position[2]);
    const float3 offset = ray.o - center;
    if ((l.flags & PSY_LIGHT_FLAG_SPHERE) != 0u) {
        // sphere geometry with sphere_light_pdf (analytic_light_sampling.h:282-307)
        if (!(l.radius > 0.0f)) return false;
        const float cd2 = dot(offset, offset);
        const float r2 = l.radius * l.radius;
        float cap = sin_squared_to_one_minus_cosine(r2 / maxf(cd2, 1.0e-30f));
        if (l.type == PSY_LIGHT_SPOT) cap = minf(cap, spot_spread_cap(l));
        const SphereHit h = intersect_sphere(ray.o, ray.d, tmin, tmax, center, l.radius);
        if (!h.valid) return false;
        float pdf;
        if (cd2 > r2) {
            pdf = kInvTwoPi / maxf(cap, 1.0e-30f);
        } else if (had_transmission) {
            pdf = 0.5f * kInvTwoPi;
        } else {
            const float c = dot(mis_n, ray.d);
            pdf = c > 0.0f ? c * kInvPi : 0.0f;
        }
        float eval = point_eval_factor(l.radius, (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u);
        if (l.type == PSY_LIGHT_SPOT) {
            if (cd2 > r2) eval *= spot_attenuation(l, -ray.d);
            if (!(dot(ray.d, offset) < 0.0f)) return false;
        }
        if (!(eval > 0.0f)) return false;
        out = {true, 0u, h.distance, pdf, eval};
        return true;
    }
    const float3 n = light_safe_normalize(offset, -ray.d);
    const float plane = dot(offset, n);
    const float cosine = dot(n, -ray.d);
    const float t = safe_div(plane, cosine);
    const float3 radial = (ray.o + ray.d * t) - center;
    const bool hit = plane * cosine > 0.0f && t >= 0.0f && dot(radial, radial) < l.radius * l.radius && t > tmin &&
                     t < tmax && l.radius > 0.0f;
    if (!hit) return false;
    float eval = point_eval_factor(l.radius, (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u);
    if (l.type == PSY_LIGHT_SPOT) {
        eval *= spot_attenuation(l, -ray.d);
        if (!(dot(ray.d, offset) < 0.0f)) return false;
    }
    if (!(eval > 0.0f)) return false;
    out = {true, 0u, t, point_disk_pdf(t * t, cosine, l.radius), eval};
    return true;
}

// ClosestEventStageImpl's lamp loop (src/luisa/path_kernel_closest_event.cpp:56-230):
// the nearest eligible lamp strictly before `event_distance`, ties to the
// lower index.
static LampHit closest_lamp(const Scene &s, const Ray &ray, float tmin, float event_distance, uint32_t ray_visibility,
                            uint32_t excluded, float3 mis_n, bool had_transmission) {
    LampHit best{false, kInvalid, event_distance, 0.0f, 0.0f};
    const bool camera_path = (ray_visibility & PSY_VISIBILITY_CAMERA) != 0u;
    for (uint32_t i = 0; i < s.lights.size(); ++i) {
        const psy_light_desc &l = s.lights[i];
        if (l.type == PSY_LIGHT_DISTANT || i == excluded) continue;
        if ((l.visibility & ray_visibility) == 0u) continue;
        if (!camera_path && (l.flags & kLightUseMis) == 0u) continue;
        LampHit h{};
        const bool ok = l.type == PSY_LIGHT_AREA ? lamp_area(l, ray, tmin, best.distance, h)
                                                 : lamp_disk(l, ray, tmin, best.distance, mis_n, had_transmission, h);
        if (ok) {
            best = h;
            best.index = i;
        }
    }
    return best;
}

// --------------------------------------------------------------- shadow

// make_trace_shadow_callable (src/luisa/path_tracer_geometry.cpp:75-174):
// iterated closest hits; transparent surfaces multiply their extinction and
// advance tmin by one ULP, opaque ones stop the ray.
static float3 trace_shadow(const Scene &s, Ray ray, Identity source, Identity light, uint32_t transparent_depth,
                           uint32_t transparent_max) {
    float3 transmittance = f3(1.0f);
    for (int guard = 0; guard < 4096; ++guard) {
        const Hit h = closest_hit(s, ray, PSY_VISIBILITY_SHADOW, source, light);
        if (!h.valid) return transmittance;
        if (transparent_depth >= transparent_max) return f3(0.0f);
        const Instance &inst = s.instances[h.instance];
        const Mesh &m = s.meshes[inst.mesh];
        const Material &mat = s.materials[m.mat.empty() ? inst.material : m.mat[h.prim]];
        const float3 t = clamp3(transparent_extinction(mat), 0.0f, 1.0f);
        if (!(max_component(t) > 0.0f)) return f3(0.0f);
        transmittance *= t;
        transparent_depth += 1u;
        const uint32_t next = float_bits(h.t) + 1u;
        ray.tmin = h.t == 0.0f ? std::numeric_limits<float>::min() : bits_float(next);
    }
    return f3(0.0f);
}

// -------------------------------------------------------------- integrator

struct Settings {
    psy_render_settings raw;
    uint32_t maximum, minimum, max_diffuse, max_glossy, max_transmission, transparent_min, transparent_max, steps;
    float inv_rr_threshold;
    bool use_light_tree;
    float htan, vtan, shift_x, shift_y;
    float ortho_span;     // orthographic_viewplane_span().vertical
    bool depth_of_field;  // perspective with aperture and focal distance
    std::array<float, 1024> filter;
    SobolTable sobol;
};

// cycles_kernel_bounce_limits (src/luisa/cycles_integrator_limits.h:62-85)
// and the camera parameters of path_tracer_kernel.cpp:189-280.
static void derive_settings(Settings &st, const Scene &s, const psy_render_settings &r, uint32_t total) {
    st.raw = r;
    auto synced = [](uint32_t v) { return v == 0xffffffffu ? v : v + 1u; };
    st.maximum = synced(r.max_bounces);
    st.minimum = synced(r.min_bounces);
    st.max_diffuse = synced(r.diffuse_bounces);
    st.max_glossy = synced(r.glossy_bounces);
    st.max_transmission = synced(r.transmission_bounces);
    st.transparent_min = synced(r.transparent_min_bounces);
    st.transparent_max = r.transparent_max_bounces;
    const uint64_t required = 2ull * st.maximum + std::max(st.transparent_max, 1u) + 1ull;
    st.steps = static_cast<uint32_t>(std::min<uint64_t>(required, 1024ull));
    st.inv_rr_threshold = (!r.use_light_tree && r.light_sampling_threshold > 0.0f)
                              ? r.film_exposure / r.light_sampling_threshold : 0.0f;
    // path_tracer_kernel.cpp:206-209: the tree is used only when it exists
    st.use_light_tree = r.use_light_tree != 0u && s.tree_usable;
    const float aspect = static_cast<float>(std::max(r.full_width, 1u)) / static_cast<float>(std::max(r.full_height, 1u));
    const bool hfit = s.camera.sensor_fit == 1u || (s.camera.sensor_fit == 0u && aspect >= 1.0f);
    st.vtan = hfit ? std::tan(s.camera.horizontal_field_of_view * 0.5f) / aspect
                   : std::tan(s.camera.field_of_view * 0.5f);
    st.htan = st.vtan * aspect;
    st.shift_x = s.camera.lens_shift_x * (hfit ? 1.0f : 1.0f / aspect);
    st.shift_y = s.camera.lens_shift_y * (hfit ? aspect : 1.0f);
    // camera_sampling.h:47-53 and path_tracer_kernel.cpp:275-278
    st.ortho_span = hfit ? s.camera.orthographic_scale / aspect : s.camera.orthographic_scale;
    st.depth_of_field = s.camera.projection == PSY_CAMERA_PERSPECTIVE && s.camera.aperture_radius > 0.0f &&
                        s.camera.focal_distance > 0.0f;
    st.filter = pixel_filter_table(r.pixel_filter, r.filter_width);
    st.sobol.sequence_size = sobol_sequence_size_for_samples(total);
    st.sobol.rows = sobol_generate_table(st.sobol.sequence_size);
}

static float power_heuristic(float a, float b) {
    const float a2 = a * a, b2 = b * b;
    return a2 / maxf(a2 + b2, 1.0e-20f);
}

// forward_light_weight / nee_light_weight (src/luisa/path_tracer_lighting.cpp:35-72).
static float forward_light_weight(uint32_t mode, float forward_pdf, float nee_pdf, bool competing, bool available) {
    if (mode == PSY_DIRECT_LIGHT_FORWARD) return 1.0f;
    if (mode == PSY_DIRECT_LIGHT_NEE) return (competing && available) ? 0.0f : 1.0f;
    return (competing && available) ? power_heuristic(forward_pdf, nee_pdf) : 1.0f;
}
static float nee_light_weight(uint32_t mode, float nee_pdf, float forward_pdf) {
    if (mode == PSY_DIRECT_LIGHT_NEE) return 1.0f;
    if (mode == PSY_DIRECT_LIGHT_FORWARD) return forward_pdf <= 0.0f ? 1.0f : 0.0f;
    return power_heuristic(nee_pdf, forward_pdf);
}

// film_clamp_light (include/psycles/luisa/cycles_film_light.h:15-49).
static float3 clamp_contribution(float3 c, uint32_t depth, const Settings &st) {
    c = {std::isfinite(c.x) ? c.x : 0.0f, std::isfinite(c.y) ? c.y : 0.0f, std::isfinite(c.z) ? c.z : 0.0f};
    const float limit = depth > 0u ? st.raw.sample_clamp_indirect : st.raw.sample_clamp_direct;
    const float mag = std::fabs(c.x) + std::fabs(c.y) + std::fabs(c.z);
    if (limit > 0.0f && mag > limit) return c * (limit / maxf(mag, 1.0e-20f));
    return c;
}

// Light-threshold roulette (path_tracer_lighting.cpp:83-111).
static float light_roulette_weight(float3 unshadowed, float random, float inv_threshold) {
    const float m = max_abs_component(unshadowed);
    const float p = m * inv_threshold;
    const bool roulette = inv_threshold > 0.0f && p < 1.0f;
    const bool survives = !roulette || random < p;
    const float inv_p = roulette ? 1.0f / maxf(p, 1.0e-20f) : 1.0f;
    return survives ? inv_p : 0.0f;
}

// Path flags / visibility of include/psycles/luisa/cycles_path_state.h:20-59.
constexpr uint32_t kFlagReflect = 1u, kFlagSingular = 2u, kFlagTransparent = 4u, kFlagImportanceBake = 8u,
                   kFlagDiffuseAncestor = 16u, kFlagMisSkip = 128u, kFlagMisHadTransmission = 64u,
                   kFlagSinglePassDone = 256u, kFlagTransparentBackground = 512u,
                   kFlagTerminateOnNextSurface = 1024u, kFlagTerminateAfterTransparent = 4096u,
                   kFlagSurfacePass = 1u << 18u, kFlagVolumePass = 1u << 19u;
constexpr uint32_t kVisCamera = 1u, kVisTransmit = 2u, kVisDiffuse = 4u, kVisGlossy = 8u, kVisVolumeScatter = 16u;

struct PathState {
    uint32_t flag, visibility, bounce, diffuse_bounce, glossy_bounce, transmission_bounce, transparent_bounce,
        rng_offset;
};

// cycles_path_state::next_surface (cycles_path_state.h:205-338).
PathState next_surface(const PathState &before, uint32_t label, uint32_t runtime, uint32_t maximum,
                       uint32_t max_diffuse, uint32_t max_glossy, uint32_t max_transmission, uint32_t max_transparent) {
    const bool transparent = (label & (kLabelTransparent | 512u)) != 0u;
    PathState t = before;
    t.transparent_bounce += 1u;
    t.rng_offset += kBounceDimensions;
    t.flag |= kFlagTransparent;
    if (t.transparent_bounce >= max_transparent) t.flag |= kFlagTerminateOnNextSurface;
    if ((runtime & 4096u) != 0u) t.flag |= kFlagMisSkip;
    if (transparent) return t;

    PathState s = before;
    s.bounce += 1u;
    s.rng_offset += kBounceDimensions;
    if (s.bounce >= maximum) s.flag |= kFlagTerminateAfterTransparent;
    s.visibility = 0u;
    s.flag &= ~(kFlagReflect | kFlagSingular | kFlagTransparent | kFlagImportanceBake | kFlagMisSkip |
                kFlagMisHadTransmission);
    const bool reflection = (label & kLabelReflect) != 0u;
    const bool diffuse = (label & kLabelDiffuse) != 0u;
    const bool glossy = (label & kLabelGlossy) != 0u;
    const bool transmit_transparent = (label & 128u) != 0u;
    if (reflection) s.flag |= kFlagReflect;
    if (reflection || !transmit_transparent) s.flag &= ~kFlagTransparentBackground;
    const bool diffuse_reflection = reflection && diffuse;
    const bool glossy_reflection = reflection && !diffuse;
    const bool transmission = !reflection;
    if (diffuse_reflection) s.diffuse_bounce += 1u;
    if (glossy_reflection) s.glossy_bounce += 1u;
    if (transmission) s.transmission_bounce += 1u;
    if (diffuse_reflection && s.diffuse_bounce >= max_diffuse) s.flag |= kFlagTerminateAfterTransparent;
    if (glossy_reflection && s.glossy_bounce >= max_glossy) s.flag |= kFlagTerminateAfterTransparent;
    if (transmission && s.transmission_bounce >= max_transmission) s.flag |= kFlagTerminateAfterTransparent;
    if (transmission) s.visibility |= kVisTransmit;
    s.visibility |= diffuse ? kVisDiffuse : kVisGlossy;
    if (diffuse) s.flag |= kFlagDiffuseAncestor;
    if (!diffuse && !glossy) s.flag |= kFlagSingular | kFlagMisSkip;
    if ((runtime & kRuntimeBsdfHasTransmission) != 0u) s.flag |= kFlagMisHadTransmission;
    if ((s.flag & (kFlagSurfacePass | kFlagVolumePass)) == 0u && (s.flag & kFlagTransparentBackground) == 0u)
        s.flag |= kFlagSurfacePass;
    return s;
}

// contract_visibility (cycles_path_state.h:449-491).
static uint32_t contract_visibility(uint32_t v) {
    const uint32_t tv = (v & kVisTransmit) ? (v & ~(kVisDiffuse | kVisGlossy)) : v;
    uint32_t r = 0u;
    if (tv & kVisCamera) r |= PSY_VISIBILITY_CAMERA;
    if (tv & kVisTransmit) r |= PSY_VISIBILITY_TRANSMISSION;
    if (tv & kVisDiffuse) r |= PSY_VISIBILITY_DIFFUSE;
    if (tv & kVisGlossy) r |= PSY_VISIBILITY_GLOSSY;
    if (tv & kVisVolumeScatter) r |= PSY_VISIBILITY_VOLUME_SCATTER;
    return r;
}

// continuation_probability (cycles_path_state.h:413-447).
static float continuation_probability(uint32_t flag, uint32_t bounce, uint32_t transparent_bounce, uint32_t minimum,
                                      uint32_t transparent_minimum, float3 throughput) {
    const bool transparent = (flag & kFlagTransparent) != 0u;
    const bool before_min = transparent ? transparent_bounce <= transparent_minimum : bounce <= minimum;
    const float rr = minf(std::sqrt(max_abs_component(throughput)), 1.0f);
    return before_min ? 1.0f : rr;
}

struct PathOutput {
    float3 radiance{};
    float transparency{0.0f};
    float3 normal{};
    float3 albedo{};
};

static void trace_set3(float *dst, float3 v) {
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}
static void trace_add3(float *dst, float3 v) {
    dst[0] += v.x;
    dst[1] += v.y;
    dst[2] += v.z;
}

// One camera sample through the path loop: begin_path_sample
// (src/luisa/path_kernel_setup.cpp:485-700), PathKernelPipeline::emit
// (src/luisa/path_kernel_pipeline.cpp:73-183) and accumulate_path_sample
// (path_kernel_setup.cpp:903-997).
// make_triangle_emitter_callable (path_tracer_light_tree.cpp:762-797): the
// emitter identity of an emissive (object, primitive), or invalid.
static uint32_t tree_emitter(const Scene &s, uint32_t object, uint32_t primitive) {
    const std::array<uint32_t, 3> key{object, primitive, 0u};
    auto it = std::lower_bound(s.tree_lookup.begin(), s.tree_lookup.end(), key);
    if (it != s.tree_lookup.end() && (*it)[0] == object && (*it)[1] == primitive) return (*it)[2];
    return lt::kLtInvalid;
}

// sample_regular_polygon / sample_aperture (include/psycles/luisa/camera_sampling.h:118-152).
static float2 sample_aperture(float2 r, uint32_t blades, float rotation) {
    if (blades == 0u) return sample_uniform_disk(r);
    const float corners = static_cast<float>(blades);
    float u = r.x, v = r.y;
    const float corner = std::floor(u * corners);
    u = u * corners - corner;
    u = std::sqrt(u);
    v *= u;
    u = 1.0f - u;
    const float half_corner = kPi / corners;
    const float2 point = f2((u + v) * cos_(half_corner), (u - v) * sin_(half_corner));
    const float angle = rotation + corner * (2.0f * half_corner);
    const float c = cos_(angle), sn = sin_(angle);
    return f2(c * point.x - sn * point.y, sn * point.x + c * point.y);
}

static PathOutput render_path(const Scene &s, const Settings &st, uint32_t x, uint32_t y, uint32_t sample,
                              psy_path_trace *trace) {
    const psy_render_settings &r = st.raw;
    // sample_camera_dimensions (src/luisa/path_tracer_camera.cpp:10-45)
    const uint32_t cycles_y = r.full_height - 1u - y;
    const uint32_t rng_hash = pixel_hash(x, cycles_y, r.seed);
    const float4 fs = st.sobol.sample_4d(sample, rng_hash, kDimFilter);
    float2 filter = sample == 0u ? f2(0.5f, 0.5f) : f2(fs.x, fs.y);
    // construct_camera_ray (path_tracer_camera.cpp:47-246): perspective,
    // orthographic or equirectangular panorama, thin-lens depth of field
    const float jx = pixel_filter_sample(st.filter, filter.x);
    const float jy = 1.0f - pixel_filter_sample(st.filter, filter.y);
    const float W = static_cast<float>(r.full_width), H = static_cast<float>(r.full_height);
    const float sx = 2.0f * (static_cast<float>(x) + jx) / W - 1.0f + 2.0f * st.shift_x;
    const float sy = 1.0f - 2.0f * (static_cast<float>(y) + jy) / H + 2.0f * st.shift_y;
    float3 local_origin = f3(0.0f);
    float3 local_dir = f3(0.0f, 0.0f, -1.0f);
    float clip_cos = 1.0f;
    if (s.camera.projection == PSY_CAMERA_PERSPECTIVE) {
        local_dir = normalize(f3(sx * st.htan, sy * st.vtan, -1.0f));
        clip_cos = -local_dir.z;
    } else if (s.camera.projection == PSY_CAMERA_ORTHOGRAPHIC) {
        const float aspect = W / H;
        local_origin = f3(sx * st.ortho_span * aspect * 0.5f, sy * st.ortho_span * 0.5f, 0.0f);
    } else {
        const float longitude = sx * kPi;
        const float latitude = sy * kPi * 0.5f;
        const float cos_lat = cos_(latitude);
        local_dir = f3(cos_lat * sin_(longitude), sin_(latitude), -cos_lat * cos_(longitude));
    }
    if (st.depth_of_field) {
        // sample_3d at camera_lens_time_dimension (path_tracer_camera.cpp:35-45): lens = .yz
        const float4 lt = st.sobol.sample_4d(sample, rng_hash, 1u);
        float2 lens = sample_aperture(f2(lt.y, lt.z), s.camera.aperture_blades, s.camera.aperture_rotation) *
                      s.camera.aperture_radius;
        lens.x /= maxf(s.camera.aperture_ratio, 1.0e-5f);
        const float focus_scale = s.camera.focal_distance / maxf(-local_dir.z, 1.0e-6f);
        const float3 focus = local_dir * focus_scale;
        local_origin = f3(lens.x, lens.y, 0.0f);
        local_dir = normalize(focus - local_origin);
    }
    const mat4 cam = mat4_from_column_major(s.camera.camera_to_world);
    float3 origin = transform_point(cam, local_origin);
    const float3 dir = safe_normalize(transform_direction(cam, local_dir), f3(0.0f, 0.0f, -1.0f));
    const float safe_cos = maxf(std::fabs(clip_cos), 1.0e-20f);
    const float near_t = s.camera.near_clip / safe_cos;
    const float far_t = (s.camera.far_clip - s.camera.near_clip) / safe_cos;
    origin = origin + dir * near_t;
    Ray ray{origin, dir, 0.0f, far_t};

    if (trace) {
        trace->pixel_x = x;
        trace->pixel_y = y;
        trace->sample = sample;
        trace->rng_hash = rng_hash;
        trace->filter[0] = filter.x;
        trace->filter[1] = filter.y;
        trace_set3(trace->ray_origin, ray.o);
        trace_set3(trace->ray_direction, ray.d);
        trace->valid = 1u;
        trace->event_count = 0u;
    }

    PathOutput out;
    PathState ps{kFlagMisSkip | kFlagTransparentBackground, kVisCamera, 0, 0, 0, 0, 0, kBounceDimensions};
    float3 throughput = f3(1.0f);
    float3 radiance = f3(0.0f);
    float transparency = 0.0f;
    float previous_bsdf_pdf = 0.0f;
    bool previous_delta = true;
    float3 previous_mis_normal = f3(0.0f);
    bool primary_recorded = false;
    bool terminate_on_next_surface = false, terminate_after_transparent = false;
    uint32_t ray_visibility = PSY_VISIBILITY_CAMERA;
    uint32_t ray_events = 0u;
    Identity source;
    // path_tracer_kernel.cpp:206-223: NEE only when a light can be picked and
    // the mode is not forward path tracing; without it every emitter is
    // weighted as forward path tracing.
    const bool available = st.use_light_tree ? !s.tree.emitters.empty() : s.emitter_count > 0u;
    const bool nee = r.next_event_estimation != 0u && r.direct_light_sampling != PSY_DIRECT_LIGHT_FORWARD && available;
    const uint32_t mode = nee ? r.direct_light_sampling : PSY_DIRECT_LIGHT_FORWARD;

    for (uint32_t step = 0u; step < st.steps; ++step) {
        psy_path_event *ev = nullptr;
        if (trace && step < PSY_TRACE_MAX_EVENTS) {
            ev = &trace->events[step];
            std::memset(ev, 0, sizeof(*ev));
            ev->closure_index = kInvalid;
            ev->hit_object = kInvalid;
            ev->hit_primitive = kInvalid;
            ev->light_kind = kKindSentinel;
            ev->rng_offset = ps.rng_offset;
            trace->event_count = step + 1u;
        }
        // PathBounceSetupStage (src/luisa/path_kernel_bounce_setup.cpp:48-146)
        const float terminate_sample = st.sobol.sample_4d(sample, rng_hash, ps.rng_offset + kDimTerminate).x;
        const float4 ls4 = st.sobol.sample_4d(sample, rng_hash, ps.rng_offset + kDimLight);
        const float3 light_sample = f3(ls4.x, ls4.y, ls4.z);
        // with the light tree the pick needs the shading point (below)
        DistEntry selected = st.use_light_tree ? DistEntry{0.0f, 0.0f, kKindSentinel, 0u}
                                               : distribution_sample(s, light_sample.z);
        const float light_terminate = st.sobol.sample_4d(sample, rng_hash, ps.rng_offset + kDimLightTerminate).x;
        const float4 bs4 = st.sobol.sample_4d(sample, rng_hash, ps.rng_offset + kDimBsdf);
        const float3 bsdf_sample = f3(bs4.x, bs4.y, bs4.z);
        const Hit hit = closest_hit(s, ray, ray_visibility, source, Identity{});
        if (ev) {
            ev->random_terminate = terminate_sample;
            trace_set3(ev->random_light, light_sample);
            ev->random_light_terminate = light_terminate;
            trace_set3(ev->random_bsdf, bsdf_sample);
            ev->light_kind = selected.kind;
            ev->light_index = selected.index;
            ev->hit_t = hit.t;
            ev->hit_u = hit.u;
            ev->hit_v = hit.v;
            if (hit.valid) {
                ev->hit_object = hit.object;
                ev->hit_primitive = hit.cycles_prim;
            }
        }
        const uint32_t depth = ps.bounce;
        // Lamps in front of the mesh event are transparent events: they add
        // their emission, count a transparent bounce and move tmin past
        // themselves, without a new bounce or new Sobol dimensions
        // (path_kernel_pipeline.cpp:78-126, path_kernel_forward_light.cpp:14-118).
        bool lamp_terminated = false;
        {
            const float event_distance = hit.valid ? hit.t : ray.tmax;
            uint32_t excluded = kInvalid;
            float tmin = ray.tmin;
            for (;;) {
                const LampHit lh = closest_lamp(s, ray, tmin, event_distance, ray_visibility, excluded,
                                                previous_mis_normal, (ps.flag & kFlagMisHadTransmission) != 0u);
                if (!lh.valid) break;
                float selection_pdf = s.light_selection_pdf;
                if (st.use_light_tree)
                    selection_pdf = lt::tree_pdf(s.tree, static_cast<uint32_t>(s.emitters.size()) + lh.index, ray.o,
                                                 previous_mis_normal, (ps.flag & kFlagMisHadTransmission) != 0u);
                const float light_pdf = lh.pdf * selection_pdf;
                const bool competing = depth > 0u && !previous_delta;
                const float w = forward_light_weight(mode, previous_bsdf_pdf, light_pdf, competing, light_pdf > 0.0f);
                const psy_light_desc &l = s.lights[lh.index];
                const float3 lr = f3(l.color[0], l.color[1], l.color[2]) * (l.power * lh.eval_factor);
                const float3 c = clamp_contribution(throughput * lr * w, depth, st);
                radiance += c;
                if (ev) trace_add3(ev->emission, c);
                ps.transparent_bounce += 1u;
                tmin = lh.distance == 0.0f ? std::numeric_limits<float>::min() : bits_float(float_bits(lh.distance) + 1u);
                excluded = lh.index;
                if (ps.transparent_bounce >= st.transparent_max) {
                    lamp_terminated = true;
                    break;
                }
            }
        }
        if (lamp_terminated) {
            if (ev) ev->terminated = 1u;
            break;
        }
        if (!hit.valid) {
            // BackgroundEventStage (src/luisa/path_kernel_background_event.cpp:14-160):
            // the constant world is not part of the light distribution, so
            // the forward weight is one.
            const float3 c = clamp_contribution(throughput * s.background * 1.0f, depth, st);
            const bool world_visible = (s.world_visibility & ray_visibility) != 0u;
            const bool transparent_bg = r.transparent_background != 0u && (ps.flag & kFlagTransparentBackground) != 0u;
            if (transparent_bg) {
                transparency += (throughput.x + throughput.y + throughput.z) * (1.0f / 3.0f);
            } else if (world_visible) {
                radiance += c;
                if (ev) trace_add3(ev->emission, c);
            }
            if (ev) ev->terminated = 1u;
            break;
        }
        const SurfacePoint sp = surface_point(s, hit, ray);
        const Material &mat = s.materials[sp.material];
        const ClosurePoint cpt{sp.n, sp.ng, -ray.d, mat.bump_correction, sp.back_facing};
        const SurfaceClosures closures = collect_surface(mat, cpt);
        // SurfaceShadingStageImpl::emit (src/luisa/path_kernel_surface_shading.cpp:117-250)
        float emission_weight = 1.0f;
        if (nee && !s.emitters.empty() && mat.emission_sampling != 0u && mat.has_emission) {
            const bool competing = depth > 0u && !previous_delta;
            float selection_pdf = 0.5f * length(cross(sp.wp1 - sp.wp0, sp.wp2 - sp.wp0)) * s.triangle_area_pdf;
            if (st.use_light_tree)  // light_tree.forward_pdf (path_tracer_light_tree.cpp:785-823)
                selection_pdf = lt::tree_pdf(s.tree, tree_emitter(s, sp.object, sp.cycles_prim), ray.o,
                                             previous_mis_normal, (ps.flag & kFlagMisHadTransmission) != 0u);
            const float light_pdf = emissive_forward_pdf(selection_pdf, mat.emission_sampling, ray.o, sp.position,
                                                         sp.wp0, sp.wp1, sp.wp2,
                                                         // the geometric normal before the back-face flip
                                                         // (path_kernel_surface_shading.cpp:130-134)
                                                         sp.back_facing ? -sp.ng : sp.ng);
            const bool light_available = light_pdf > 0.0f;
            emission_weight = forward_light_weight(mode, previous_bsdf_pdf, light_pdf, competing, light_available);
        }
        const float3 emission_contribution = clamp_contribution(throughput * closures.emission * emission_weight, depth, st);
        radiance += emission_contribution;
        if (ev) trace_add3(ev->emission, emission_contribution);
        if (terminate_on_next_surface) {
            if (ev) ev->terminated = 1u;
            break;
        }
        const float cp = continuation_probability(ps.flag, ps.bounce, ps.transparent_bounce, st.minimum,
                                                  st.transparent_min, throughput);
        if (ev) ev->continuation_probability = cp;
        if (cp <= 0.0f) {
            if (ev) ev->terminated = 1u;
            break;
        }
        if (cp != 1.0f) {
            if (terminate_sample >= cp) {
                if (ev) ev->terminated = 1u;
                break;
            }
            throughput /= cp;
        }
        if (depth == 0u) {
            const Aov aov = surface_aov(closures, cpt);
            out.albedo += throughput * aov.albedo;
            const float3 alpha = clamp3(f3(1.0f) - aov.transparency, 0.0f, 1.0f);
            const float average_alpha = (alpha.x + alpha.y + alpha.z) * (1.0f / 3.0f);
            const bool writes_normal = !primary_recorded &&
                                       (r.pass_alpha_threshold == 0.0f || average_alpha >= r.pass_alpha_threshold);
            if (writes_normal) {
                out.normal = aov.normal;
                primary_recorded = true;
                ps.flag |= kFlagSinglePassDone;
            }
        }
        const uint32_t runtime = runtime_flags(closures, sp.back_facing);
        if (st.use_light_tree) {
            // light_tree.surface_sample after shading (path_kernel_pipeline.cpp:150-159)
            float pdf = 0.0f;
            const uint32_t slot = lt::tree_sample(s.tree, light_sample.z, sp.position, sp.n,
                                                  (runtime & kRuntimeBsdfHasTransmission) != 0u, pdf);
            if (slot != lt::kLtInvalid && s.tree.emitters[slot].emitter_id < s.emitter_count) {
                selected = s.distribution[s.tree.emitters[slot].emitter_id];
                selected.selection_pdf = pdf;
            }
            if (ev) {
                ev->light_kind = selected.kind;
                ev->light_index = selected.index;
            }
        }
        // SurfaceGeometryStage lobe mask (path_kernel_surface_geometry.cpp:62-84)
        const uint32_t lobe_mask = terminate_after_transparent ? kEventTransparent : 0xffffffffu;
        // Direct lighting (path_kernel_pipeline.cpp:160-172)
        if (nee && (runtime & kRuntimeBsdfHasEval) != 0u) {
            float3 contribution = f3(0.0f);
            if (selected.kind == kKindTriangle) {
                // EmissiveMeshLightingComponent (src/luisa/path_kernel_nee_emissive_mesh.cpp:32-296)
                const Emitter &em = s.emitters[selected.index];
                const TriSample ls = sample_triangle(sp.position, em.p0, em.p1, em.p2, f2(light_sample.x, light_sample.y));
                const bool side = sampled_side(em.emission_sampling, em.ng, ls.direction);
                const float pdf = ls.pdf * selected.selection_pdf;
                const bool valid = ls.valid && side && em.area > 0.0f && pdf > 0.0f;
                if (valid) {
                    const bool is_transmission = dot(ls.direction, sp.n) < 0.0f;
                    const bool same_primitive = em.cycles_prim == sp.cycles_prim && em.object == sp.object;
                    const float3 oriented = is_transmission ? -sp.ng : sp.ng;
                    const bool reject_self = same_primitive && dot(ls.direction, oriented) > 0.0f;
                    if (!reject_self) {
                        const float3 light_radiance = material_emission(s.materials[em.material]);
                        const Evaluation e = evaluate_mixture(closures, cpt, ls.direction, lobe_mask, -1);
                        float mis = 1.0f;
                        mis = nee_light_weight(mode, pdf, e.pdf);
                        const float3 weighted = e.f * light_radiance * (mis / pdf);
                        if (any_nonzero(weighted)) {
                            const float3 unshadowed = weighted * f3(1.0f);
                            const float3 surviving = unshadowed * light_roulette_weight(unshadowed, light_terminate, st.inv_rr_threshold);
                            if (any_nonzero(surviving)) {
                                const float3 so = surface_shadow_origin(s, sp, ls.direction);
                                const float3 off = ls.position - so;
                                const float dist = std::sqrt(maxf(length_squared(off), 1.0e-20f));
                                const Ray shadow{so, off / dist, 0.0f, dist};
                                const float3 tr = trace_shadow(s, shadow, Identity{sp.object, sp.cycles_prim},
                                                               Identity{em.object, em.cycles_prim},
                                                               ps.transparent_bounce, st.transparent_max);
                                if (tr.x > 0.0f || tr.y > 0.0f || tr.z > 0.0f)
                                    contribution = clamp_contribution(throughput * surviving * tr, depth, st);
                            }
                        }
                    }
                }
            } else if (selected.kind == kKindAnalytic) {
                // AnalyticLightingComponent (src/luisa/path_kernel_nee_analytic.cpp:98-428)
                const psy_light_desc &l = s.lights[selected.index];
                if (!(depth > l.max_bounces)) {
                    const float2 lxy = f2(light_sample.x, light_sample.y);
                    AnalyticSample a = l.type == PSY_LIGHT_DISTANT ? sample_distant(l, lxy)
                                       : l.type == PSY_LIGHT_AREA  ? sample_area(l, sp.position, lxy)
                                                                    : sample_point_or_spot(l, sp.position, sp.n,
                                                                                           (runtime & kRuntimeBsdfHasTransmission) != 0u, lxy);
                    const float light_pdf = a.pdf * selected.selection_pdf;
                    if (a.valid && light_pdf > 0.0f) {
                        const float3 light_radiance = f3(l.color[0], l.color[1], l.color[2]) * (l.power * a.eval_factor);
                        const Evaluation e = evaluate_mixture(closures, cpt, a.direction, lobe_mask, -1);
                        // MIS only for lamps a BSDF ray can also hit (path_kernel_nee_analytic.cpp:286-292)
                        const float mis = (l.flags & kLightForward) != 0u ? nee_light_weight(mode, light_pdf, e.pdf) : 1.0f;
                        const float3 weighted = e.f * light_radiance * (mis / maxf(light_pdf, 1.0e-20f));
                        if (any_nonzero(weighted)) {
                            const float3 unshadowed = weighted * f3(1.0f);
                            const float3 surviving = unshadowed * light_roulette_weight(unshadowed, light_terminate, st.inv_rr_threshold);
                            if (any_nonzero(surviving)) {
                                const float3 so = surface_shadow_origin(s, sp, a.direction);
                                const float3 off = a.position - so;
                                const float fd = std::sqrt(maxf(length_squared(off), 1.0e-20f));
                                const bool distant = l.type == PSY_LIGHT_DISTANT;
                                const Ray shadow{so, distant ? a.direction : off / fd, 0.0f, distant ? 1.0e30f : fd};
                                const float3 tr = trace_shadow(s, shadow, Identity{sp.object, sp.cycles_prim}, Identity{},
                                                               ps.transparent_bounce, st.transparent_max);
                                if (tr.x > 0.0f || tr.y > 0.0f || tr.z > 0.0f)
                                    contribution = clamp_contribution(throughput * surviving * tr, depth, st);
                            }
                        }
                    }
                }
            }
            radiance += contribution;
            if (ev) trace_set3(ev->nee, contribution);
        }
        // SurfaceScatterStageImpl::emit (src/luisa/path_kernel_surface_scatter.cpp:136-291)
        const SurfaceSample ss = sample_surface(closures, cpt, bsdf_sample.z, f2(bsdf_sample.x, bsdf_sample.y),
                                                lobe_mask);
        if (ev) {
            ev->closure_index = ss.closure_index;
            ev->bsdf_pdf = ss.eval.pdf;
            trace_set3(ev->wi, ss.wi);
        }
        if (!ss.valid || ss.eval.pdf <= 0.0f) {
            if (ev) ev->terminated = 1u;
            break;
        }
        const bool transparent = (ss.eval.events & kEventTransparent) != 0u;
        const bool singular = (ss.eval.events & kEventSingular) != 0u;
        const uint32_t label = label_from_events(ss.eval.events);
        throughput *= ss.eval.f / ss.eval.pdf;
        if (ev) {
            ev->label = label;
            trace_set3(ev->throughput, throughput);
        }
        if (any_nan(throughput) || throughput.x < 0.0f || throughput.y < 0.0f || throughput.z < 0.0f) {
            if (ev) ev->terminated = 1u;
            break;
        }
        ray_events = transparent ? (ray_events | ss.eval.events) : ss.eval.events;
        ps = next_surface(ps, label, runtime, st.maximum, st.max_diffuse, st.max_glossy, st.max_transmission,
                          st.transparent_max);
        ray_visibility = contract_visibility(ps.visibility);
        terminate_on_next_surface = (ps.flag & kFlagTerminateOnNextSurface) != 0u;
        terminate_after_transparent = (ps.flag & kFlagTerminateAfterTransparent) != 0u;
        if (!transparent) {
            previous_bsdf_pdf = ss.eval.pdf;
            previous_delta = singular;
            previous_mis_normal = sp.n;
        }
        if (ev) {
            ev->bounce = ps.bounce;
            ev->transparent_bounce = ps.transparent_bounce;
            ev->flag = ps.flag;
            ev->visibility = ps.visibility;
        }
        if (transparent) {
            const uint32_t next = float_bits(hit.t) + 1u;
            ray.tmin = hit.t == 0.0f ? std::numeric_limits<float>::min() : bits_float(next);
        } else {
            const float3 wi = normalize(ss.wi);
            ray.o = surface_ray_origin(s, sp, wi);
            ray.d = wi;
            ray.tmin = 0.0f;
            ray.tmax = 1.0e30f;
        }
        source = Identity{sp.object, sp.cycles_prim};
    }
    if (any_nan(radiance)) radiance = f3(0.0f);
    out.radiance = radiance;
    out.transparency = transparency;
    if (trace) trace_set3(trace->radiance, radiance);
    return out;
}

// ------------------------------------------------------------ scene prep

static std::unique_ptr<Scene> prepare_scene(const psy_scene_desc *d, bool brute_force) {
    auto s = std::make_unique<Scene>();
    s->brute_force = brute_force;
    uint32_t prim_offset = 0u;
    for (uint32_t i = 0; i < d->mesh_count; ++i) {
        const psy_mesh_desc &md = d->meshes[i];
        Mesh m;
        m.p.resize(md.vertex_count);
        for (uint32_t v = 0; v < md.vertex_count; ++v)
            m.p[v] = f3(md.positions[3 * v], md.positions[3 * v + 1], md.positions[3 * v + 2]);
        m.smooth = md.smooth != 0u && md.normals != nullptr;
        if (m.smooth) {
            m.n.resize(md.vertex_count);
            for (uint32_t v = 0; v < md.vertex_count; ++v)
                m.n[v] = f3(md.normals[3 * v], md.normals[3 * v + 1], md.normals[3 * v + 2]);
        }
        m.idx.assign(md.indices, md.indices + 3ull * md.triangle_count);
        if (md.materials) m.mat.assign(md.materials, md.materials + md.triangle_count);
        m.prim_offset = prim_offset;
        prim_offset += md.triangle_count;
        if (!brute_force) build_mesh_bvh(m);
        s->meshes.push_back(std::move(m));
    }
    for (uint32_t i = 0; i < d->material_count; ++i) {
        const psy_material_desc &md = d->materials[i];
        Material m;
        m.code.assign(md.closures, md.closures + md.closure_count);
        if (md.values) m.values.assign(md.values, md.values + md.value_count);
        m.root = md.root;
        m.scalars.assign(md.scalars, md.scalars + md.scalar_count);
        for (uint32_t v = 0; v < md.vector_count; ++v)
            m.vectors.push_back(f3(md.vectors[3 * v], md.vectors[3 * v + 1], md.vectors[3 * v + 2]));
        m.emission_sampling = md.emission_sampling;
        m.bump_correction = (md.flags & PSY_MATERIAL_NO_BUMP_MAP_CORRECTION) == 0u;
        m.has_emission = program_has(m, PSY_CLOSURE_EMISSION);
        m.has_transparent = program_has(m, PSY_CLOSURE_TRANSPARENT);
        m.ggx_e = d->ggx_e;
        m.ggx_eavg = d->ggx_eavg;
        s->materials.push_back(std::move(m));
    }
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const psy_instance_desc &id = d->instances[i];
        Instance inst;
        inst.o2w = mat4_from_column_major(id.object_to_world);
        inst.w2o = affine_inverse(inst.o2w);
        inst.nrm = normal_matrix(inst.w2o);
        inst.mesh = id.mesh;
        inst.material = id.material;
        inst.visibility = id.visibility;
        s->instances.push_back(inst);
    }
    s->lights.assign(d->lights, d->lights + d->light_count);
    for (psy_light_desc &l : s->lights) {
        bool extent = true;  // path_tracer_scene.cpp:1787-1830
        if (l.type == PSY_LIGHT_POINT || l.type == PSY_LIGHT_SPOT) extent = l.radius > 0.0f;
        if (l.type == PSY_LIGHT_AREA) extent = l.size_u != 0.0f && l.size_v != 0.0f && l.spread > 0.0f;
        if (l.type == PSY_LIGHT_DISTANT) extent = l.angle > 0.0f;
        if ((l.flags & PSY_LIGHT_FLAG_USE_MIS) != 0u && extent) {
            l.flags |= kLightUseMis;
            if (l.type != PSY_LIGHT_DISTANT) l.flags |= kLightForward;
        }
    }
    s->camera = d->camera;
    s->background = f3(d->background[0], d->background[1], d->background[2]);
    s->world_visibility = d->world_visibility;

    // Emissive triangles in instance order then primitive order, with world
    // vertices through the Cycles FMA transform and the world geometric
    // normal of _geometry (path_kernel_emissive_triangle.cpp:80-150).
    std::vector<float> areas;
    for (uint32_t i = 0; i < s->instances.size(); ++i) {
        const Instance &inst = s->instances[i];
        const Mesh &m = s->meshes[inst.mesh];
        const uint32_t tc = static_cast<uint32_t>(m.idx.size() / 3u);
        for (uint32_t k = 0; k < tc; ++k) {
            const uint32_t mi = m.mat.empty() ? inst.material : m.mat[k];
            const Material &mat = s->materials[mi];
            if (!mat.has_emission || mat.emission_sampling == 0u) continue;
            Emitter e;
            e.instance = i;
            e.prim = k;
            e.material = mi;
            e.object = i;
            e.cycles_prim = m.prim_offset + k;
            e.emission_sampling = mat.emission_sampling;
            const float3 lp0 = m.p[m.idx[3 * k]], lp1 = m.p[m.idx[3 * k + 1]], lp2 = m.p[m.idx[3 * k + 2]];
            e.p0 = transform_point(inst.o2w, lp0);
            e.p1 = transform_point(inst.o2w, lp1);
            e.p2 = transform_point(inst.o2w, lp2);
            const float3 ln = normalize_or(cross(lp1 - lp0, lp2 - lp0), f3(0.0f, 0.0f, 1.0f));
            e.ng = normalize_or(transform_direction(inst.nrm, ln), f3(0.0f, 0.0f, 1.0f));
            e.area = 0.5f * length(cross(e.p1 - e.p0, e.p2 - e.p0));
            s->emitters.push_back(e);
            areas.push_back(e.area);
        }
    }
    // build_cycles_light_distribution (src/sampling/light_distribution.cpp:25-150),
    // without the environment entry.
    auto valid_area = [](float a) { return std::isfinite(a) && a > 0.0f ? a : 0.0f; };
    const uint32_t tri_count = static_cast<uint32_t>(areas.size());
    const uint32_t light_count = static_cast<uint32_t>(s->lights.size());
    s->emitter_count = tri_count + light_count;
    float total = 0.0f;
    for (uint32_t i = 0; i < tri_count; ++i) {
        s->distribution.push_back({total, 0.0f, kKindTriangle, i});
        total += valid_area(areas[i]);
    }
    const float triangle_area = total;
    const float light_area = light_count > 0u ? (total > 0.0f ? total / static_cast<float>(light_count) : 1.0f) : 0.0f;
    for (uint32_t i = 0; i < light_count; ++i) {
        s->distribution.push_back({total, 0.0f, kKindAnalytic, i});
        total += light_area;
    }
    s->distribution.push_back({total, 0.0f, kKindSentinel, 0u});
    if (triangle_area > 0.0f) {
        s->triangle_area_pdf = 1.0f / triangle_area;
        if (light_count > 0u) s->triangle_area_pdf *= 0.5f;
    }
    if (light_count > 0u) {
        s->light_selection_pdf = 1.0f / static_cast<float>(light_count);
        if (triangle_area > 0.0f) s->light_selection_pdf *= 0.5f;
    }
    for (uint32_t i = 0; i < tri_count; ++i) s->distribution[i].selection_pdf = valid_area(areas[i]) * s->triangle_area_pdf;
    for (uint32_t i = tri_count; i < s->emitter_count; ++i) s->distribution[i].selection_pdf = s->light_selection_pdf;
    if (total > 0.0f) {
        const float inv = 1.0f / total;
        for (uint32_t i = 0; i < s->emitter_count; ++i) s->distribution[i].cumulative *= inv;
        s->distribution.back().cumulative = 1.0f;
    }
    // Light tree over the same population (path_tracer_light_sampling_scene.cpp:154-240):
    // triangles carry identities 0..T-1, analytic lights T..T+L-1.
    std::vector<lt::LtEmitter> population;
    for (uint32_t i = 0; i < tri_count; ++i) {
        const Emitter &e = s->emitters[i];
        const float3 estimate = emission_estimate(s->materials[e.material]);
        const float p0[3] = {e.p0.x, e.p0.y, e.p0.z}, p1[3] = {e.p1.x, e.p1.y, e.p1.z},
                    p2[3] = {e.p2.x, e.p2.y, e.p2.z}, em[3] = {estimate.x, estimate.y, estimate.z};
        const mat4 &m = s->instances[e.instance].o2w;
        const bool mirror = dot(m.c0, cross(m.c1, m.c2)) < 0.0f;
        population.push_back(lt::lt_triangle_emitter(i, p0, p1, p2, em, e.emission_sampling, mirror));
    }
    for (uint32_t i = 0; i < light_count; ++i) population.push_back(lt::lt_analytic_emitter(tri_count + i, &s->lights[i]));
    if (!population.empty()) {
        s->tree = lt::lt_build(population, 8u);
        const lt::LightTree &t = s->tree;
        s->tree_usable = t.root < t.nodes.size() && !t.emitters.empty() && t.emitter_to_tree.size() == t.emitters.size() &&
                         t.emitter_to_leaf.size() == t.emitters.size() && t.nodes[t.root].measure.energy > 0.0f;
    }
    for (uint32_t i = 0; i < tri_count; ++i) s->tree_lookup.push_back({s->emitters[i].object, s->emitters[i].cycles_prim, i});
    std::sort(s->tree_lookup.begin(), s->tree_lookup.end());
    return s;
}

}  // namespace oracle

// ----------------------------------------------------------------- C ABI

using namespace oracle;

extern "C" {

// Film sums for the window (row-major): combined (rgb, transparency),
// normal (xyz, count), albedo (xyz, count), sample count.  Accumulates into
// the caller's buffers, so progressive calls compose.
}  // extern "C"

namespace {

// Renders the window rows whose index is a multiple of `row_stride` over a
// prepared scene, accumulating into window-sized film sums.
void render_window(const Scene &scene, const psy_render_settings *settings, uint32_t first, uint32_t count,
                   uint32_t total, uint32_t row_stride, float *combined, float *normal, float *albedo,
                   uint32_t *sample_count, int threads, int trace_x, int trace_y, int trace_sample,
                   psy_path_trace *trace) {
    Settings st;
    derive_settings(st, scene, *settings, total);
    const psy_render_settings &r = *settings;
    const uint32_t wx = r.window_x, wy = r.window_y;
    const uint32_t ww = r.window_width ? r.window_width : r.full_width;
    const uint32_t wh = r.window_height ? r.window_height : r.full_height;
    if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    if (row_stride == 0u) row_stride = 1u;
    std::atomic<uint32_t> next_row{0u};
    auto worker = [&]() {
        for (;;) {
            const uint32_t row = row_stride * next_row.fetch_add(1u);
            if (row >= wh) return;
            for (uint32_t col = 0; col < ww; ++col) {
                const uint32_t x = wx + col, y = wy + row;
                const size_t pix = static_cast<size_t>(row) * ww + col;
                for (uint32_t k = 0; k < count; ++k) {
                    const uint32_t sample = first + k;
                    psy_path_trace *tr = nullptr;
                    if (trace && int(x) == trace_x && int(y) == trace_y && int(sample) == trace_sample) tr = trace;
                    const PathOutput o = render_path(scene, st, x, y, sample, tr);
                    combined[4 * pix + 0] += o.radiance.x;
                    combined[4 * pix + 1] += o.radiance.y;
                    combined[4 * pix + 2] += o.radiance.z;
                    combined[4 * pix + 3] += o.transparency;
                    normal[4 * pix + 0] += o.normal.x;
                    normal[4 * pix + 1] += o.normal.y;
                    normal[4 * pix + 2] += o.normal.z;
                    normal[4 * pix + 3] += 1.0f;
                    albedo[4 * pix + 0] += o.albedo.x;
                    albedo[4 * pix + 1] += o.albedo.y;
                    albedo[4 * pix + 2] += o.albedo.z;
                    albedo[4 * pix + 3] += 1.0f;
                    sample_count[pix] += 1u;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

}  // namespace

extern "C" {

int oracle_render(const psy_scene_desc *desc, const psy_render_settings *settings, uint32_t first, uint32_t count,
                  uint32_t total, float *combined, float *normal, float *albedo, uint32_t *sample_count,
                  int threads, int brute_force, int trace_x, int trace_y, int trace_sample, psy_path_trace *trace) {
    if (!desc || !settings || !combined || !normal || !albedo || !sample_count) return 1;
    auto scene = prepare_scene(desc, brute_force != 0);
    render_window(*scene, settings, first, count, total, 1u, combined, normal, albedo, sample_count, threads, trace_x,
                  trace_y, trace_sample, trace);
    return 0;
}

// oracle_render over a scene prepared once by oracle_scene_create (so the
// BVH build and emitter tables stay out of a timed render), rendering only
// the window rows whose index is a multiple of `row_stride`.
int oracle_render_prepared(const void *scene, const psy_render_settings *settings, uint32_t first, uint32_t count,
                           uint32_t total, uint32_t row_stride, float *combined, float *normal, float *albedo,
                           uint32_t *sample_count, int threads, int trace_x, int trace_y, int trace_sample,
                           psy_path_trace *trace) {
    if (!scene || !settings || !combined || !normal || !albedo || !sample_count) return 1;
    render_window(*static_cast<const Scene *>(scene), settings, first, count, total, row_stride, combined, normal,
                  albedo, sample_count, threads, trace_x, trace_y, trace_sample, trace);
    return 0;
}

// Normalised pass exactly as write_passes divides it
// (src/luisa/path_tracer_session.cpp:98-150).
int oracle_resolve_pass(uint32_t pass_kind, const float *sums4, const uint32_t *sample_count, uint64_t pixels,
                        float exposure, float *out) {
    for (uint64_t i = 0; i < pixels; ++i) {
        const float den = static_cast<float>(std::max(sample_count[i], 1u));
        if (pass_kind == PSY_PASS_SAMPLE_COUNT) {
            out[i] = static_cast<float>(sample_count[i]);
            continue;
        }
        const float *v = sums4 + 4 * i;
        if (pass_kind == PSY_PASS_COMBINED) {
            const float k = exposure / den;
            out[4 * i + 0] = v[0] * k;
            out[4 * i + 1] = v[1] * k;
            out[4 * i + 2] = v[2] * k;
            out[4 * i + 3] = clampf(1.0f - v[3] / den, 0.0f, 1.0f);
        } else {
            for (int c = 0; c < 4; ++c) out[4 * i + c] = v[c] / den;
        }
    }
    return 0;
}

void oracle_sobol_table(uint32_t size, float *out) {
    const auto t = sobol_generate_table(size);
    std::memcpy(out, t.data(), t.size() * sizeof(float4));
}
uint64_t oracle_sobol_fingerprint(uint32_t size) { return sobol_table_fingerprint(sobol_generate_table(size)); }
uint32_t oracle_sobol_sequence_size(uint32_t samples) { return sobol_sequence_size_for_samples(samples); }
void oracle_pixel_filter_table(uint32_t filter, float width, float *out) {
    const auto t = pixel_filter_table(filter, width);
    std::memcpy(out, t.data(), sizeof(float) * 1024);
}
uint32_t oracle_pixel_hash(uint32_t x, uint32_t y, uint32_t seed) { return pixel_hash(x, y, seed); }
uint32_t oracle_shuffled_sample_index(uint32_t sample, uint32_t dim, uint32_t seed, uint32_t size) {
    return shuffled_sample_index(sample, dim, seed, size);
}
void oracle_sample_cosine_hemisphere(const float *n, const float *r, float *out_dir, float *out_pdf) {
    const HemisphereSample h = sample_cosine_hemisphere(f3(n[0], n[1], n[2]), f2(r[0], r[1]));
    out_dir[0] = h.direction.x;
    out_dir[1] = h.direction.y;
    out_dir[2] = h.direction.z;
    *out_pdf = h.pdf;
}
// Visible-normal samples of the glossy closures (`beckmann` 0: GGX).
void oracle_sample_visible_normal(int beckmann, const float *n, const float *incoming, float alpha, const float *r,
                                  float *out_half) {
    const float3 nn = f3(n[0], n[1], n[2]), in = f3(incoming[0], incoming[1], incoming[2]);
    const float3 h = beckmann ? sample_beckmann_visible_normal(nn, in, alpha, f2(r[0], r[1]))
                              : sample_ggx_visible_normal(nn, in, alpha, f2(r[0], r[1]));
    out_half[0] = h.x;
    out_half[1] = h.y;
    out_half[2] = h.z;
}
void oracle_make_orthonormals(const float *n, float *t, float *b) {
    const Basis bs = make_orthonormals(f3(n[0], n[1], n[2]));
    t[0] = bs.tangent.x; t[1] = bs.tangent.y; t[2] = bs.tangent.z;
    b[0] = bs.bitangent.x; b[1] = bs.bitangent.y; b[2] = bs.bitangent.z;
}
// state: flag, visibility, bounce, diffuse, glossy, transmission, transparent, rng_offset
// limits: maximum, max_diffuse, max_glossy, max_transmission, max_transparent
void oracle_next_surface(const uint32_t *state, uint32_t label, uint32_t runtime, const uint32_t *limits,
                         uint32_t *out) {
    const PathState b{state[0], state[1], state[2], state[3], state[4], state[5], state[6], state[7]};
    const PathState n = next_surface(b, label, runtime, limits[0], limits[1], limits[2], limits[3], limits[4]);
    const uint32_t v[8] = {n.flag, n.visibility, n.bounce, n.diffuse_bounce, n.glossy_bounce, n.transmission_bounce,
                           n.transparent_bounce, n.rng_offset};
    std::memcpy(out, v, sizeof(v));
}
uint32_t oracle_contract_visibility(uint32_t v) { return contract_visibility(v); }
// diffuse_intensity of one diffuse closure (normal, authored colour,
// roughness) for a viewer direction and a light direction.
void oracle_diffuse_intensity(const float *normal, const float *color, float roughness, const float *incoming,
                              const float *outgoing, float *out) {
    PhysicalClosure c{};
    c.op = PSY_CLOSURE_DIFFUSE;
    c.normal = f3(normal[0], normal[1], normal[2]);
    c.color = f3(color[0], color[1], color[2]);
    c.roughness = roughness;
    const float3 v = diffuse_intensity(c, f3(incoming[0], incoming[1], incoming[2]),
                                       f3(outgoing[0], outgoing[1], outgoing[2]));
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

// Prepared scene handle for traversal parity tests.
void *oracle_scene_create(const psy_scene_desc *desc, int brute_force) {
    return prepare_scene(desc, brute_force != 0).release();
}
void oracle_scene_destroy(void *scene) { delete static_cast<Scene *>(scene); }

// Closest hits of `count` world rays (origin, direction, tmin, tmax):
// writes (t, u, v) and (object, cycles primitive), 0xffffffff on a miss.
void oracle_scene_closest(const void *scene, const float *rays8, uint32_t count, uint32_t visibility,
                          float *out_tuv, uint32_t *out_ids) {
    const Scene &s = *static_cast<const Scene *>(scene);
    for (uint32_t i = 0; i < count; ++i) {
        const float *q = rays8 + 8 * i;
        const Ray r{f3(q[0], q[1], q[2]), f3(q[3], q[4], q[5]), q[6], q[7]};
        const Hit h = closest_hit(s, r, visibility, Identity{}, Identity{});
        out_tuv[3 * i + 0] = h.t;
        out_tuv[3 * i + 1] = h.u;
        out_tuv[3 * i + 2] = h.v;
        out_ids[2 * i + 0] = h.valid ? h.object : kInvalid;
        out_ids[2 * i + 1] = h.valid ? h.cycles_prim : kInvalid;
    }
}



// Light-tree build over emitter records, with the record layout and outputs
// of the reference shim's ref_build_light_tree (oracle/ref_shim.cpp) so a
// test compares the two word for word.
static void put_measure(const lt::LtMeasure &m, float *o) {
    for (int k = 0; k < 3; ++k) {
        o[k] = m.bounds.lo[k];
        o[3 + k] = m.bounds.hi[k];
        o[7 + k] = m.orientation.axis[k];
    }
    o[6] = m.bounds.empty ? 1.0f : 0.0f;
    o[10] = m.orientation.theta_o;
    o[11] = m.orientation.theta_e;
    o[12] = m.orientation.empty ? 1.0f : 0.0f;
    o[13] = m.energy;
}

int oracle_build_light_tree(const float *in, uint32_t n, uint32_t max_leaf, uint32_t node_capacity, float *node_measure,
                            uint32_t *node_topology, float *emitter_measure, uint32_t *emitter_ids, uint32_t *to_tree,
                            uint32_t *to_leaf, uint32_t *root, uint32_t *node_count) {
    std::vector<lt::LtEmitter> source(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float *r = in + 20u * i;
        lt::LtEmitter &e = source[i];
        for (int k = 0; k < 3; ++k) {
            e.measure.bounds.lo[k] = r[k];
            e.measure.bounds.hi[k] = r[3 + k];
            e.measure.orientation.axis[k] = r[7 + k];
            e.centroid[k] = r[14 + k];
        }
        e.measure.bounds.empty = r[6] != 0.0f;
        e.measure.orientation.theta_o = r[10];
        e.measure.orientation.theta_e = r[11];
        e.measure.orientation.empty = r[12] != 0.0f;
        e.measure.energy = r[13];
        e.distant = r[17] != 0.0f;
        e.emitter_id = static_cast<uint32_t>(r[18]);
    }
    try {
        const lt::LightTree t = lt::lt_build(source, max_leaf);
        if (t.nodes.size() > node_capacity) return 2;
        for (size_t k = 0; k < t.nodes.size(); ++k) {
            const lt::LtNode &nd = t.nodes[k];
            put_measure(nd.measure, node_measure + 14u * k);
            uint32_t *w = node_topology + 6u * k;
            w[0] = nd.parent;
            w[1] = nd.left;
            w[2] = nd.right;
            w[3] = nd.first;
            w[4] = nd.count;
            w[5] = nd.kind;
        }
        for (size_t k = 0; k < t.emitters.size(); ++k) {
            put_measure(t.emitters[k].measure, emitter_measure + 14u * k);
            emitter_ids[k] = t.emitters[k].emitter_id;
        }
        for (size_t k = 0; k < t.emitter_to_tree.size(); ++k) {
            to_tree[k] = t.emitter_to_tree[k];
            to_leaf[k] = t.emitter_to_leaf[k];
        }
        *root = t.root;
        *node_count = static_cast<uint32_t>(t.nodes.size());
        return 0;
    } catch (...) {
        return 1;
    }
}

// Light-tree selection over a prepared scene (oracle_scene_create) for
// `count` shading points.  queries: 8 floats per point (position xyz,
// random u, normal xyz, has_transmission 0/1).  Writes the selected emitter
// identity (0xffffffff for none) with its selection pdf, and the reverse pdf
// of emitter pdf_emitters[i] from the same point.  Returns 1 when the scene
// has no usable tree.
int oracle_light_tree_query(const void *scene, const float *queries, const uint32_t *pdf_emitters, uint32_t count,
                            uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf) {
    const Scene &s = *static_cast<const Scene *>(scene);
    if (!s.tree_usable) return 1;
    for (uint32_t i = 0; i < count; ++i) {
        const float *q = queries + 8u * i;
        const float3 p = f3(q[0], q[1], q[2]), n = f3(q[4], q[5], q[6]);
        const bool tr = q[7] != 0.0f;
        float pdf = 0.0f;
        const uint32_t slot = lt::tree_sample(s.tree, q[3], p, n, tr, pdf);
        out_emitters[i] = slot == lt::kLtInvalid ? slot : s.tree.emitters[slot].emitter_id;
        out_sample_pdf[i] = slot == lt::kLtInvalid ? 0.0f : pdf;
        out_reverse_pdf[i] = lt::tree_pdf(s.tree, pdf_emitters[i], p, n, tr);
    }
    return 0;
}

uint32_t oracle_scene_emitter_count(const void *scene) { return static_cast<const Scene *>(scene)->emitter_count; }

// The flat light distribution's pick for each random number u: the entry's
// kind, index and selection pdf.
void oracle_distribution_sample(const void *scene, const float *u, uint32_t count, uint32_t *out_kind,
                                uint32_t *out_index, float *out_pdf) {
    const Scene &s = *static_cast<const Scene *>(scene);
    for (uint32_t i = 0; i < count; ++i) {
        const DistEntry e = distribution_sample(s, u[i]);
        out_kind[i] = e.kind;
        out_index[i] = e.index;
        out_pdf[i] = e.selection_pdf;
    }
}

// Emitter identity of an emissive (object, cycles primitive) pair.
uint32_t oracle_light_tree_triangle_emitter(const void *scene, uint32_t object, uint32_t primitive) {
    return tree_emitter(*static_cast<const Scene *>(scene), object, primitive);
}

}  // extern "C"
