// Many-light tree (host build + device layout).
//
// Host: emitter measures of emissive triangles and analytic lights
// (make_triangle_light_tree_emitter / make_analytic_light_tree_emitter,
// src/luisa/path_tracer_light_tree_scene.cpp:131-256) and the Cycles tree
// build with the 12-bucket surface-area-orientation heuristic and a separate
// distant branch (build_cycles_light_tree, src/sampling/light_tree.cpp:86-287).
// Device: the packed node / emitter records the sampling kernels read.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace psy {

struct LtBounds {
    float lo[3] = {0.0f, 0.0f, 0.0f};
    float hi[3] = {0.0f, 0.0f, 0.0f};
    bool empty = true;
};

struct LtOrientation {
    float axis[3] = {0.0f, 0.0f, 0.0f};
    float theta_o = 0.0f;
    float theta_e = 0.0f;
    bool empty = true;
};

struct LtMeasure {
    LtBounds bounds;
    LtOrientation orientation;
    float energy = 0.0f;
};

struct LtEmitter {
    LtMeasure measure;
    float centroid[3] = {0.0f, 0.0f, 0.0f};
    uint32_t emitter_id = 0u;
    bool distant = false;
};

enum LtKind : uint32_t { kLtInner = 0u, kLtLeaf = 1u, kLtDistant = 2u };
constexpr uint32_t kLtInvalid = 0xffffffffu;

struct LtNode {
    LtMeasure measure;
    uint32_t parent = kLtInvalid, left = kLtInvalid, right = kLtInvalid;
    uint32_t first = 0u, count = 0u;
    uint32_t kind = kLtLeaf;
};

struct LightTree {
    std::vector<LtEmitter> emitters;
    std::vector<LtNode> nodes;
    std::vector<uint32_t> emitter_to_tree, emitter_to_leaf;
    uint32_t root = kLtInvalid;
};

LtMeasure lt_merge(const LtMeasure &a, const LtMeasure &b);
float lt_cost(const LtMeasure &m);
LightTree lt_build(const std::vector<LtEmitter> &emitters, uint32_t max_leaf = 8u);

// world-space triangle (vertices already transformed) with an emission
// estimate (the constant emission colour) and EmissionSampling mode;
// `mirror` is true when the instance transform has a negative determinant.
LtEmitter lt_triangle_emitter(uint32_t id, const float p0[3], const float p1[3], const float p2[3],
                              const float emission[3], uint32_t sampling, bool mirror);
LtEmitter lt_analytic_emitter(uint32_t id, const void *light_desc);

// Device records: 16-byte lanes as the reference packs them
// (src/luisa/path_tracer_light_tree_scene.cpp:102-128).
constexpr uint32_t kLtFlagOrientation = 1u, kLtFlagBounds = 2u, kLtFlagDistant = 4u;

// `cone` holds the orientation cone's cosines and sine the importance
// bounds use, computed on the host in double and rounded once:
// cos(theta_o), sin(theta_o), cos(theta_o + theta_e), cos(theta_e - theta_o).
struct alignas(16) LtNodeGpu {
    float4 min_energy;      // bounds min, energy
    float4 max_theta_o;     // bounds max, theta_o
    float4 axis_theta_e;    // cone axis, theta_e
    float4 cone;
    uint4 topology;         // parent, left, right, kind
    uint4 emitters;         // first, count, flags, pad
};

struct alignas(16) LtEmitterGpu {
    float4 min_energy;
    float4 max_theta_o;
    float4 axis_theta_e;
    float4 cone;
    uint4 identity;         // distribution index, flags, emitter id, pad
};

}  // namespace psy
