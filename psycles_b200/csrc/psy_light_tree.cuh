// Device light-tree sampling and pdf for surface points: the
// importance-guided descent with min/max importance bounds, leaf reservoir
// selection, and the reverse pdf of a forward-hit emitter
// (src/luisa/path_tracer_light_tree.cpp:19-880, surface case).
#pragma once

#include "psy_light_tree.h"
#include "psy_math.cuh"
#include "psy_scene.h"

namespace psy {

constexpr float kLtSafe = 1.0e-20f;
constexpr float kLtPi = 3.14159265358979323846f;
constexpr float kLtHalfPi = 0.5f * kLtPi;

__device__ __forceinline__ f3 lt_safe_normalize(f3 v, f3 fallback) {
    const float l2 = dot(v, v);
    return l2 > kLtSafe ? v * (1.0f / sqrtf(maxf_(l2, kLtSafe))) : fallback;
}
__device__ __forceinline__ float lt_sin_from_cos(float c) { return sqrtf(maxf_(1.0f - c * c, 0.0f)); }

// cos_bound_subtended_angle (path_tracer_light_tree.cpp:40-52).
__device__ __forceinline__ float lt_cos_subtended(f3 bmax, f3 centroid, f3 point) {
    const float d2 = dot(point - centroid, point - centroid);
    const float r2 = dot(bmax - centroid, bmax - centroid);
    return d2 <= r2 ? -1.0f : sqrtf(maxf_(1.0f - r2 / maxf_(d2, kLtSafe), 0.0f));
}

// bounded_importance, surface case (path_tracer_light_tree.cpp:86-193).
__device__ __forceinline__ f2 lt_bounded_importance(f3 n, bool has_transmission, f3 p2c, float cos_u, f3 axis,
                                                    float theta_o, float theta_e, float4 cone, float max_d,
                                                    float min_d, float energy) {
    cos_u = clampf_(cos_u, -1.0f, 1.0f);
    const float sin_u = lt_sin_from_cos(cos_u);
    bool visible = energy > 0.0f;
    const float inc_cos = has_transmission ? fabsf(dot(p2c, n)) : dot(p2c, n);
    const float inc_sin = lt_sin_from_cos(clampf_(inc_cos, -1.0f, 1.0f));
    const float min_inc = inc_cos >= cos_u ? 1.0f : inc_cos * cos_u + inc_sin * sin_u;
    const float max_inc = maxf_(inc_cos * cos_u - inc_sin * sin_u, 0.0f);
    visible = visible && (has_transmission || min_inc >= 0.0f);
    const float th_cos = clampf_(dot(axis, -p2c), -1.0f, 1.0f);
    const float th_sin = lt_sin_from_cos(th_cos);
    const float tmu_cos = th_cos * cos_u + th_sin * sin_u;
    const float to_cos = cone.x;
    const float to_sin = cone.y;
    const bool fully = th_cos >= cos_u || tmu_cos >= to_cos;
    const bool partially = !fully && (theta_o + theta_e > kLtPi || tmu_cos > cone.z);
    const float tmu_sin = lt_sin_from_cos(clampf_(tmu_cos, -1.0f, 1.0f));
    const float min_out = fully ? 1.0f : (partially ? tmu_cos * to_cos + tmu_sin * to_sin : 0.0f);
    visible = visible && (fully || partially);
    min_d = maxf_(min_d, kLtSafe);
    max_d = maxf_(max_d, kLtSafe);
    const float geometric = 1.0f / (min_d * min_d);
    const float maximum = visible ? fabsf(min_inc * energy * min_out * geometric) : 0.0f;
    const float tpu_cos = th_cos * cos_u - th_sin * sin_u;
    const bool min_zero = (theta_e - theta_o < 0.0f) || (th_cos < 0.0f) || (cos_u < 0.0f) ||
                          (tpu_cos < cone.w);
    const float tpu_sin = lt_sin_from_cos(clampf_(tpu_cos, -1.0f, 1.0f));
    const float max_out = tpu_cos * to_cos - tpu_sin * to_sin;
    const float minimum = (min_zero || !visible) ? 0.0f : fabsf(max_inc * energy * max_out / (max_d * max_d));
    return {maximum, minimum};
}

// measure_importance (path_tracer_light_tree.cpp:195-277).
__device__ __noinline__ f2 lt_measure_importance(float4 min_energy, float4 max_theta_o, float4 axis_theta_e,
                                                    float4 cone, uint32_t flags, f3 point, f3 n,
                                                    bool has_transmission) {
    f2 result = {0.0f, 0.0f};
    const bool has_orientation = (flags & kLtFlagOrientation) != 0u;
    const bool has_bounds = (flags & kLtFlagBounds) != 0u;
    const bool distant = (flags & kLtFlagDistant) != 0u;
    if (!(has_orientation && min_energy.w > 0.0f)) return result;
    const f3 axis = lt_safe_normalize(ld3(axis_theta_e), mk3(0.0f, 0.0f, 1.0f));
    f3 p2c = -axis;
    float cos_u = cone.z;
    float emitter_distance = 1.0f;
    bool visible = true;
    if (!distant) {
        visible = has_bounds;
        const f3 bmin = ld3(min_energy), bmax = ld3(max_theta_o);
        const f3 centroid = (bmin + bmax) * 0.5f;
        const f3 extent = bmax - centroid;
        const f3 an = mk3(fabsf(n.x), fabsf(n.y), fabsf(n.z));
        const f3 ae = mk3(fabsf(extent.x), fabsf(extent.y), fabsf(extent.z));
        visible = has_transmission || (dot(n, centroid - point) + dot(an, ae) > 0.0f);
        const f3 delta = centroid - point;
        emitter_distance = length(delta);
        p2c = lt_safe_normalize(delta, -axis);
        cos_u = lt_cos_subtended(bmax, centroid, point);
        emitter_distance = maxf_(0.5f * length(centroid - bmax), emitter_distance);
    }
    if (visible)
        result = lt_bounded_importance(n, has_transmission, p2c, cos_u, axis, max_theta_o.w, axis_theta_e.w, cone,
                                       emitter_distance, emitter_distance, min_energy.w);
    return result;
}

__device__ __forceinline__ f2 lt_emitter_importance(const SceneView &s, uint32_t e, f3 point, f3 n, bool tr) {
    const LtEmitterGpu em = s.lt_emitters[e];
    return lt_measure_importance(em.min_energy, em.max_theta_o, em.axis_theta_e, em.cone, em.identity.y, point, n, tr);
}

// child_importance (path_tracer_light_tree.cpp:321-356).
__device__ __forceinline__ f2 lt_child_importance(const SceneView &s, uint32_t node_index, f3 point, f3 n, bool tr) {
    const LtNodeGpu node = s.lt_nodes[node_index];
    const bool inner = node.topology.w == kLtInner;
    if (inner || node.emitters.y > 1u)
        return lt_measure_importance(node.min_energy, node.max_theta_o, node.axis_theta_e, node.cone, node.emitters.z,
                                     point, n, tr);
    if (node.emitters.y == 1u) return lt_emitter_importance(s, node.emitters.x, point, n, tr);
    return {0.0f, 0.0f};
}

// left_probability (path_tracer_light_tree.cpp:358-398): (probability, valid).
__device__ __forceinline__ f2 lt_left_probability(const SceneView &s, uint32_t left, uint32_t right, f3 point, f3 n,
                                                  bool tr) {
    const f2 li = lt_child_importance(s, left, point, n, tr);
    const f2 ri = lt_child_importance(s, right, point, n, tr);
    const float max_total = li.x + ri.x;
    const float min_total = li.y + ri.y;
    const float max_p = li.x / maxf_(max_total, kLtSafe);
    const float min_p = min_total > 0.0f ? li.y / maxf_(min_total, kLtSafe)
                                         : 0.5f * ((li.x > 0.0f ? 1.0f : 0.0f) + (ri.x == 0.0f ? 1.0f : 0.0f));
    return {0.5f * (max_p + min_p), max_total > 0.0f ? 1.0f : 0.0f};
}

__device__ __forceinline__ void lt_reservoir_update(uint32_t current, float weight, uint32_t &selected,
                                                    float &selected_weight, float &total, float &random) {
    if (!(weight > 0.0f)) return;
    total += weight;
    if (selected == kLtInvalid) {
        selected = current;
        selected_weight = weight;
    } else {
        const float threshold = weight / total;
        if (random <= threshold) {
            selected = current;
            selected_weight = weight;
            random = random / threshold;
        } else {
            random = (random - threshold) / maxf_(1.0f - threshold, kLtSafe);
        }
        random = clampf_(random, 0.0f, 1.0f);
    }
}

// select_leaf_emitter (path_tracer_light_tree.cpp:430-527).
__device__ __forceinline__ void lt_select_leaf(const SceneView &s, const LtNodeGpu &node, f3 point, f3 n, bool tr,
                                               float &random, uint32_t &selected, float &selection_pdf) {
    float sel_max = 0.0f, sel_min = 0.0f, tot_max = 0.0f, tot_min = 0.0f;
    uint32_t positive = 0u;
    const bool sample_max = random > 0.5f;
    if (node.emitters.y > 1u) random = random * 2.0f - (sample_max ? 1.0f : 0.0f);
    for (uint32_t i = 0; i < node.emitters.y; ++i) {
        const uint32_t e = node.emitters.x + i;
        const f2 imp = lt_emitter_importance(s, e, point, n, tr);
        tot_max += imp.x;
        tot_min += imp.y;
        positive += imp.x > 0.0f ? 1u : 0u;
        const float primary = sample_max ? imp.x : imp.y;
        const float primary_total = sample_max ? tot_max : tot_min;
        if (primary > 0.0f) {
            if (selected == kLtInvalid) {
                selected = e;
                sel_max = imp.x;
                sel_min = imp.y;
            } else {
                const float threshold = primary / primary_total;
                if (random <= threshold) {
                    selected = e;
                    sel_max = imp.x;
                    sel_min = imp.y;
                    random = random / threshold;
                } else {
                    random = (random - threshold) / maxf_(1.0f - threshold, kLtSafe);
                }
                random = clampf_(random, 0.0f, 1.0f);
            }
        }
    }
    if (positive > 0u && tot_min == 0.0f) {
        if (sample_max) {
            sel_min = 1.0f;
            tot_min = static_cast<float>(positive);
        } else {
            selected = kLtInvalid;
            float sel_uniform = 0.0f, tot_uniform = 0.0f;
            for (uint32_t i = 0; i < node.emitters.y; ++i) {
                const uint32_t e = node.emitters.x + i;
                const f2 imp = lt_emitter_importance(s, e, point, n, tr);
                lt_reservoir_update(e, imp.x > 0.0f ? 1.0f : 0.0f, selected, sel_uniform, tot_uniform, random);
                if (selected == e) {
                    sel_max = imp.x;
                    sel_min = 1.0f;
                }
            }
            tot_min = tot_uniform;
        }
    }
    if (selected != kLtInvalid)
        selection_pdf *= 0.5f * (sel_max / maxf_(tot_max, kLtSafe) + sel_min / maxf_(tot_min, kLtSafe));
}

// make_sample_callable, surface case (path_tracer_light_tree.cpp:547-637):
// the selected emitter's distribution entry with the tree's selection pdf.
__device__ __noinline__ DistEntryGpu lt_sample(const SceneView &s, float u, f3 point, f3 n, bool tr) {
    DistEntryGpu result{0.0f, 0.0f, 3u, 0u};
    if (s.lt_node_count == 0u || s.lt_emitter_count == 0u || s.lt_root >= s.lt_node_count) return result;
    float random = clampf_(u, 0.0f, 1.0f);
    float selection_pdf = 1.0f;
    uint32_t node_index = s.lt_root;
    uint32_t selected = kLtInvalid;
    for (uint32_t steps = 0; steps <= s.lt_node_count; ++steps) {
        const LtNodeGpu node = s.lt_nodes[node_index];
        if (node.topology.w != kLtInner) {
            lt_select_leaf(s, node, point, n, tr, random, selected, selection_pdf);
            break;
        }
        const f2 p = lt_left_probability(s, node.topology.y, node.topology.z, point, n, tr);
        if (p.y <= 0.0f) break;
        const float right_p = 1.0f - p.x;
        const bool right = random <= right_p;
        node_index = right ? node.topology.z : node.topology.y;
        selection_pdf *= right ? right_p : p.x;
        random = right ? random / maxf_(right_p, kLtSafe) : (random - right_p) / maxf_(p.x, kLtSafe);
        random = clampf_(random, 0.0f, 1.0f);
    }
    if (selected != kLtInvalid) {
        const uint32_t d = s.lt_emitters[selected].identity.x;
        if (d < s.emitter_count) {
            result = s.distribution[d];
            result.selection_pdf = selection_pdf;
        }
    }
    return result;
}

// make_pdf_callable, surface case (path_tracer_light_tree.cpp:639-760).
__device__ __noinline__ float lt_pdf(const SceneView &s, uint32_t emitter_id, f3 point, f3 n, bool tr) {
    if (s.lt_node_count == 0u || s.lt_emitter_count == 0u || emitter_id >= s.lt_emitter_count) return 0.0f;
    const uint2 mapping = s.lt_mapping[emitter_id];
    const uint32_t target = mapping.x;
    uint32_t current = mapping.y;
    if (!(target < s.lt_emitter_count && current < s.lt_node_count)) return 0.0f;
    const LtNodeGpu leaf = s.lt_nodes[current];
    float t_max = 0.0f, t_min = 0.0f, tot_max = 0.0f, tot_min = 0.0f;
    uint32_t positive = 0u;
    for (uint32_t i = 0; i < leaf.emitters.y; ++i) {
        const uint32_t e = leaf.emitters.x + i;
        const f2 imp = lt_emitter_importance(s, e, point, n, tr);
        tot_max += imp.x;
        tot_min += imp.y;
        positive += imp.x > 0.0f ? 1u : 0u;
        if (e == target) {
            t_max = imp.x;
            t_min = imp.y;
        }
    }
    if (!(t_max > 0.0f)) return 0.0f;
    float result = 0.5f * (t_max / maxf_(tot_max, kLtSafe) +
                           (tot_min > 0.0f ? t_min / maxf_(tot_min, kLtSafe)
                                           : 1.0f / maxf_(static_cast<float>(positive), 1.0f)));
    for (uint32_t steps = 0; current != s.lt_root && steps <= s.lt_node_count; ++steps) {
        const uint32_t parent_index = s.lt_nodes[current].topology.x;
        if (parent_index >= s.lt_node_count) return 0.0f;
        const LtNodeGpu parent = s.lt_nodes[parent_index];
        const f2 p = lt_left_probability(s, parent.topology.y, parent.topology.z, point, n, tr);
        if (p.y <= 0.0f) return 0.0f;
        result *= current == parent.topology.y ? p.x : 1.0f - p.x;
        current = parent_index;
    }
    return current == s.lt_root ? result : 0.0f;
}

// make_triangle_emitter_callable (path_tracer_light_tree.cpp:762-797).
__device__ __forceinline__ uint32_t lt_triangle_emitter(const SceneView &s, uint32_t object, uint32_t primitive) {
    uint32_t first = 0u, length = s.lt_lookup_count;
    while (length > 0u) {
        const uint32_t half = length >> 1u;
        const uint32_t middle = first + half;
        const uint4 entry = s.lt_lookup[middle];
        if (entry.x < object || (entry.x == object && entry.y < primitive)) {
            first = middle + 1u;
            length = length - half - 1u;
        } else {
            length = half;
        }
    }
    if (first < s.lt_lookup_count) {
        const uint4 entry = s.lt_lookup[first];
        if (entry.x == object && entry.y == primitive) return entry.z;
    }
    return kLtInvalid;
}

}  // namespace psy
