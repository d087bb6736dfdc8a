// TEST INFRASTRUCTURE ONLY -- CPU oracle (see oracle_math.h).
//
// Many-light tree: host build (build_cycles_light_tree,
// src/sampling/light_tree.cpp:86-402, and the emitter measures of
// src/luisa/path_tracer_light_tree_scene.cpp:131-256) and the surface-point
// sampling / pdf of src/luisa/path_tracer_light_tree.cpp:19-880.  The
// builder is checked against the reference's own light_tree.cpp compiled
// into oracle/_ref.
#pragma once

#include "../include/psycles_cuda.h"
#include "oracle_math.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <vector>

namespace oracle {
namespace lt {

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

inline LtMeasure lt_merge(const LtMeasure &a, const LtMeasure &b);
inline float lt_cost(const LtMeasure &m);

namespace detail {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kHalfPiF = 0.5f * kPiF;
constexpr float kTwoPiF = 2.0f * kPiF;
constexpr size_t kBuckets = 12u;

struct V {
    float x, y, z;
};
inline V vv(const float *p) { return {p[0], p[1], p[2]}; }
inline void st(float *d, V v) {
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
}
inline V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V mul(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dotp(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float len(V a) { return std::sqrt(std::max(dotp(a, a), 0.0f)); }
inline V normalize_or(V v, V fallback) {
    const float m = len(v);
    return m > 1.0e-20f ? mul(v, 1.0f / m) : fallback;
}
inline V crossp(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float comp(const float *v, size_t axis) { return v[axis]; }
inline bool finite3(const float *v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

inline LtBounds merge_bounds(const LtBounds &a, const LtBounds &b) {
    if (a.empty) return b;
    if (b.empty) return a;
    LtBounds r;
    r.empty = false;
    for (int k = 0; k < 3; ++k) {
        r.lo[k] = std::min(a.lo[k], b.lo[k]);
        r.hi[k] = std::max(a.hi[k], b.hi[k]);
    }
    return r;
}

inline LtOrientation merge_orientation(const LtOrientation &a, const LtOrientation &b) {
    if (a.empty) return b;
    if (b.empty) return a;
    const LtOrientation *wide = &a, *narrow = &b;
    if (b.theta_o > a.theta_o) std::swap(wide, narrow);
    const V wa = vv(wide->axis), na = vv(narrow->axis);
    const float cosine = std::clamp(dotp(wa, na), -1.0f, 1.0f);
    const float axis_angle = std::acos(cosine);
    const float emission_angle = std::max(a.theta_e, b.theta_e);
    LtOrientation r;
    r.empty = false;
    r.theta_e = emission_angle;
    if (wide->theta_o + 5.0e-4f >= std::min(kPiF, axis_angle + narrow->theta_o)) {
        st(r.axis, wa);
        r.theta_o = wide->theta_o;
        return r;
    }
    const float theta_o = 0.5f * (axis_angle + wide->theta_o + narrow->theta_o);
    if (theta_o >= kPiF) {
        st(r.axis, wa);
        r.theta_o = kPiF;
        return r;
    }
    const float rotation = theta_o - wide->theta_o;
    V orthogonal = sub(na, mul(wa, cosine));
    if (cosine < -0.9995f) {
        const V c = std::abs(wa.x) < 0.9f ? V{1.0f, 0.0f, 0.0f} : V{0.0f, 1.0f, 0.0f};
        orthogonal = normalize_or({wa.y * c.z - wa.z * c.y, wa.z * c.x - wa.x * c.z, wa.x * c.y - wa.y * c.x},
                                  {0.0f, 0.0f, 1.0f});
    } else {
        orthogonal = normalize_or(orthogonal, {0.0f, 0.0f, 1.0f});
    }
    st(r.axis, normalize_or(add(mul(wa, std::cos(rotation)), mul(orthogonal, std::sin(rotation))), wa));
    r.theta_o = theta_o;
    return r;
}

inline LtMeasure valid_measure(const LtMeasure &m) {
    if (!std::isfinite(m.energy) || m.energy <= 0.0f) return {};
    LtMeasure r = m;
    if (!r.bounds.empty && (!finite3(r.bounds.lo) || !finite3(r.bounds.hi))) r.bounds = {};
    if (!r.orientation.empty) {
        st(r.orientation.axis, normalize_or(vv(r.orientation.axis), {0.0f, 0.0f, 1.0f}));
        r.orientation.theta_o = std::clamp(r.orientation.theta_o, 0.0f, kPiF);
        r.orientation.theta_e = std::clamp(r.orientation.theta_e, 0.0f, kPiF);
    }
    return r;
}

struct Bucket {
    LtMeasure measure;
    uint32_t count = 0u;
};

class Builder {
  public:
    LightTree tree;
    uint32_t max_leaf;

    uint32_t append(uint32_t parent) {
        const uint32_t index = uint32_t(tree.nodes.size());
        LtNode n;
        n.parent = parent;
        tree.nodes.push_back(n);
        return index;
    }

    uint32_t build_local(uint32_t begin, uint32_t end, uint32_t parent) {
        const uint32_t node_index = append(parent);
        const uint32_t count = end - begin;
        if (count == 0u) {
            tree.nodes[node_index].kind = kLtLeaf;
            return node_index;
        }
        LtMeasure node_measure;
        LtBounds cb;
        for (uint32_t i = begin; i < end; ++i) {
            const LtEmitter &e = tree.emitters[i];
            node_measure = lt_merge(node_measure, e.measure);
            LtBounds point;
            point.empty = false;
            for (int k = 0; k < 3; ++k) point.lo[k] = point.hi[k] = e.centroid[k];
            cb = merge_bounds(cb, point);
        }
        tree.nodes[node_index].measure = node_measure;
        size_t split_axis = std::numeric_limits<size_t>::max();
        uint32_t split_middle = begin + count / 2u;
        float best_cost = std::numeric_limits<float>::infinity();
        const float parent_cost = lt_cost(node_measure);
        const float extent[3] = {cb.hi[0] - cb.lo[0], cb.hi[1] - cb.lo[1], cb.hi[2] - cb.lo[2]};
        const float max_extent = std::max({extent[0], extent[1], extent[2]});
        if (count > 1u && parent_cost > 0.0f && max_extent > 0.0f) {
            for (size_t axis = 0; axis < 3u; ++axis) {
                const float axis_extent = extent[axis];
                if (!(axis_extent > 0.0f)) continue;
                std::array<Bucket, kBuckets> buckets{};
                for (uint32_t i = begin; i < end; ++i) {
                    const float relative = (comp(tree.emitters[i].centroid, axis) - cb.lo[axis]) / axis_extent;
                    const size_t b = std::min<size_t>(
                        static_cast<size_t>(std::max(relative, 0.0f) * static_cast<float>(kBuckets)), kBuckets - 1u);
                    buckets[b].measure = lt_merge(buckets[b].measure, tree.emitters[i].measure);
                    ++buckets[b].count;
                }
                std::array<Bucket, kBuckets - 1u> left{}, right{};
                left.front() = buckets.front();
                for (size_t b = 1u; b + 1u < kBuckets; ++b) {
                    left[b].measure = lt_merge(left[b - 1u].measure, buckets[b].measure);
                    left[b].count = left[b - 1u].count + buckets[b].count;
                }
                right.back() = buckets.back();
                for (size_t b = kBuckets - 2u; b-- > 0u;) {
                    right[b].measure = lt_merge(right[b + 1u].measure, buckets[b + 1u].measure);
                    right[b].count = right[b + 1u].count + buckets[b + 1u].count;
                }
                const float regularization = max_extent / axis_extent;
                for (size_t split = 0u; split + 1u < kBuckets; ++split) {
                    if (left[split].count == 0u || right[split].count == 0u) continue;
                    const float cost = regularization * (lt_cost(left[split].measure) + lt_cost(right[split].measure));
                    if (cost < parent_cost && cost < best_cost) {
                        best_cost = cost;
                        split_axis = axis;
                        split_middle = begin + left[split].count;
                    }
                }
            }
        }
        const bool should_split = count > max_leaf || split_axis != std::numeric_limits<size_t>::max();
        if (!should_split) {
            LtNode &n = tree.nodes[node_index];
            n.kind = kLtLeaf;
            n.first = begin;
            n.count = count;
            for (uint32_t i = begin; i < end; ++i) {
                tree.emitter_to_tree[tree.emitters[i].emitter_id] = i;
                tree.emitter_to_leaf[tree.emitters[i].emitter_id] = node_index;
            }
            return node_index;
        }
        if (split_axis != std::numeric_limits<size_t>::max()) {
            const size_t ax = split_axis;
            std::nth_element(tree.emitters.begin() + begin, tree.emitters.begin() + split_middle,
                             tree.emitters.begin() + end, [ax](const LtEmitter &a, const LtEmitter &b) {
                                 const float av = comp(a.centroid, ax), bv = comp(b.centroid, ax);
                                 return av < bv || (av == bv && a.emitter_id < b.emitter_id);
                             });
        }
        tree.nodes[node_index].kind = kLtInner;
        const uint32_t l = build_local(begin, split_middle, node_index);
        const uint32_t r = build_local(split_middle, end, node_index);
        tree.nodes[node_index].left = l;
        tree.nodes[node_index].right = r;
        return node_index;
    }
};

inline float average_absolute(V v) { return (std::abs(v.x) + std::abs(v.y) + std::abs(v.z)) / 3.0f; }

}  // namespace detail
using namespace detail;

// merge_light_tree_measures / light_tree_measure_cost
// (src/sampling/light_tree.cpp:86-180).
inline LtMeasure lt_merge(const LtMeasure &a, const LtMeasure &b) {
    if (!(a.energy > 0.0f)) return b;
    if (!(b.energy > 0.0f)) return a;
    LtMeasure r;
    r.bounds = merge_bounds(a.bounds, b.bounds);
    r.orientation = merge_orientation(a.orientation, b.orientation);
    r.energy = a.energy + b.energy;
    return r;
}

inline float lt_cost(const LtMeasure &m) {
    if (!(m.energy > 0.0f) || m.orientation.empty) return 0.0f;
    float spatial = 0.0f;
    if (!m.bounds.empty) {
        const V e = sub(vv(m.bounds.hi), vv(m.bounds.lo));
        spatial = 2.0f * (e.x * e.y + e.x * e.z + e.y * e.z);
        if (spatial == 0.0f) spatial = len(e);
    }
    const float theta_w = std::min(kPiF, m.orientation.theta_o + m.orientation.theta_e);
    const float cos_o = std::cos(m.orientation.theta_o);
    const float sin_o = std::sin(m.orientation.theta_o);
    const float orientation = kTwoPiF * (1.0f - cos_o) +
                              kHalfPiF * (2.0f * theta_w * sin_o - std::cos(m.orientation.theta_o - 2.0f * theta_w) -
                                          2.0f * m.orientation.theta_o * sin_o + cos_o);
    return m.energy * spatial * orientation;
}

// build_cycles_light_tree (src/sampling/light_tree.cpp:289-402).
inline LightTree lt_build(const std::vector<LtEmitter> &source, uint32_t max_leaf = 8u) {
    Builder b;
    b.max_leaf = std::max(max_leaf, 1u);
    b.tree.emitters.reserve(source.size());
    for (const LtEmitter &s : source) {
        LtEmitter e = s;
        e.measure = valid_measure(s.measure);
        if (!finite3(e.centroid)) e.centroid[0] = e.centroid[1] = e.centroid[2] = 0.0f;
        b.tree.emitters.push_back(e);
    }
    if (b.tree.emitters.empty()) return std::move(b.tree);
    std::vector<bool> seen(b.tree.emitters.size(), false);
    for (const LtEmitter &e : b.tree.emitters) {
        if (e.emitter_id >= seen.size() || seen[e.emitter_id])
            throw std::invalid_argument("light-tree emitter identities must be a dense permutation");
        seen[e.emitter_id] = true;
    }
    b.tree.emitter_to_tree.assign(b.tree.emitters.size(), kLtInvalid);
    b.tree.emitter_to_leaf.assign(b.tree.emitters.size(), kLtInvalid);
    const uint32_t distant_begin = uint32_t(
        std::stable_partition(b.tree.emitters.begin(), b.tree.emitters.end(), [](const LtEmitter &e) { return !e.distant; }) -
        b.tree.emitters.begin());
    const uint32_t n = uint32_t(b.tree.emitters.size());
    b.tree.root = b.append(kLtInvalid);
    b.tree.nodes[b.tree.root].kind = kLtInner;
    const uint32_t local = b.build_local(0u, distant_begin, b.tree.root);
    const uint32_t distant = b.append(b.tree.root);
    {
        LtNode &d = b.tree.nodes[distant];
        d.kind = kLtDistant;
        d.first = distant_begin;
        d.count = n - distant_begin;
        for (uint32_t i = distant_begin; i < n; ++i) {
            d.measure = lt_merge(d.measure, b.tree.emitters[i].measure);
            b.tree.emitter_to_tree[b.tree.emitters[i].emitter_id] = i;
            b.tree.emitter_to_leaf[b.tree.emitters[i].emitter_id] = distant;
        }
    }
    LtNode &root = b.tree.nodes[b.tree.root];
    root.left = local;
    root.right = distant;
    root.measure = lt_merge(b.tree.nodes[local].measure, b.tree.nodes[distant].measure);
    return std::move(b.tree);
}

// make_triangle_light_tree_emitter (path_tracer_light_tree_scene.cpp:131-186):
// world-space vertices, the material's constant emission estimate and its
// EmissionSampling mode; `mirror` for a negative-determinant transform.
inline LtEmitter lt_triangle_emitter(uint32_t id, const float *p0, const float *p1, const float *p2,
                                     const float *emission, uint32_t sampling, bool mirror) {
    const V v0 = vv(p0), v1 = vv(p1), v2 = vv(p2);
    const V c = crossp(sub(v1, v0), sub(v2, v0));
    const float area = 0.5f * len(c);
    const bool front_only = sampling == PSY_EMISSION_SAMPLING_FRONT;
    const bool back_only = sampling == PSY_EMISSION_SAMPLING_BACK;
    V axis = front_only || back_only ? normalize_or(c, {0.0f, 0.0f, 1.0f}) : normalize_or(sub(v0, v1), {1.0f, 0.0f, 0.0f});
    if (back_only) axis = mul(axis, -1.0f);
    if ((front_only || back_only) && mirror) axis = mul(axis, -1.0f);
    LtEmitter e;
    e.measure.bounds.empty = false;
    for (int k = 0; k < 3; ++k) {
        e.measure.bounds.lo[k] = std::min({p0[k], p1[k], p2[k]});
        e.measure.bounds.hi[k] = std::max({p0[k], p1[k], p2[k]});
    }
    st(e.measure.orientation.axis, axis);
    e.measure.orientation.theta_o = front_only || back_only ? 0.0f : kHalfPiF;
    e.measure.orientation.theta_e = kHalfPiF;
    e.measure.orientation.empty = false;
    e.measure.energy = area * average_absolute(vv(emission));
    st(e.centroid, mul(add(add(v0, v1), v2), 1.0f / 3.0f));
    e.emitter_id = id;
    e.distant = false;
    return e;
}

// make_analytic_light_tree_emitter (path_tracer_light_tree_scene.cpp:188-256)
// for a light with the constant shader (emission estimate one).
inline LtEmitter lt_analytic_emitter(uint32_t id, const void *desc) {
    const psy_light_desc &l = *static_cast<const psy_light_desc *>(desc);
    const V position = vv(l.position), ax = vv(l.axis_x), ay = vv(l.axis_y), az = vv(l.axis_z);
    V strength = mul(vv(l.color), l.power);  // constant light shader: emission estimate 1
    const bool normalize = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    if (!normalize) {
        float area = 1.0f;
        if (l.type == PSY_LIGHT_POINT || l.type == PSY_LIGHT_SPOT) {
            area = l.radius > 0.0f ? 4.0f * kPiF * l.radius * l.radius : 4.0f;
        } else if (l.type == PSY_LIGHT_AREA) {
            area = std::abs(l.size_u * l.size_v);
            if ((l.flags & PSY_LIGHT_FLAG_ELLIPSE) != 0u) area *= 0.25f * kPiF;
        } else if (l.type == PSY_LIGHT_DISTANT && l.angle > 0.0f) {
            const float s = std::sin(0.5f * l.angle);
            area = kPiF * s * s;
        }
        strength = mul(strength, area);
    }
    LtEmitter e;
    st(e.measure.orientation.axis, mul(az, -1.0f));
    e.measure.orientation.empty = false;
    bool distant = false;
    if (l.type == PSY_LIGHT_AREA) {
        e.measure.orientation.theta_e = 0.5f * l.spread;
        const V hu = mul(ax, 0.5f * l.size_u), hv = mul(ay, 0.5f * l.size_v);
        const V corners[4] = {add(position, add(hu, hv)), add(position, sub(hu, hv)), add(position, sub(hv, hu)),
                              sub(position, add(hu, hv))};
        e.measure.bounds.empty = false;
        for (int k = 0; k < 3; ++k) {
            float lo = (&corners[0].x)[k], hi = lo;
            for (int c = 1; c < 4; ++c) {
                lo = std::min(lo, (&corners[c].x)[k]);
                hi = std::max(hi, (&corners[c].x)[k]);
            }
            e.measure.bounds.lo[k] = lo;
            e.measure.bounds.hi[k] = hi;
        }
        strength = mul(strength, 1.0f / kPiF);
    } else if (l.type == PSY_LIGHT_POINT) {
        e.measure.orientation.theta_o = kPiF;
        e.measure.orientation.theta_e = kHalfPiF;
    } else if (l.type == PSY_LIGHT_SPOT) {
        float theta_e = std::min(0.5f * l.spot_angle, kHalfPiF);
        if (std::abs(kHalfPiF - theta_e) >= 1.0e-6f)
            theta_e = std::atan(std::tan(theta_e) * std::max(l.axis_scale[0], l.axis_scale[1]) /
                                std::max(l.axis_scale[2], 1.0e-20f));
        e.measure.orientation.theta_e = theta_e;
    } else if (l.type == PSY_LIGHT_DISTANT) {
        e.measure.orientation.theta_e = 0.5f * l.angle;
        distant = true;
    }
    if (l.type == PSY_LIGHT_POINT || l.type == PSY_LIGHT_SPOT) {
        const V r = {l.radius, l.radius, l.radius};
        const V lo = sub(position, r), hi = add(position, r);
        e.measure.bounds.empty = false;
        e.measure.bounds.lo[0] = std::min(lo.x, hi.x);
        e.measure.bounds.lo[1] = std::min(lo.y, hi.y);
        e.measure.bounds.lo[2] = std::min(lo.z, hi.z);
        e.measure.bounds.hi[0] = std::max(lo.x, hi.x);
        e.measure.bounds.hi[1] = std::max(lo.y, hi.y);
        e.measure.bounds.hi[2] = std::max(lo.z, hi.z);
        strength = mul(strength, 0.25f / kPiF);
    }
    e.measure.energy = average_absolute(strength);
    st(e.centroid, position);
    e.emitter_id = id;
    e.distant = distant;
    return e;
}

// ------------------------------------------------------------ sampling
// Surface-point importance sampling of the tree and the reverse pdf of a
// forward-hit emitter (src/luisa/path_tracer_light_tree.cpp:19-760), over
// the unpacked tree.  Trigonometry of float arguments goes through the
// oracle's double-rounded cos_/sin_.

constexpr float kSafe = 1.0e-20f;
constexpr float kPi = 3.14159265358979323846f;

// (maximum, minimum) importance.
struct Importance {
    float hi = 0.0f, lo = 0.0f;
};

inline float sin_from_cos(float c) { return std::sqrt(maxf(1.0f - c * c, 0.0f)); }

inline float3 tree_normalize(float3 v, float3 fallback) {
    const float l2 = dot(v, v);
    return l2 > kSafe ? v * (1.0f / std::sqrt(maxf(l2, kSafe))) : fallback;
}

// bounded_importance, surface case (path_tracer_light_tree.cpp:86-193).
inline Importance bounded_importance(float3 n, bool transmission, float3 to_centroid, float cos_spread, float3 axis,
                                     float theta_o, float theta_e, float far_d, float near_d, float energy) {
    const float cu = clampf(cos_spread, -1.0f, 1.0f);
    const float su = sin_from_cos(cu);
    const float cos_in = transmission ? std::abs(dot(to_centroid, n)) : dot(to_centroid, n);
    const float sin_in = sin_from_cos(clampf(cos_in, -1.0f, 1.0f));
    // incidence cosines at the best and worst point of the cluster
    const float best_in = cos_in >= cu ? 1.0f : cos_in * cu + sin_in * su;
    const float worst_in = maxf(cos_in * cu - sin_in * su, 0.0f);
    bool visible = energy > 0.0f && (transmission || best_in >= 0.0f);
    const float cos_t = clampf(dot(axis, -to_centroid), -1.0f, 1.0f);
    const float sin_t = sin_from_cos(cos_t);
    const float cos_tm = cos_t * cu + sin_t * su;  // cos(theta - theta_u)
    const float co = cos_(theta_o), so = sin_(theta_o);
    const bool inside = cos_t >= cu || cos_tm >= co;
    const bool edge = !inside && (theta_o + theta_e > kPi || cos_tm > cos_(theta_o + theta_e));
    const float sin_tm = sin_from_cos(clampf(cos_tm, -1.0f, 1.0f));
    const float best_out = inside ? 1.0f : (edge ? cos_tm * co + sin_tm * so : 0.0f);
    visible = visible && (inside || edge);
    const float dn = maxf(near_d, kSafe), df = maxf(far_d, kSafe);
    Importance r;
    r.hi = visible ? std::abs(best_in * energy * best_out * (1.0f / (dn * dn))) : 0.0f;
    const float cos_tp = cos_t * cu - sin_t * su;  // cos(theta + theta_u)
    const bool lo_zero = theta_e - theta_o < 0.0f || cos_t < 0.0f || cu < 0.0f || cos_tp < cos_(theta_e - theta_o);
    const float sin_tp = sin_from_cos(clampf(cos_tp, -1.0f, 1.0f));
    const float worst_out = cos_tp * co - sin_tp * so;
    r.lo = (lo_zero || !visible) ? 0.0f : std::abs(worst_in * energy * worst_out / (df * df));
    return r;
}

// measure_importance (path_tracer_light_tree.cpp:195-277).
inline Importance measure_importance(const LtMeasure &m, bool distant, float3 p, float3 n, bool transmission) {
    if (m.orientation.empty || !(m.energy > 0.0f)) return {};
    const float3 axis = tree_normalize(f3(m.orientation.axis[0], m.orientation.axis[1], m.orientation.axis[2]),
                                       f3(0.0f, 0.0f, 1.0f));
    float3 to_centroid = -axis;
    float cos_spread = cos_(m.orientation.theta_o + m.orientation.theta_e);
    float d = 1.0f;
    if (!distant) {
        const float3 lo = f3(m.bounds.lo[0], m.bounds.lo[1], m.bounds.lo[2]);
        const float3 hi = f3(m.bounds.hi[0], m.bounds.hi[1], m.bounds.hi[2]);
        const float3 c = (lo + hi) * 0.5f;
        const float3 half = hi - c;
        const float3 an = f3(std::abs(n.x), std::abs(n.y), std::abs(n.z));
        const float3 ah = f3(std::abs(half.x), std::abs(half.y), std::abs(half.z));
        if (!(transmission || dot(n, c - p) + dot(an, ah) > 0.0f)) return {};
        d = length(c - p);
        to_centroid = tree_normalize(c - p, -axis);
        const float d2 = dot(p - c, p - c), r2 = dot(hi - c, hi - c);
        cos_spread = d2 <= r2 ? -1.0f : std::sqrt(maxf(1.0f - r2 / maxf(d2, kSafe), 0.0f));
        d = maxf(0.5f * length(c - hi), d);
    }
    return bounded_importance(n, transmission, to_centroid, cos_spread, axis, m.orientation.theta_o,
                              m.orientation.theta_e, d, d, m.energy);
}

inline Importance emitter_importance(const LightTree &t, uint32_t e, float3 p, float3 n, bool tr) {
    return measure_importance(t.emitters[e].measure, t.emitters[e].distant, p, n, tr);
}

// child_importance (path_tracer_light_tree.cpp:321-356).
inline Importance child_importance(const LightTree &t, uint32_t node, float3 p, float3 n, bool tr) {
    const LtNode &c = t.nodes[node];
    if (c.kind == kLtInner || c.count > 1u) return measure_importance(c.measure, c.kind == kLtDistant, p, n, tr);
    if (c.count == 1u) return emitter_importance(t, c.first, p, n, tr);
    return {};
}

// left_probability (path_tracer_light_tree.cpp:358-398); false when both
// children are unimportant.
inline bool left_probability(const LightTree &t, const LtNode &parent, float3 p, float3 n, bool tr, float &left) {
    const Importance a = child_importance(t, parent.left, p, n, tr);
    const Importance b = child_importance(t, parent.right, p, n, tr);
    const float hi = a.hi + b.hi, lo = a.lo + b.lo;
    const float p_hi = a.hi / maxf(hi, kSafe);
    const float p_lo = lo > 0.0f ? a.lo / maxf(lo, kSafe) : 0.5f * ((a.hi > 0.0f ? 1.0f : 0.0f) + (b.hi == 0.0f ? 1.0f : 0.0f));
    left = 0.5f * (p_hi + p_lo);
    return hi > 0.0f;
}

// One step of a weighted reservoir that reuses the random number.
inline void reservoir_step(uint32_t candidate, float weight, float &total, float &u, uint32_t &chosen) {
    total += weight;
    if (chosen == kLtInvalid) {
        chosen = candidate;
        return;
    }
    const float keep = weight / total;
    if (u <= keep) {
        chosen = candidate;
        u = u / keep;
    } else {
        u = (u - keep) / maxf(1.0f - keep, kSafe);
    }
    u = clampf(u, 0.0f, 1.0f);
}

// select_leaf_emitter (path_tracer_light_tree.cpp:430-527): the emitter and
// the leaf's factor of the selection pdf (the mean of the max- and
// min-importance proposals).
inline uint32_t select_leaf(const LightTree &t, const LtNode &leaf, float3 p, float3 n, bool tr, float &u,
                            float &factor) {
    const bool by_max = u > 0.5f;
    if (leaf.count > 1u) u = u * 2.0f - (by_max ? 1.0f : 0.0f);
    std::vector<Importance> imp(leaf.count);
    float sum_hi = 0.0f, sum_lo = 0.0f, total = 0.0f;
    uint32_t positive = 0u, chosen = kLtInvalid;
    for (uint32_t k = 0; k < leaf.count; ++k) {
        imp[k] = emitter_importance(t, leaf.first + k, p, n, tr);
        sum_hi += imp[k].hi;
        sum_lo += imp[k].lo;
        positive += imp[k].hi > 0.0f ? 1u : 0u;
        const float w = by_max ? imp[k].hi : imp[k].lo;
        if (w > 0.0f) reservoir_step(k, w, total, u, chosen);
    }
    float chosen_lo = chosen != kLtInvalid ? imp[chosen].lo : 0.0f;
    if (positive > 0u && sum_lo == 0.0f) {
        // no emitter has a positive minimum: the min proposal is uniform
        // over the emitters with positive maximum importance
        if (by_max) {
            chosen_lo = 1.0f;
            sum_lo = static_cast<float>(positive);
        } else {
            chosen = kLtInvalid;
            float uniform_total = 0.0f;
            for (uint32_t k = 0; k < leaf.count; ++k)
                if (imp[k].hi > 0.0f) reservoir_step(k, 1.0f, uniform_total, u, chosen);
            chosen_lo = 1.0f;
            sum_lo = uniform_total;
        }
    }
    if (chosen == kLtInvalid) return kLtInvalid;
    factor *= 0.5f * (imp[chosen].hi / maxf(sum_hi, kSafe) + chosen_lo / maxf(sum_lo, kSafe));
    return leaf.first + chosen;
}

// make_sample_callable, surface case (path_tracer_light_tree.cpp:547-637):
// the tree slot of the chosen emitter (kLtInvalid for none) and its pdf.
inline uint32_t tree_sample(const LightTree &t, float u, float3 p, float3 n, bool tr, float &pdf) {
    pdf = 1.0f;
    if (t.nodes.empty() || t.emitters.empty() || t.root >= t.nodes.size()) return kLtInvalid;
    float r = clampf(u, 0.0f, 1.0f);
    uint32_t node = t.root;
    for (size_t guard = 0; guard <= t.nodes.size(); ++guard) {
        const LtNode &c = t.nodes[node];
        if (c.kind != kLtInner) return select_leaf(t, c, p, n, tr, r, pdf);
        float left = 0.0f;
        if (!left_probability(t, c, p, n, tr, left)) return kLtInvalid;
        const float right = 1.0f - left;
        if (r <= right) {
            node = c.right;
            pdf *= right;
            r = r / maxf(right, kSafe);
        } else {
            node = c.left;
            pdf *= left;
            r = (r - right) / maxf(left, kSafe);
        }
        r = clampf(r, 0.0f, 1.0f);
    }
    return kLtInvalid;
}

// make_pdf_callable, surface case (path_tracer_light_tree.cpp:639-760).
inline float tree_pdf(const LightTree &t, uint32_t emitter_id, float3 p, float3 n, bool tr) {
    if (t.nodes.empty() || emitter_id >= t.emitter_to_tree.size()) return 0.0f;
    const uint32_t slot = t.emitter_to_tree[emitter_id];
    uint32_t node = t.emitter_to_leaf[emitter_id];
    if (slot >= t.emitters.size() || node >= t.nodes.size()) return 0.0f;
    const LtNode &leaf = t.nodes[node];
    float sum_hi = 0.0f, sum_lo = 0.0f;
    Importance mine;
    uint32_t positive = 0u;
    for (uint32_t k = 0; k < leaf.count; ++k) {
        const Importance i = emitter_importance(t, leaf.first + k, p, n, tr);
        sum_hi += i.hi;
        sum_lo += i.lo;
        positive += i.hi > 0.0f ? 1u : 0u;
        if (leaf.first + k == slot) mine = i;
    }
    if (!(mine.hi > 0.0f)) return 0.0f;
    float pdf = 0.5f * (mine.hi / maxf(sum_hi, kSafe) +
                        (sum_lo > 0.0f ? mine.lo / maxf(sum_lo, kSafe) : 1.0f / maxf(static_cast<float>(positive), 1.0f)));
    for (size_t guard = 0; node != t.root && guard <= t.nodes.size(); ++guard) {
        const uint32_t up = t.nodes[node].parent;
        if (up >= t.nodes.size()) return 0.0f;
        const LtNode &parent = t.nodes[up];
        float left = 0.0f;
        if (!left_probability(t, parent, p, n, tr, left)) return 0.0f;
        pdf *= node == parent.left ? left : 1.0f - left;
        node = up;
    }
    return node == t.root ? pdf : 0.0f;
}

}  // namespace lt
}  // namespace oracle
