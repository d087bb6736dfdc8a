// Host build of the many-light tree.  Restates the Cycles light-tree
// construction of the reference: measure merges
// (src/sampling/light_tree.cpp:289-388), the SAOH cost (:376-402), the
// 12-bucket recursive build with a dedicated distant branch (:86-287), and
// the emitter measures of src/luisa/path_tracer_light_tree_scene.cpp:131-256.
// Compiled with -ffp-contract=off: the float operation order matches the
// reference construction, so the trees agree bit for bit.
#include "psy_light_tree.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../../include/psycles_cuda.h"

namespace psy {
namespace {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kHalfPiF = 0.5f * kPiF;
constexpr float kTwoPiF = 2.0f * kPiF;
constexpr size_t kBuckets = 12u;

struct V {
    float x, y, z;
};
V vv(const float *p) { return {p[0], p[1], p[2]}; }
void st(float *d, V v) {
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
}
V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V mul(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dotp(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float len(V a) { return std::sqrt(std::max(dotp(a, a), 0.0f)); }
V normalize_or(V v, V fallback) {
    const float m = len(v);
    return m > 1.0e-20f ? mul(v, 1.0f / m) : fallback;
}
V crossp(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float comp(const float *v, size_t axis) { return v[axis]; }
bool finite3(const float *v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

LtBounds merge_bounds(const LtBounds &a, const LtBounds &b) {
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

LtOrientation merge_orientation(const LtOrientation &a, const LtOrientation &b) {
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

LtMeasure valid_measure(const LtMeasure &m) {
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

// Subtrees of large nodes near the root are built on their own threads,
// each into a node list of its own that is spliced in after the left
// subtree: the node order (pre-order) and every field equal the sequential
// build's.  Emitter ranges of sibling subtrees are disjoint, so they share
// the emitter array and the identity maps.
constexpr uint32_t kParallelDepth = 3u;      // up to 8 subtrees in flight
constexpr uint32_t kParallelMinCount = 4096u;

class Builder {
  public:
    LightTree &tree;                 // emitters and identity maps (shared)
    std::vector<LtNode> &nodes;      // this builder's node list
    uint32_t max_leaf;

    Builder(LightTree &t, std::vector<LtNode> &n, uint32_t leaf) : tree(t), nodes(n), max_leaf(leaf) {}

    uint32_t append(uint32_t parent) {
        const uint32_t index = uint32_t(nodes.size());
        LtNode n;
        n.parent = parent;
        nodes.push_back(n);
        return index;
    }

    uint32_t build_local(uint32_t begin, uint32_t end, uint32_t parent, uint32_t depth = 0u) {
        const uint32_t node_index = append(parent);
        const uint32_t count = end - begin;
        if (count == 0u) {
            nodes[node_index].kind = kLtLeaf;
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
        nodes[node_index].measure = node_measure;
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
            LtNode &n = nodes[node_index];
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
        nodes[node_index].kind = kLtInner;
        uint32_t l = kLtInvalid, r = kLtInvalid;
        if (depth < kParallelDepth && end - begin >= kParallelMinCount) {
            std::vector<LtNode> right_nodes;
            Builder right(tree, right_nodes, max_leaf);
            std::thread worker([&]() { right.build_local(split_middle, end, kLtInvalid, depth + 1u); });
            l = build_local(begin, split_middle, node_index, depth + 1u);
            worker.join();
            // splice: the right subtree's nodes follow the left subtree's
            const uint32_t offset = uint32_t(nodes.size());
            auto shift = [offset](uint32_t v) { return v == kLtInvalid ? v : v + offset; };
            for (LtNode &n : right_nodes) {
                n.parent = shift(n.parent);
                n.left = shift(n.left);
                n.right = shift(n.right);
            }
            right_nodes.front().parent = node_index;
            nodes.insert(nodes.end(), right_nodes.begin(), right_nodes.end());
            for (uint32_t i = split_middle; i < end; ++i) tree.emitter_to_leaf[tree.emitters[i].emitter_id] += offset;
            r = offset;
        } else {
            l = build_local(begin, split_middle, node_index, depth + 1u);
            r = build_local(split_middle, end, node_index, depth + 1u);
        }
        nodes[node_index].left = l;
        nodes[node_index].right = r;
        return node_index;
    }
};

float average_absolute(V v) { return (std::abs(v.x) + std::abs(v.y) + std::abs(v.z)) / 3.0f; }

}  // namespace

LtMeasure lt_merge(const LtMeasure &a, const LtMeasure &b) {
    if (!(a.energy > 0.0f)) return b;
    if (!(b.energy > 0.0f)) return a;
    LtMeasure r;
    r.bounds = merge_bounds(a.bounds, b.bounds);
    r.orientation = merge_orientation(a.orientation, b.orientation);
    r.energy = a.energy + b.energy;
    return r;
}

float lt_cost(const LtMeasure &m) {
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

LightTree lt_build(const std::vector<LtEmitter> &source, uint32_t max_leaf) {
    LightTree result;
    Builder b(result, result.nodes, std::max(max_leaf, 1u));
    b.tree.emitters.reserve(source.size());
    for (const LtEmitter &s : source) {
        LtEmitter e = s;
        e.measure = valid_measure(s.measure);
        if (!finite3(e.centroid)) e.centroid[0] = e.centroid[1] = e.centroid[2] = 0.0f;
        b.tree.emitters.push_back(e);
    }
    if (b.tree.emitters.empty()) return result;
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
    return result;
}

LtEmitter lt_triangle_emitter(uint32_t id, const float *p0, const float *p1, const float *p2, const float *emission,
                              uint32_t sampling, bool mirror) {
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

LtEmitter lt_analytic_emitter(uint32_t id, const void *desc) {
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

}  // namespace psy
