// TEST INFRASTRUCTURE ONLY.  A C shim over the reference's own host
// sampling code (tabulated-Sobol LUT, flat light distribution, pixel-filter
// table, many-light tree build), compiled from the reference sources where they lie by
// oracle/Makefile (`make ref`) into oracle/_ref/.  Tests use it to pin the
// oracle's and the product's host tables to the reference's code.
#include <psycles/sampling/light_distribution.h>
#include <psycles/sampling/light_tree.h>
#include <psycles/sampling/pixel_filter.h>
#include <psycles/sampling/tabulated_sobol.h>

#include <cstring>
#include <span>
#include <vector>

#include "cycles_shader_tables_4_5_10.inl"

extern "C" {

int ref_sobol_generate_table(unsigned size, float *out) {
    try {
        const auto t = psycles::sampling::tabulated_sobol::generate_table(size);
        std::memcpy(out, t.data(), t.size() * sizeof(float) * 4u);
        return 0;
    } catch (...) {
        return 1;
    }
}

unsigned ref_sobol_sequence_size(unsigned samples) {
    return psycles::sampling::tabulated_sobol::sequence_size_for_samples(samples);
}

void ref_pixel_filter_table(unsigned filter, float width, float *out) {
    const auto t = psycles::sampling::make_pixel_filter_table(
        static_cast<psycles::contract::PixelFilter>(filter), width);
    std::memcpy(out, t.data(), sizeof(float) * t.size());
}

// entries_out: (emitter_count + 1) * 4 floats: cumulative, selection_pdf,
// kind (as float), index (as float).  Returns emitter_count.
unsigned ref_light_distribution(const float *areas, unsigned triangle_count, unsigned analytic_count,
                                int include_environment, float *entries_out, float *pdfs_out) {
    const auto d = psycles::sampling::build_cycles_light_distribution(
        std::span<const float>{areas, triangle_count}, analytic_count, include_environment != 0);
    for (std::size_t i = 0; i < d.entries.size(); ++i) {
        entries_out[4 * i + 0] = d.entries[i].cumulative;
        entries_out[4 * i + 1] = d.entries[i].selection_pdf;
        entries_out[4 * i + 2] = static_cast<float>(static_cast<unsigned>(d.entries[i].kind));
        entries_out[4 * i + 3] = static_cast<float>(d.entries[i].index);
    }
    pdfs_out[0] = d.triangle_area_pdf;
    pdfs_out[1] = d.light_selection_pdf;
    return d.emitter_count;
}

// Light-tree build.  Emitter records are 20 floats: bounds lo[3], hi[3],
// bounds-empty, cone axis[3], theta_o, theta_e, orientation-empty, energy,
// centroid[3], distant, emitter id, pad.  Outputs: per node 14 measure
// floats (the first 14 of the record layout) and 6 words (parent, left,
// right, first emitter, emitter count, kind); per tree slot the 14 measure
// floats and the emitter id; the two identity-indexed mappings.  Returns 0,
// 1 when the builder throws, 2 when node_capacity is too small.
static void put_measure(const psycles::sampling::LightTreeMeasure &m, float *o) {
    o[0] = m.bounds.minimum.x; o[1] = m.bounds.minimum.y; o[2] = m.bounds.minimum.z;
    o[3] = m.bounds.maximum.x; o[4] = m.bounds.maximum.y; o[5] = m.bounds.maximum.z;
    o[6] = m.bounds.empty ? 1.0f : 0.0f;
    o[7] = m.orientation.axis.x; o[8] = m.orientation.axis.y; o[9] = m.orientation.axis.z;
    o[10] = m.orientation.theta_o; o[11] = m.orientation.theta_e;
    o[12] = m.orientation.empty ? 1.0f : 0.0f;
    o[13] = m.energy;
}

int ref_build_light_tree(const float *in, unsigned n, unsigned max_leaf, unsigned node_capacity, float *node_measure,
                         unsigned *node_topology, float *emitter_measure, unsigned *emitter_ids, unsigned *to_tree,
                         unsigned *to_leaf, unsigned *root, unsigned *node_count) {
    using namespace psycles::sampling;
    std::vector<LightTreeEmitter> source(n);
    for (unsigned i = 0; i < n; ++i) {
        const float *r = in + 20u * i;
        LightTreeEmitter &e = source[i];
        e.measure.bounds.minimum = {r[0], r[1], r[2]};
        e.measure.bounds.maximum = {r[3], r[4], r[5]};
        e.measure.bounds.empty = r[6] != 0.0f;
        e.measure.orientation.axis = {r[7], r[8], r[9]};
        e.measure.orientation.theta_o = r[10];
        e.measure.orientation.theta_e = r[11];
        e.measure.orientation.empty = r[12] != 0.0f;
        e.measure.energy = r[13];
        e.centroid = {r[14], r[15], r[16]};
        e.distant = r[17] != 0.0f;
        e.emitter_id = static_cast<std::uint32_t>(r[18]);
    }
    try {
        const CyclesLightTree t = build_cycles_light_tree(std::span<const LightTreeEmitter>{source}, max_leaf);
        if (t.nodes.size() > node_capacity) return 2;
        for (std::size_t k = 0; k < t.nodes.size(); ++k) {
            const LightTreeNode &nd = t.nodes[k];
            put_measure(nd.measure, node_measure + 14u * k);
            unsigned *w = node_topology + 6u * k;
            w[0] = nd.parent; w[1] = nd.left; w[2] = nd.right;
            w[3] = nd.first_emitter; w[4] = nd.emitter_count; w[5] = static_cast<unsigned>(nd.kind);
        }
        for (std::size_t k = 0; k < t.emitters.size(); ++k) {
            put_measure(t.emitters[k].measure, emitter_measure + 14u * k);
            emitter_ids[k] = t.emitters[k].emitter_id;
        }
        for (std::size_t k = 0; k < t.emitter_to_tree.size(); ++k) {
            to_tree[k] = t.emitter_to_tree[k];
            to_leaf[k] = t.emitter_to_leaf[k];
        }
        *root = t.root;
        *node_count = static_cast<unsigned>(t.nodes.size());
        return 0;
    } catch (...) {
        return 1;
    }
}

// Cycles' GGX albedo tables as the reference ships them
// (src/luisa/cycles_shader_tables_4_5_10.inl, table_ggx_E: 32 x 32,
// table_ggx_Eavg: 32), for scenes with MULTI_GGX glossy closures.
void ref_ggx_tables(float *e, float *eavg) {
    for (int i = 0; i < 1024; ++i) e[i] = psycles::luisa_backend::cycles45_tables::table_ggx_E[i];
    for (int i = 0; i < 32; ++i) eavg[i] = psycles::luisa_backend::cycles45_tables::table_ggx_Eavg[i];
}

}  // extern "C"
