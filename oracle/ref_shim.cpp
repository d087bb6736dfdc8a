// TEST INFRASTRUCTURE ONLY.  A C shim over the reference's own host
// sampling code (tabulated-Sobol LUT, flat light distribution, pixel-filter
// table), compiled from the reference sources where they lie by
// oracle/Makefile (`make ref`) into oracle/_ref/.  Tests use it to pin the
// oracle's and the product's host tables to the reference's code.
#include <psycles/sampling/light_distribution.h>
#include <psycles/sampling/pixel_filter.h>
#include <psycles/sampling/tabulated_sobol.h>

#include <cstring>
#include <span>

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

}  // extern "C"
