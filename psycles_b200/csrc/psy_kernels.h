// Host-side launch wrappers of the wavefront kernels (psy_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "psy_scene.h"

namespace psy {

// Launch shapes (psy_tuning): grid caps in blocks per SM, and the queue
// size from which the shading queue is sorted by material.
struct LaunchConfig {
    int sms = 148;
    uint32_t stream_blocks_per_sm = 16;     // raygen / film / shade grid-stride kernels
    uint32_t traversal_blocks_per_sm = 12;  // persistent closest-hit and shadow kernels
    uint32_t shade_blocks_per_sm = 32;
    uint32_t sort_threshold = 1u << 16;     // 0: never sort
    uint32_t shadow_sort_threshold = 0;     // shadow queue by direction (off: it measured slower); 0: never
    uint32_t ray_sort_threshold = 0;        // closest-hit queue by origin cell and octant (off: it measured slower)
    uint32_t stream_block = 256;            // threads per block of raygen and film
};

int launch_grid(uint32_t work, int block, const LaunchConfig &lc);
void launch_raygen(cudaStream_t st, const LaunchConfig &lc, const RenderParams &p, const PathBuffers &b, uint32_t pixels,
                   uint32_t paths, uint32_t sample_base, uint32_t trace_path, psy_path_trace *trace);
void launch_set_counters(cudaStream_t st, uint32_t *counters, uint32_t n);
void launch_intersect(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const PathBuffers &b, uint32_t max_work);
void launch_shade(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                  uint32_t max_work, uint32_t step, uint32_t trace_path, psy_path_trace *trace);
void launch_shadow(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                   uint32_t max_work, uint32_t step, uint32_t trace_path, psy_path_trace *trace);
void launch_swap(cudaStream_t st, uint32_t *counters);
void launch_begin_round(cudaStream_t st, uint32_t *counters, uint32_t *round, BatchItem *items,
                        const uint32_t *plan_rounds, const BatchItem *plan_items, uint32_t *cursor, uint32_t max_items);
void launch_count_rays(cudaStream_t st, const uint32_t *counters, unsigned long long *stats);
// Pass readback: `mismatch` (one word, cleared first) is set when a pixel's
// sample count differs from `expected`; the resolve writes a pass as the
// film's consumer sees it (kind: 0 Combined, 1 Normal / Albedo, 2 Sample
// Count), float4 per pixel (one float for the sample count).
void launch_check_counts(cudaStream_t st, const uint32_t *counts, uint32_t n, uint32_t expected, uint32_t *mismatch);
void launch_resolve_pass(cudaStream_t st, const float4 *film, const uint32_t *counts, uint32_t n, uint32_t kind,
                         float exposure, float *out);
void launch_film(cudaStream_t st, const LaunchConfig &lc, const PathBuffers &b, uint32_t pixels, uint32_t samples, float4 *combined,
                 float4 *normal, float4 *albedo, uint32_t *sample_count, uint32_t trace_path, psy_path_trace *trace);
// Batched wavefront.  round (device memory): paths, film pixels, items.
void launch_raygen_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const BatchItem *items, const uint32_t *round,
                         const PathBuffers &b, uint32_t max_paths);
void launch_intersect_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work);
void launch_shade_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work,
                        uint32_t step);
void launch_shadow_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work,
                         uint32_t step);
void launch_film_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const BatchItem *items, const uint32_t *round,
                       const PathBuffers &b, uint32_t max_pixels);
void launch_debug_light_tree(cudaStream_t st, const SceneView &s, const float4 *queries, const uint32_t *pdf_emitters,
                             uint32_t count, uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf);
void launch_debug_light_distribution(cudaStream_t st, const SceneView &s, const float *u, uint32_t count,
                                     uint32_t *out_kind, uint32_t *out_index, float *out_pdf);
void launch_debug_sobol(cudaStream_t st, const float4 *table, uint32_t size, const uint32_t *queries, uint32_t count,
                        float4 *out, uint32_t *out_index);
// Reads (after synchronising `st`) and clears the device's count of
// traversal pushes that found the stack full.
cudaError_t take_stack_overflows(cudaStream_t st, uint32_t *count);

}  // namespace psy
