// Host-side launch wrappers of the wavefront kernels (psy_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "psy_scene.h"

namespace psy {

int launch_grid(uint32_t work, int block, int sms);
void launch_raygen(cudaStream_t st, int sms, const RenderParams &p, const PathBuffers &b, uint32_t pixels,
                   uint32_t paths, uint32_t sample_base, uint32_t trace_path, psy_path_trace *trace);
void launch_set_counters(cudaStream_t st, uint32_t *counters, uint32_t n);
void launch_intersect(cudaStream_t st, int sms, const SceneView &s, const PathBuffers &b, uint32_t max_work);
void launch_shade(cudaStream_t st, int sms, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                  uint32_t max_work, uint32_t step, uint32_t trace_path, psy_path_trace *trace);
void launch_shadow(cudaStream_t st, int sms, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                   uint32_t max_work, uint32_t step, uint32_t trace_path, psy_path_trace *trace);
void launch_swap(cudaStream_t st, uint32_t *counters);
void launch_begin_round(cudaStream_t st, uint32_t *counters, uint32_t *round, BatchItem *items,
                        const uint32_t *plan_rounds, const BatchItem *plan_items, uint32_t *cursor, uint32_t max_items);
void launch_count_rays(cudaStream_t st, const uint32_t *counters, unsigned long long *stats);
void launch_film(cudaStream_t st, int sms, const PathBuffers &b, uint32_t pixels, uint32_t samples, float4 *combined,
                 float4 *normal, float4 *albedo, uint32_t *sample_count, uint32_t trace_path, psy_path_trace *trace);
// Batched wavefront.  round (device memory): paths, film pixels, items.
void launch_raygen_batch(cudaStream_t st, int sms, const JobGpu *jobs, const BatchItem *items, const uint32_t *round,
                         const PathBuffers &b, uint32_t max_paths);
void launch_intersect_batch(cudaStream_t st, int sms, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work);
void launch_shade_batch(cudaStream_t st, int sms, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work,
                        uint32_t step);
void launch_shadow_batch(cudaStream_t st, int sms, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work,
                         uint32_t step);
void launch_film_batch(cudaStream_t st, int sms, const JobGpu *jobs, const BatchItem *items, const uint32_t *round,
                       const PathBuffers &b, uint32_t max_pixels);
void launch_debug_light_tree(cudaStream_t st, const SceneView &s, const float4 *queries, const uint32_t *pdf_emitters,
                             uint32_t count, uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf);
void launch_debug_sobol(cudaStream_t st, const float4 *table, uint32_t size, const uint32_t *queries, uint32_t count,
                        float4 *out, uint32_t *out_index);

}  // namespace psy
