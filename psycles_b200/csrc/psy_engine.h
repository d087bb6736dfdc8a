// Multi-job wavefront engine shared by batched renders (psy_batch.cpp) and
// the render server (psy_server.cpp).
//
// Jobs occupy slots of a device job table (render parameters, scene view,
// film).  A wavefront is a list of items, one per job at most: a contiguous
// sample range of that job over its window pixels, laid out item after item
// and sample-major inside an item.  Every kernel reads its path's job record;
// the film kernel adds each pixel's samples one at a time in sample order,
// so a job's film does not depend on how its samples were grouped or which
// other jobs shared its wavefronts.
//
// A call enqueues a plan of one or more wavefronts: their headers and items
// are uploaded once and a device cursor selects the current wavefront, so
// with graphs on one captured CUDA graph serves every wavefront of every
// call with the same step count.
#pragma once

#include "psy_host_internal.h"

#include <cstdint>
#include <vector>

namespace psy::host {

struct PlanJob {
    uint32_t slot;       // job-table slot the items name
    uint32_t pixels;     // window pixels
    uint64_t next, end;  // sample cursor
};

// One wavefront over `jobs`, visited round-robin from `start`: each
// unfinished job gets as many samples as fit in `capacity` paths.  Returns
// the paths used; `film_pixels` is the sum of the items' pixels.
uint32_t plan_wavefront(std::vector<PlanJob> &jobs, uint32_t start, uint32_t capacity,
                        std::vector<BatchItem> &items, uint32_t &film_pixels);

struct EnginePlan {
    std::vector<uint32_t> rounds;    // 4 words per wavefront: paths, film pixels, items, glossy
    std::vector<BatchItem> items;    // max_jobs records per wavefront
    uint64_t samples = 0;
    uint32_t waves() const { return uint32_t(rounds.size() / 4u); }
    // Appends one planned wavefront (padded to `max_jobs` records);
    // `glossy`: one of its jobs' scenes holds glossy closures, so the
    // wavefront shades with the glossy-capable kernel.
    void add(const std::vector<BatchItem> &wave, uint32_t paths, uint32_t film_pixels, uint32_t max_jobs,
             bool glossy);
};

struct EngineRun {
    uint32_t wavefronts = 0, graph_launches = 0, kernel_launches = 0;
};

class WavefrontEngine {
  public:
    ~WavefrontEngine();
    psy_status init(psy_context *context, uint32_t capacity, uint32_t max_jobs, bool use_graph,
                    uint32_t check_interval);
    uint32_t max_jobs() const { return max_jobs_; }
    uint32_t capacity() const { return arena_.capacity; }
    // Path state for at least `paths` paths (and the job array).
    psy_status reserve(uint32_t paths);
    // Asynchronous upload of job records to slots [first, first + n).
    psy_status set_jobs(uint32_t first, const JobGpu *jobs, uint32_t n);
    // Enqueues every wavefront of `plan` with `steps` path steps (no host
    // synchronisation with graphs; without graphs a live-path check every
    // check_interval steps ends a wavefront early).
    psy_status run(const EnginePlan &plan, uint32_t steps, EngineRun &out);
    // Event-timed device span and ray counts since the last reset_counters.
    psy_status reset_counters();
    psy_status elapsed(float *ms, uint64_t *closest_rays, uint64_t *shadow_rays);
    cudaStream_t stream() const;

  private:
    uint32_t issue(uint32_t steps, bool allow_exit, psy_status &status);
    psy_status ensure_graph(uint32_t steps);
    psy_status ensure_plan_room(size_t waves);

    psy_context *context_ = nullptr;
    uint32_t max_jobs_ = 0, check_interval_ = 4;
    bool use_graph_ = false;
    PathArena arena_;
    DeviceBuffer jobs_, items_, round_, cursor_, plan_rounds_, plan_items_;
    size_t plan_waves_ = 0;
    cudaEvent_t ev_begin_ = nullptr, ev_end_ = nullptr;
    bool began_ = false;
    cudaGraphExec_t graph_ = nullptr;
    uint32_t graph_steps_ = 0, graph_capacity_ = 0;
    uint64_t plan_generation_ = 0, graph_generation_ = 0;
};

// Device bytes a job needs besides the resident scene and the shared path
// state: its film (three float4 passes and a sample counter per window
// pixel), Sobol table and pixel-filter table.
uint64_t job_device_bytes(uint32_t pixels, uint32_t total_samples);

}  // namespace psy::host
