// Multi-job wavefront engine (see psy_engine.h).
#include "psy_engine.h"

#include "psy_kernels.h"

#include <algorithm>

namespace psy::host {

uint32_t plan_wavefront(std::vector<PlanJob> &jobs, uint32_t start, uint32_t capacity,
                        std::vector<BatchItem> &items, uint32_t &film_pixels) {
    items.clear();
    film_pixels = 0u;
    uint32_t used = 0u;
    const uint32_t n = uint32_t(jobs.size());
    for (uint32_t k = 0; k < n; ++k) {
        PlanJob &pj = jobs[(start + k) % n];
        if (pj.next >= pj.end || pj.pixels == 0u) continue;
        const uint32_t fit = (capacity - used) / pj.pixels;
        if (fit == 0u) continue;
        const uint32_t take = uint32_t(std::min<uint64_t>(fit, pj.end - pj.next));
        BatchItem it{};
        it.job = pj.slot;
        it.path_begin = used;
        it.pixels = pj.pixels;
        it.samples = take;
        it.sample_base = uint32_t(pj.next);
        it.film_begin = film_pixels;
        items.push_back(it);
        used += take * pj.pixels;
        film_pixels += pj.pixels;
        pj.next += take;
    }
    return used;
}

void EnginePlan::add(const std::vector<BatchItem> &wave, uint32_t paths, uint32_t film_pixels, uint32_t max_jobs,
                     bool glossy) {
    rounds.insert(rounds.end(), {paths, film_pixels, uint32_t(wave.size()), glossy ? 1u : 0u});
    const size_t base = items.size();
    items.resize(base + max_jobs, BatchItem{});
    std::copy(wave.begin(), wave.end(), items.begin() + base);
    for (const BatchItem &it : wave) samples += uint64_t(it.samples) * it.pixels;
}

uint64_t job_device_bytes(uint32_t pixels, uint32_t total_samples) {
    const uint64_t film = uint64_t(pixels) * (3u * 16u + 4u);
    const uint64_t sobol = uint64_t(psy_sobol_sequence_size_for_samples(std::max(total_samples, 1u))) * 256u * 16u;
    return film + sobol + 4096u;
}

WavefrontEngine::~WavefrontEngine() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (ev_begin_) cudaEventDestroy(ev_begin_);
    if (ev_end_) cudaEventDestroy(ev_end_);
}

cudaStream_t WavefrontEngine::stream() const { return context_->stream; }

psy_status WavefrontEngine::init(psy_context *context, uint32_t capacity, uint32_t max_jobs, bool use_graph,
                                 uint32_t check_interval) {
    context_ = context;
    max_jobs_ = max_jobs;
    use_graph_ = use_graph;
    check_interval_ = check_interval ? check_interval : 4u;
    PSY_CUDA_TRY(cudaSetDevice(context->device));
    PSY_CUDA_TRY(jobs_.alloc(sizeof(JobGpu) * max_jobs));
    PSY_CUDA_TRY(cudaMemset(jobs_.ptr, 0, sizeof(JobGpu) * max_jobs));
    PSY_CUDA_TRY(items_.alloc(sizeof(BatchItem) * max_jobs));
    PSY_CUDA_TRY(round_.alloc(16));
    PSY_CUDA_TRY(cursor_.alloc(16));
    PSY_CUDA_TRY(cudaEventCreate(&ev_begin_));
    PSY_CUDA_TRY(cudaEventCreate(&ev_end_));
    return reserve(capacity);
}

psy_status WavefrontEngine::reserve(uint32_t paths) { return arena_.ensure(std::max(paths, arena_.capacity), true); }

psy_status WavefrontEngine::set_jobs(uint32_t first, const JobGpu *jobs, uint32_t n) {
    if (first + n > max_jobs_) return fail(PSY_ERROR_RANGE, "job slot beyond the engine's table");
    if (n == 0u) return PSY_OK;
    PSY_CUDA_TRY(cudaMemcpyAsync(jobs_.as<JobGpu>() + first, jobs, sizeof(JobGpu) * n, cudaMemcpyHostToDevice,
                                 context_->stream));
    return PSY_OK;
}

psy_status WavefrontEngine::ensure_plan_room(size_t waves) {
    if (waves <= plan_waves_) return PSY_OK;
    const size_t w = std::max<size_t>(waves, 2u * plan_waves_);
    PSY_CUDA_TRY(plan_rounds_.alloc(w * 16u));
    PSY_CUDA_TRY(plan_items_.alloc(w * max_jobs_ * sizeof(BatchItem)));
    plan_waves_ = w;
    ++plan_generation_;  // a captured graph names the old plan buffers
    return PSY_OK;
}

// The launches of one wavefront.  Every kernel sizes its grid from the
// capacity and reads the live counts from device memory; steps past the
// last live path find empty queues and return at once.
uint32_t WavefrontEngine::issue(uint32_t steps, bool allow_exit, psy_status &status) {
    cudaStream_t st = context_->stream;
    const LaunchConfig &lc = context_->launch;
    const JobGpu *jt = jobs_.as<JobGpu>();
    const BatchItem *it = items_.as<BatchItem>();
    const uint32_t *rd = round_.as<uint32_t>();
    const uint32_t cap = arena_.capacity;
    PathBuffers b = arena_.view;
    status = PSY_OK;
    launch_begin_round(st, b.counters, round_.as<uint32_t>(), items_.as<BatchItem>(), plan_rounds_.as<uint32_t>(),
                       plan_items_.as<BatchItem>(), cursor_.as<uint32_t>(), max_jobs_);
    launch_raygen_batch(st, lc, jt, it, rd, b, cap);
    uint32_t launches = 2u;
    for (uint32_t step = 0; step < steps; ++step) {
        launch_intersect_batch(st, lc, jt, b, cap);
        launch_shade_batch(st, lc, jt, b, cap, step);
        launch_count_rays(st, b.counters, arena_.stats.as<unsigned long long>());
        launch_shadow_batch(st, lc, jt, b, cap, step);
        launch_swap(st, b.counters);
        std::swap(b.queue_in, b.queue_out);
        launches += 5u;
        if (allow_exit && (step + 1u) % check_interval_ == 0u) {
            uint32_t left = 0u;
            if (cudaMemcpyAsync(&left, b.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                status = fail(PSY_ERROR_CUDA, "wavefront: reading the live path count failed");
                return launches;
            }
            if (left == 0u) break;
        }
    }
    launch_film_batch(st, lc, jt, it, rd, b, cap);
    return launches + 1u;
}

psy_status WavefrontEngine::ensure_graph(uint32_t steps) {
    if (graph_ && graph_steps_ == steps && graph_capacity_ == arena_.capacity && graph_generation_ == plan_generation_)
        return PSY_OK;
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    cudaStream_t st = context_->stream;
    PSY_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    psy_status s = PSY_OK;
    issue(steps, false, s);
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(st, &g);
    if (s != PSY_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (end != cudaSuccess) return fail(PSY_ERROR_CUDA, std::string("wavefront graph capture: ") + cudaGetErrorString(end));
    const cudaError_t inst = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (inst != cudaSuccess) {
        graph_ = nullptr;
        return fail(PSY_ERROR_CUDA, std::string("wavefront graph instantiate: ") + cudaGetErrorString(inst));
    }
    graph_steps_ = steps;
    graph_capacity_ = arena_.capacity;
    graph_generation_ = plan_generation_;
    return PSY_OK;
}

psy_status WavefrontEngine::reset_counters() {
    PSY_CUDA_TRY(cudaMemsetAsync(arena_.stats.ptr, 0, 64, context_->stream));
    began_ = false;
    return PSY_OK;
}

psy_status WavefrontEngine::run(const EnginePlan &plan, uint32_t steps, EngineRun &out) {
    const uint32_t waves = plan.waves();
    if (waves == 0u) return PSY_OK;
    cudaStream_t st = context_->stream;
    const psy_status room = ensure_plan_room(waves);
    if (room != PSY_OK) return room;
    PSY_CUDA_TRY(cudaMemcpyAsync(plan_rounds_.ptr, plan.rounds.data(), sizeof(uint32_t) * plan.rounds.size(),
                                 cudaMemcpyHostToDevice, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(plan_items_.ptr, plan.items.data(), sizeof(BatchItem) * plan.items.size(),
                                 cudaMemcpyHostToDevice, st));
    PSY_CUDA_TRY(cudaMemsetAsync(cursor_.ptr, 0, 16, st));
    if (use_graph_) {
        const psy_status g = ensure_graph(steps);
        if (g != PSY_OK) return g;
    }
    if (!began_) {
        PSY_CUDA_TRY(cudaEventRecord(ev_begin_, st));
        began_ = true;
    }
    for (uint32_t w = 0; w < waves; ++w) {
        if (use_graph_) {
            PSY_CUDA_TRY(cudaGraphLaunch(graph_, st));
            out.graph_launches += 1u;
            out.kernel_launches += 3u + 5u * steps;
        } else {
            psy_status s = PSY_OK;
            out.kernel_launches += issue(steps, true, s);
            if (s != PSY_OK) return s;
        }
        out.wavefronts += 1u;
    }
    PSY_CUDA_TRY(cudaEventRecord(ev_end_, st));
    return PSY_OK;
}

psy_status WavefrontEngine::elapsed(float *ms, uint64_t *closest_rays, uint64_t *shadow_rays) {
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaStreamSynchronize(context_->stream));
    uint32_t overflows = 0u;
    PSY_CUDA_TRY(take_stack_overflows(context_->stream, &overflows));
    if (overflows != 0u) return fail(PSY_ERROR_UNSUPPORTED, "traversal stack overflow on the device");
    *ms = 0.0f;
    if (began_) PSY_CUDA_TRY(cudaEventElapsedTime(ms, ev_begin_, ev_end_));
    unsigned long long rays[2] = {0ull, 0ull};
    PSY_CUDA_TRY(cudaMemcpy(rays, arena_.stats.ptr, sizeof(rays), cudaMemcpyDeviceToHost));
    *closest_rays = rays[0];
    *shadow_rays = rays[1];
    return PSY_OK;
}

}  // namespace psy::host
