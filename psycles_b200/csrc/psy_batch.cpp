// Batched wavefronts: sample ranges of many sessions rendered in shared
// path state.  No counterpart in the reference, whose sessions dispatch one
// at a time (LuisaRenderSession::render_samples,
// src/luisa/path_tracer_session.cpp:272-397).
//
// A wavefront is a list of items, one per session at most: a contiguous
// sample range of that session over its window pixels.  Paths are laid out
// item after item, sample-major inside an item, so the film kernel can add
// each pixel's samples in sample order; a session's samples advance in order
// across wavefronts, which makes its film independent of how its samples
// were grouped.  Every kernel of the wavefront reads its path's job record
// (render parameters, scene view, film).  With graphs on, the launch
// sequence of a wavefront (counters, camera rays, every path step, film) is
// captured once and replayed; the wavefront's shape lives in device memory.
#include "psy_host_internal.h"
#include "psy_kernels.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

using namespace psy::host;

namespace {

constexpr uint32_t kDefaultBatchCapacity = 1u << 22;
constexpr uint32_t kDefaultMaxJobs = 256u;

struct PlanJob {
    uint32_t pixels;
    uint64_t next, end;  // sample cursor
};

// One wavefront: visits the jobs from `start` round-robin and gives each
// unfinished job as many samples as fit.  Returns the paths used.
uint32_t plan_wavefront(std::vector<PlanJob> &jobs, uint32_t start, uint32_t capacity,
                        std::vector<psy::BatchItem> &items, uint32_t &film_pixels) {
    items.clear();
    film_pixels = 0u;
    uint32_t used = 0u;
    const uint32_t n = uint32_t(jobs.size());
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t j = (start + k) % n;
        PlanJob &pj = jobs[j];
        if (pj.next >= pj.end || pj.pixels == 0u) continue;
        const uint32_t fit = (capacity - used) / pj.pixels;
        if (fit == 0u) continue;
        const uint32_t take = uint32_t(std::min<uint64_t>(fit, pj.end - pj.next));
        psy::BatchItem it{};
        it.job = j;
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
    // the path and film layouts are ordered by item; the kernels' binary
    // searches need items sorted by path_begin, which they are
    return used;
}

}  // namespace

struct psy_batch {
    psy_context *context = nullptr;
    psy_batch_config config{};
    PathArena arena;
    DeviceBuffer jobs, items, round, cursor, plan_rounds, plan_items;
    size_t plan_round_bytes = 0, plan_item_bytes = 0;
    psy_batch_stats stats{};
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_steps = 0u, graph_capacity = 0u;
    const void *graph_rounds = nullptr, *graph_items = nullptr;

    // Device room for a call's plan (grown, never shrunk, so a captured
    // graph stays valid across calls of the same shape).
    psy_status ensure_plan(size_t rounds, size_t items_bytes) {
        if (rounds * 16u > plan_round_bytes) {
            PSY_CUDA_TRY(plan_rounds.alloc(rounds * 16u * 2u));
            plan_round_bytes = rounds * 16u * 2u;
        }
        if (items_bytes > plan_item_bytes) {
            PSY_CUDA_TRY(plan_items.alloc(items_bytes * 2u));
            plan_item_bytes = items_bytes * 2u;
        }
        return PSY_OK;
    }

    ~psy_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev_begin) cudaEventDestroy(ev_begin);
        if (ev_end) cudaEventDestroy(ev_end);
    }

    // The launches of one wavefront of at most `capacity` paths and `steps`
    // path steps (every kernel sizes its grid from the capacity and reads
    // the live counts from device memory).  Steps past the last live path
    // find empty queues and return at once.
    uint32_t issue(cudaStream_t st, uint32_t steps, uint32_t check_interval, bool allow_exit, psy_status &status) {
        const int sms = context->sms;
        const psy::JobGpu *jt = jobs.as<psy::JobGpu>();
        const psy::BatchItem *it = items.as<psy::BatchItem>();
        const uint32_t *rd = round.as<uint32_t>();
        const uint32_t cap = arena.capacity;
        psy::PathBuffers b = arena.view;
        uint32_t launches = 0u;
        status = PSY_OK;
        psy::launch_begin_round(st, b.counters, round.as<uint32_t>(), items.as<psy::BatchItem>(),
                                plan_rounds.as<uint32_t>(), plan_items.as<psy::BatchItem>(), cursor.as<uint32_t>(),
                                config.max_jobs);
        psy::launch_raygen_batch(st, sms, jt, it, rd, b, cap);
        launches += 2u;
        for (uint32_t step = 0; step < steps; ++step) {
            psy::launch_intersect_batch(st, sms, jt, b, cap);
            psy::launch_shade_batch(st, sms, jt, b, cap, step);
            psy::launch_count_rays(st, b.counters, arena.stats.as<unsigned long long>());
            psy::launch_shadow_batch(st, sms, jt, b, cap, step);
            psy::launch_swap(st, b.counters);
            std::swap(b.queue_in, b.queue_out);
            launches += 5u;
            if (allow_exit && check_interval && (step + 1u) % check_interval == 0u) {
                uint32_t left = 0u;
                if (cudaMemcpyAsync(&left, b.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess) {
                    status = fail(PSY_ERROR_CUDA, "batch: reading the live path count failed");
                    return launches;
                }
                if (left == 0u) break;
            }
        }
        psy::launch_film_batch(st, sms, jt, it, rd, b, cap);
        return launches + 1u;
    }

    psy_status ensure_graph(cudaStream_t st, uint32_t steps, uint32_t &launches) {
        if (graph && graph_steps == steps && graph_capacity == arena.capacity && graph_rounds == plan_rounds.ptr &&
            graph_items == plan_items.ptr) {
            launches = 3u + 5u * steps;
            return PSY_OK;
        }
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        PSY_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        psy_status s = PSY_OK;
        launches = issue(st, steps, 0u, false, s);
        cudaGraph_t g = nullptr;
        const cudaError_t end = cudaStreamEndCapture(st, &g);
        if (s != PSY_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (end != cudaSuccess) return fail(PSY_ERROR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(end));
        const cudaError_t inst = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (inst != cudaSuccess) {
            graph = nullptr;
            return fail(PSY_ERROR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(inst));
        }
        graph_steps = steps;
        graph_capacity = arena.capacity;
        graph_rounds = plan_rounds.ptr;
        graph_items = plan_items.ptr;
        return PSY_OK;
    }
};

extern "C" {

psy_status psy_batch_create(psy_context *context, const psy_batch_config *config, psy_batch **out) {
    if (!context || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto b = std::make_unique<psy_batch>();
    b->context = context;
    if (config) b->config = *config;
    if (b->config.path_capacity == 0u) b->config.path_capacity = kDefaultBatchCapacity;
    if (b->config.max_jobs == 0u) b->config.max_jobs = kDefaultMaxJobs;
    if (b->config.check_interval == 0u) b->config.check_interval = 4u;
    if (b->config.max_jobs > 65536u) return fail(PSY_ERROR_INVALID_ARGUMENT, "batch: at most 65536 jobs");
    PSY_CUDA_TRY(cudaSetDevice(context->device));
    PSY_CUDA_TRY(b->jobs.alloc(sizeof(psy::JobGpu) * b->config.max_jobs));
    PSY_CUDA_TRY(b->items.alloc(sizeof(psy::BatchItem) * b->config.max_jobs));
    PSY_CUDA_TRY(b->round.alloc(16));
    PSY_CUDA_TRY(b->cursor.alloc(16));
    PSY_CUDA_TRY(cudaEventCreate(&b->ev_begin));
    PSY_CUDA_TRY(cudaEventCreate(&b->ev_end));
    *out = b.release();
    return PSY_OK;
}

void psy_batch_destroy(psy_batch *batch) {
    if (!batch) return;
    cudaSetDevice(batch->context->device);
    delete batch;
}

psy_status psy_batch_get_stats(const psy_batch *batch, psy_batch_stats *out) {
    if (!batch || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = batch->stats;
    return PSY_OK;
}

psy_status psy_batch_plan(const uint32_t *pixels, const uint32_t *samples, uint32_t n, uint32_t capacity,
                          uint32_t *out_items, uint32_t max_items, uint32_t *out_count) {
    if (!pixels || !samples || !out_count || (max_items && !out_items))
        return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    std::vector<PlanJob> jobs(n);
    uint32_t cap = capacity;
    for (uint32_t i = 0; i < n; ++i) {
        jobs[i] = PlanJob{pixels[i], 0u, samples[i]};
        cap = std::max(cap, pixels[i]);
    }
    std::vector<psy::BatchItem> items;
    uint32_t count = 0u, wave = 0u, film = 0u;
    for (;;) {
        plan_wavefront(jobs, wave % std::max(n, 1u), cap, items, film);
        if (items.empty()) break;
        for (const psy::BatchItem &it : items) {
            if (count < max_items) {
                uint32_t *w = out_items + 6u * count;
                w[0] = it.job;
                w[1] = wave;
                w[2] = it.path_begin;
                w[3] = it.sample_base;
                w[4] = it.samples;
                w[5] = it.film_begin;
            }
            ++count;
        }
        ++wave;
    }
    *out_count = count;
    return count > max_items ? fail(PSY_ERROR_RANGE, "batch plan: more items than max_items") : PSY_OK;
}

psy_status psy_batch_render(psy_batch *batch, psy_session *const *sessions, const uint32_t *first,
                            const uint32_t *count, const uint32_t *offset, const uint32_t *total, uint32_t n) {
    if (!batch || !sessions || !first || !count || !offset || !total)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    if (n == 0u) return fail(PSY_ERROR_RANGE, "batch: no sessions");
    if (n > batch->config.max_jobs) return fail(PSY_ERROR_RANGE, "batch: more sessions than max_jobs");
    psy_context *ctx = batch->context;
    PSY_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    std::vector<psy::JobGpu> table(n);
    std::vector<PlanJob> plan(n);
    uint32_t steps = 0u, max_pixels = 0u;
    for (uint32_t i = 0; i < n; ++i) {
        psy_session *s = sessions[i];
        if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "batch: null session");
        if (s->scene->context != ctx) return fail(PSY_ERROR_INVALID_ARGUMENT, "batch: session of another context");
        for (uint32_t k = 0; k < i; ++k)
            if (sessions[k] == s) return fail(PSY_ERROR_INVALID_ARGUMENT, "batch: a session is listed twice");
        psy::RenderParams p;
        const psy_status r = prepare_render(s, first[i], count[i], offset[i], total[i], &p);
        if (r != PSY_OK) return r;
        psy::JobGpu &j = table[i];
        j.p = p;
        j.s = s->scene->view;
        j.combined = s->combined.as<float4>();
        j.normal = s->normal.as<float4>();
        j.albedo = s->albedo.as<float4>();
        j.sample_count = s->sample_count.as<uint32_t>();
        const uint64_t begin = uint64_t(first[i]) + offset[i];
        plan[i] = PlanJob{s->pixels, begin, begin + count[i]};
        steps = std::max(steps, p.steps);
        max_pixels = std::max(max_pixels, s->pixels);
    }
    const psy_status grown = batch->arena.ensure(std::max(batch->config.path_capacity, max_pixels), true);
    if (grown != PSY_OK) return grown;
    const uint32_t cap = batch->arena.capacity;
    PSY_CUDA_TRY(cudaMemcpyAsync(batch->jobs.ptr, table.data(), sizeof(psy::JobGpu) * n, cudaMemcpyHostToDevice, st));
    PSY_CUDA_TRY(cudaMemsetAsync(batch->arena.stats.ptr, 0, 64, st));
    psy_batch_stats stats{};
    stats.jobs = n;
    // the whole call's plan: wavefront headers and items, uploaded once
    std::vector<uint32_t> rounds;
    std::vector<psy::BatchItem> all_items;
    {
        std::vector<psy::BatchItem> items;
        for (uint32_t wave = 0;; ++wave) {
            uint32_t film_pixels = 0u;
            const uint32_t paths = plan_wavefront(plan, wave % n, cap, items, film_pixels);
            if (items.empty()) break;
            rounds.insert(rounds.end(), {paths, film_pixels, uint32_t(items.size()), 0u});
            items.resize(batch->config.max_jobs, psy::BatchItem{});
            all_items.insert(all_items.end(), items.begin(), items.end());
            for (uint32_t k = 0; k < rounds[rounds.size() - 2u]; ++k)
                stats.samples += uint64_t(items[k].samples) * items[k].pixels;
        }
    }
    const uint32_t waves = uint32_t(rounds.size() / 4u);
    const psy_status room = batch->ensure_plan(waves, sizeof(psy::BatchItem) * all_items.size());
    if (room != PSY_OK) return room;
    PSY_CUDA_TRY(cudaMemcpyAsync(batch->plan_rounds.ptr, rounds.data(), sizeof(uint32_t) * rounds.size(),
                                 cudaMemcpyHostToDevice, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(batch->plan_items.ptr, all_items.data(), sizeof(psy::BatchItem) * all_items.size(),
                                 cudaMemcpyHostToDevice, st));
    PSY_CUDA_TRY(cudaMemsetAsync(batch->cursor.ptr, 0, 16, st));
    uint32_t graph_launches_per_wave = 0u;
    if (batch->config.use_graph) {
        const psy_status g = batch->ensure_graph(st, steps, graph_launches_per_wave);
        if (g != PSY_OK) return g;
    }
    PSY_CUDA_TRY(cudaEventRecord(batch->ev_begin, st));
    for (uint32_t wave = 0; wave < waves; ++wave) {
        if (batch->config.use_graph) {
            PSY_CUDA_TRY(cudaGraphLaunch(batch->graph, st));
            stats.graph_launches += 1u;
            stats.kernel_launches += graph_launches_per_wave;
        } else {
            psy_status s = PSY_OK;
            stats.kernel_launches += batch->issue(st, steps, batch->config.check_interval, true, s);
            if (s != PSY_OK) return s;
        }
        ++stats.wavefronts;
    }
    PSY_CUDA_TRY(cudaEventRecord(batch->ev_end, st));
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    PSY_CUDA_TRY(cudaEventElapsedTime(&stats.ms_total, batch->ev_begin, batch->ev_end));
    unsigned long long rays[2] = {0ull, 0ull};
    PSY_CUDA_TRY(cudaMemcpy(rays, batch->arena.stats.ptr, sizeof(rays), cudaMemcpyDeviceToHost));
    stats.closest_rays = rays[0];
    stats.shadow_rays = rays[1];
    batch->stats = stats;
    bool any_cancelled = false;
    for (uint32_t i = 0; i < n; ++i) {
        sessions[i]->rendered += count[i];
        any_cancelled = any_cancelled || sessions[i]->cancelled.load();
    }
    return any_cancelled ? fail(PSY_ERROR_CANCELLED, "batch: a session was cancelled during the call") : PSY_OK;
}

}  // extern "C"
