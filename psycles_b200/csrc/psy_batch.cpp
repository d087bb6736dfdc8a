// Batched renders: sample ranges of many sessions in shared wavefronts
// (psy_batch_* of include/psycles_cuda.h) on the multi-job wavefront engine
// (psy_engine.h).  No counterpart in the reference, whose sessions dispatch
// one at a time (LuisaRenderSession::render_samples,
// src/luisa/path_tracer_session.cpp:272-397).
#include "psy_engine.h"

#include <algorithm>
#include <memory>
#include <vector>

using namespace psy::host;

namespace {

constexpr uint32_t kDefaultMaxJobs = 256u;

}  // namespace

struct psy_batch {
    psy_context *context = nullptr;
    psy_batch_config config{};
    WavefrontEngine engine;
    psy_batch_stats stats{};
};

extern "C" {

psy_status psy_batch_create(psy_context *context, const psy_batch_config *config, psy_batch **out) {
    if (!context || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto b = std::make_unique<psy_batch>();
    b->context = context;
    if (config) b->config = *config;
    if (b->config.path_capacity == 0u) b->config.path_capacity = context->path_capacity;
    if (b->config.max_jobs == 0u) b->config.max_jobs = kDefaultMaxJobs;
    if (b->config.check_interval == 0u) b->config.check_interval = 4u;
    if (b->config.max_jobs > 65536u) return fail(PSY_ERROR_INVALID_ARGUMENT, "batch: at most 65536 jobs");
    const psy_status r = b->engine.init(context, b->config.path_capacity, b->config.max_jobs,
                                        b->config.use_graph != 0u, b->config.check_interval);
    if (r != PSY_OK) return r;
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
        jobs[i] = PlanJob{i, pixels[i], 0u, samples[i]};
        cap = std::max(cap, pixels[i]);
    }
    std::vector<psy::BatchItem> items;
    uint32_t count = 0u, film = 0u;
    for (uint32_t wave = 0;; ++wave) {
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
        table[i] = session_job(s, p);
        const uint64_t begin = uint64_t(first[i]) + offset[i];
        plan[i] = PlanJob{i, s->pixels, begin, begin + count[i]};
        steps = std::max(steps, p.steps);
        max_pixels = std::max(max_pixels, s->pixels);
    }
    WavefrontEngine &engine = batch->engine;
    psy_status r = engine.reserve(std::max(batch->config.path_capacity, max_pixels));
    if (r != PSY_OK) return r;
    if ((r = engine.set_jobs(0u, table.data(), n)) != PSY_OK) return r;
    EnginePlan ep;
    std::vector<psy::BatchItem> wave;
    for (uint32_t w = 0;; ++w) {
        uint32_t film = 0u;
        const uint32_t paths = plan_wavefront(plan, w % n, engine.capacity(), wave, film);
        if (wave.empty()) break;
        bool glossy = false;
        for (const psy::BatchItem &it : wave) glossy = glossy || sessions[it.job]->scene->view.has_glossy != 0u;
        ep.add(wave, paths, film, engine.max_jobs(), glossy);
    }
    if ((r = engine.reset_counters()) != PSY_OK) return r;
    EngineRun run;
    if ((r = engine.run(ep, steps, run)) != PSY_OK) return r;
    psy_batch_stats stats{};
    if ((r = engine.elapsed(&stats.ms_total, &stats.closest_rays, &stats.shadow_rays)) != PSY_OK) return r;
    stats.samples = ep.samples;
    stats.jobs = n;
    stats.wavefronts = run.wavefronts;
    stats.graph_launches = run.graph_launches;
    stats.kernel_launches = run.kernel_launches;
    batch->stats = stats;
    bool any_cancelled = false;
    for (uint32_t i = 0; i < n; ++i) {
        sessions[i]->rendered += count[i];
        any_cancelled = any_cancelled || sessions[i]->cancelled.load();
    }
    return any_cancelled ? fail(PSY_ERROR_CANCELLED, "batch: a session was cancelled during the call") : PSY_OK;
}

}  // extern "C"
