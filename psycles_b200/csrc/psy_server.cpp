// Render server: a persistent request loop over resident scenes
// (psy_server_* of include/psycles_cuda.h).  No counterpart in the
// reference, which renders one session per caller.
//
// Requests (render jobs and parameter-only material edits) enter one FIFO.
// A loop thread admits jobs from its head while the HBM budget and the job
// slots allow: a job gets a session (film, Sobol and filter tables) and a
// slot of the wavefront engine's job table.  Every wavefront takes samples
// from the running jobs in admission order -- the oldest job takes all the
// samples that fit and younger jobs backfill the rest (continuous batching:
// a job admitted while others are on the GPU joins the next wavefront), so
// small jobs share the device with large ones without delaying them.  Two
// wavefronts are in flight: the host plans and admits for the next while
// the GPU runs the current one.  A job is done once the wavefront holding
// its last samples has finished.  Because every pixel adds its samples in
// order, a job's passes are the same alone and in any mix.  An edit takes
// effect when it reaches the head of the FIFO, without waiting for running
// jobs: it writes a new copy of the scene's parameter block (and of a light
// tree it changes), running jobs keep reading the copy they were admitted
// with, and the old copy is freed once no running job uses the scene -- so
// each job sees exactly the edits submitted before it.
#include "psy_engine.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

using namespace psy::host;

namespace {

constexpr uint64_t kDefaultBudget = 120ull << 30;
constexpr uint32_t kDefaultRunning = 256u;

struct Job {
    uint64_t id = 0;
    psy_scene *scene = nullptr;
    psy_render_settings settings{};
    bool has_camera = false;
    psy_camera_desc camera{};
    uint32_t samples = 0;
    uint32_t state = PSY_JOB_QUEUED;
    psy_status status = PSY_OK;
    psy_session *session = nullptr;
    uint32_t slot = 0, pixels = 0, steps = 0;
    uint64_t next = 0;        // next sample to plan
    uint64_t last_wave = 0;   // wavefront holding the last planned samples
    uint64_t bytes = 0;
    std::atomic<bool> cancel{false};
    double submit_ms = 0.0, admit_ms = 0.0, done_ms = 0.0;
};

struct Edit {
    psy_scene *scene = nullptr;
    uint32_t material = 0;
    std::vector<float> scalars, vectors;
};

struct Request {
    uint64_t job = 0;              // nonzero: a job id
    std::shared_ptr<Edit> edit;    // else an edit
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * double(v.size() - 1u);
    const size_t lo = size_t(pos);
    const size_t hi = std::min(lo + 1u, v.size() - 1u);
    return v[lo] + (v[hi] - v[lo]) * (pos - double(lo));
}

}  // namespace

struct psy_server {
    psy_context *context = nullptr;
    psy_server_config config{};
    WavefrontEngine engine;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;
    std::condition_variable wake, done_cv;
    std::deque<Request> fifo;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    std::map<const psy_scene *, uint64_t> scene_bytes;
    std::set<psy_scene *> retired_scenes;  // scenes holding buffers that running jobs read
    std::vector<uint32_t> free_slots;
    uint64_t next_id = 1;
    uint64_t bytes_in_use = 0, bytes_peak = 0, fixed_bytes = 0;
    uint64_t samples_done = 0, wavefronts = 0, jobs_failed = 0, jobs_done = 0, jobs_submitted = 0;
    double busy_ms = 0.0, device_ms = 0.0;
    std::vector<double> latencies;  // submit -> done of every finished job
    psy_status loop_status = PSY_OK;
    std::string loop_error;
    bool stop = false;
    std::thread loop;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    // Under `mu`: admits jobs and applies edits from the head of the FIFO.
    void admit(std::vector<Job *> &running) {
        while (!fifo.empty()) {
            Request &head = fifo.front();
            if (head.edit) {
                // running jobs keep the parameter block they were admitted
                // with; jobs admitted from here on see the edit
                psy_scene *sc = head.edit->scene;
                const Edit &e = *head.edit;
                const psy_status r = rebind_parameters_versioned(sc, e.material, e.scalars.data(),
                                                                 uint32_t(e.scalars.size()), e.vectors.data(),
                                                                 uint32_t(e.vectors.size() / 3u));
                if (r != PSY_OK) loop_error = std::string("edit rejected: ") + psy_last_error();
                if (std::none_of(running.begin(), running.end(), [sc](const Job *j) { return j->scene == sc; }))
                    release_retired(sc);
                else
                    retired_scenes.insert(sc);
                fifo.pop_front();
                continue;
            }
            auto it = jobs.find(head.job);
            if (it == jobs.end() || it->second->cancel) {
                if (it != jobs.end()) {
                    it->second->state = PSY_JOB_CANCELLED;
                    it->second->done_ms = now_ms();
                    done_cv.notify_all();
                }
                fifo.pop_front();
                continue;
            }
            Job &j = *it->second;
            // a job that selects lights from the tree builds it first, so
            // its bytes are counted with the scene's
            if (j.settings.use_light_tree) {
                const psy_status built = ensure_light_tree(j.scene);
                if (built != PSY_OK) {
                    j.state = PSY_JOB_FAILED;
                    j.status = built;
                    j.done_ms = now_ms();
                    ++jobs_failed;
                    fifo.pop_front();
                    done_cv.notify_all();
                    continue;
                }
            }
            const uint64_t scene_now = psy_scene_device_bytes(j.scene);
            const auto counted = scene_bytes.find(j.scene);
            const uint64_t scene_extra =
                counted == scene_bytes.end() ? scene_now : scene_now - std::min(scene_now, counted->second);
            const uint64_t need = j.bytes + scene_extra;
            uint64_t resident = fixed_bytes;
            for (const auto &kv : scene_bytes) resident += kv.second;
            if (resident + need > config.hbm_budget_bytes) {  // never fits, even alone
                j.state = PSY_JOB_FAILED;
                j.status = PSY_ERROR_OUT_OF_MEMORY;
                j.done_ms = now_ms();
                ++jobs_failed;
                fifo.pop_front();
                done_cv.notify_all();
                continue;
            }
            if (bytes_in_use + need > config.hbm_budget_bytes || free_slots.empty()) return;
            // admission: the job's session holds its film and tables
            psy_session *s = nullptr;
            psy_status r = create_server_session(j.scene, j.settings, j.has_camera ? &j.camera : nullptr, &s);
            psy::RenderParams p{};
            if (r == PSY_OK) r = prepare_render(s, 0u, j.samples, 0u, j.samples, &p);
            const uint32_t slot = free_slots.back();
            psy::JobGpu rec{};
            if (r == PSY_OK) {
                rec = session_job(s, p);
                r = engine.set_jobs(slot, &rec, 1u);
            }
            if (r != PSY_OK) {
                if (s) psy_session_destroy(s);
                j.state = PSY_JOB_FAILED;
                j.status = r;
                j.done_ms = now_ms();
                ++jobs_failed;
                fifo.pop_front();
                done_cv.notify_all();
                continue;
            }
            free_slots.pop_back();
            if (scene_extra) scene_bytes[j.scene] = scene_now;
            bytes_in_use += need;
            bytes_peak = std::max(bytes_peak, bytes_in_use);
            j.session = s;
            j.slot = slot;
            j.pixels = s->pixels;
            j.steps = p.steps;
            j.next = 0u;
            j.state = PSY_JOB_RUNNING;
            j.admit_ms = now_ms();
            running.push_back(&j);
            fifo.pop_front();
        }
    }

    void run_loop() {
        std::vector<Job *> running;
        struct InFlight {
            cudaEvent_t begin = nullptr, done = nullptr;
            uint64_t wave = 0;
            double issued_ms = 0.0;
            bool active = false;
        } flight[2];
        cudaSetDevice(context->device);
        for (auto &f : flight) {
            cudaEventCreate(&f.begin);
            cudaEventCreate(&f.done);
        }
        uint64_t wave_counter = 0, finished_wave = 0;
        // a finished wavefront's device span: from the stream reaching its
        // first launch to its last kernel's end (`locked`: the caller holds mu)
        auto retire = [&](InFlight &f, bool locked) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, f.begin, f.done) == cudaSuccess) {
                if (locked) {
                    device_ms += ms;
                } else {
                    std::lock_guard<std::mutex> lock(mu);
                    device_ms += ms;
                }
            }
            f.active = false;
            finished_wave = std::max(finished_wave, f.wave + 1u);
        };
        double busy_since = -1.0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(mu);
                if (stop) break;
                admit(running);
                const bool idle = running.empty() && !flight[0].active && !flight[1].active;
                if (idle) {
                    if (busy_since >= 0.0) {
                        busy_ms += now_ms() - busy_since;
                        busy_since = -1.0;
                    }
                    wake.wait_for(lock, std::chrono::milliseconds(20));
                    continue;
                }
                if (busy_since < 0.0) busy_since = now_ms();
            }
            // plan one wavefront over the running jobs with samples left
            std::vector<PlanJob> plan;
            std::vector<Job *> planned;
            uint32_t steps = 0u;
            for (Job *j : running) {
                if (j->next >= j->samples || j->cancel) continue;
                plan.push_back(PlanJob{j->slot, j->pixels, j->next, j->samples});
                planned.push_back(j);
                steps = std::max(steps, j->steps);
            }
            InFlight &slot = flight[wave_counter & 1u];
            if (slot.active) {
                // both buffers busy: wait for the older wavefront first
                cudaEventSynchronize(slot.done);
                retire(slot, false);
            }
            if (!plan.empty()) {
                std::vector<psy::BatchItem> items;
                uint32_t film = 0u;
                // oldest job first, the others backfill the capacity it leaves
                const uint32_t paths = plan_wavefront(plan, 0u, engine.capacity(), items, film);
                EnginePlan ep;
                bool glossy = false;
                for (const Job *j : planned) glossy = glossy || j->scene->view.has_glossy != 0u;
                ep.add(items, paths, film, engine.max_jobs(), glossy);
                EngineRun run;
                psy_status r = cudaEventRecord(slot.begin, engine.stream()) == cudaSuccess ? PSY_OK : PSY_ERROR_CUDA;
                if (r == PSY_OK) r = engine.run(ep, steps, run);
                if (r == PSY_OK && cudaEventRecord(slot.done, engine.stream()) != cudaSuccess) r = PSY_ERROR_CUDA;
                if (r != PSY_OK) {
                    std::lock_guard<std::mutex> lock(mu);
                    loop_status = r;
                    loop_error = psy_last_error();
                    for (Job *j : running) {
                        j->state = PSY_JOB_FAILED;
                        j->status = r;
                        j->done_ms = now_ms();
                    }
                    running.clear();
                    done_cv.notify_all();
                    break;
                }
                for (size_t k = 0; k < plan.size(); ++k) {
                    planned[k]->next = plan[k].next;
                    planned[k]->last_wave = wave_counter;
                }
                slot.wave = wave_counter;
                slot.issued_ms = now_ms();
                slot.active = true;
                ++wave_counter;
                std::lock_guard<std::mutex> lock(mu);
                ++wavefronts;
                samples_done += ep.samples;
            } else {
                // nothing new to issue: drain the wavefronts in flight
                for (auto &f : flight) {
                    if (!f.active) continue;
                    cudaEventSynchronize(f.done);
                    retire(f, false);
                }
            }
            // retire jobs whose last wavefront has finished
            {
                std::lock_guard<std::mutex> lock(mu);
                for (auto &f : flight) {
                    if (f.active && cudaEventQuery(f.done) == cudaSuccess) retire(f, true);
                }
                bool any = false;
                for (auto it = running.begin(); it != running.end();) {
                    Job *j = *it;
                    const bool finished = (j->next >= j->samples || j->cancel) && j->last_wave < finished_wave;
                    if (!finished) {
                        ++it;
                        continue;
                    }
                    j->state = j->cancel ? PSY_JOB_CANCELLED : PSY_JOB_DONE;
                    j->done_ms = now_ms();
                    if (!j->cancel) {
                        j->session->rendered += j->samples;
                        ++jobs_done;
                        latencies.push_back(j->done_ms - j->submit_ms);
                    }
                    free_slots.push_back(j->slot);
                    it = running.erase(it);
                    any = true;
                }
                if (any) {
                    // buffers replaced by edits are freed once no running
                    // job reads their scene
                    for (auto it = retired_scenes.begin(); it != retired_scenes.end();) {
                        psy_scene *sc = *it;
                        if (std::any_of(running.begin(), running.end(), [sc](const Job *j) { return j->scene == sc; })) {
                            ++it;
                            continue;
                        }
                        release_retired(sc);
                        it = retired_scenes.erase(it);
                    }
                    done_cv.notify_all();
                }
            }
        }
        for (auto &f : flight) {
            if (f.active) cudaEventSynchronize(f.done);
            cudaEventDestroy(f.begin);
            cudaEventDestroy(f.done);
        }
        if (busy_since >= 0.0) busy_ms += now_ms() - busy_since;
    }
};

extern "C" {

uint64_t psy_scene_device_bytes(const psy_scene *s) { return s ? scene_device_bytes(s) : 0u; }

psy_status psy_server_create(psy_context *context, const psy_server_config *config, psy_server **out) {
    if (!context || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto sv = std::make_unique<psy_server>();
    sv->context = context;
    if (config) sv->config = *config;
    if (sv->config.hbm_budget_bytes == 0u) sv->config.hbm_budget_bytes = kDefaultBudget;
    if (sv->config.path_capacity == 0u) sv->config.path_capacity = context->path_capacity;
    if (sv->config.max_running == 0u) sv->config.max_running = kDefaultRunning;
    if (sv->config.max_running > 65536u) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: at most 65536 running jobs");
    const psy_status r = sv->engine.init(context, sv->config.path_capacity, sv->config.max_running,
                                         sv->config.use_graph != 0u, 4u);
    if (r != PSY_OK) return r;
    sv->fixed_bytes = uint64_t(sv->engine.capacity()) * PathArena::bytes_per_path(true);
    if (sv->fixed_bytes > sv->config.hbm_budget_bytes)
        return fail(PSY_ERROR_OUT_OF_MEMORY, "server: the path state alone exceeds the HBM budget");
    sv->bytes_in_use = sv->fixed_bytes;
    sv->bytes_peak = sv->fixed_bytes;
    for (uint32_t i = sv->config.max_running; i-- > 0u;) sv->free_slots.push_back(i);
    sv->t0 = std::chrono::steady_clock::now();
    psy_server *raw = sv.get();
    raw->loop = std::thread([raw] { raw->run_loop(); });
    *out = sv.release();
    return PSY_OK;
}

void psy_server_destroy(psy_server *sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->stop = true;
    }
    sv->wake.notify_all();
    if (sv->loop.joinable()) sv->loop.join();
    cudaSetDevice(sv->context->device);
    for (auto &kv : sv->jobs)
        if (kv.second->session) psy_session_destroy(kv.second->session);
    delete sv;
}

psy_status psy_server_submit(psy_server *sv, psy_scene *scene, const psy_render_settings *settings,
                             const psy_camera_desc *camera, uint32_t samples, uint64_t *job_id) {
    if (!sv || !scene || !settings || !job_id) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    if (samples == 0u) return fail(PSY_ERROR_RANGE, "server: a job needs at least one sample");
    if (scene->context != sv->context) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: scene of another context");
    auto j = std::make_unique<Job>();
    j->scene = scene;
    j->settings = *settings;
    j->has_camera = camera != nullptr;
    if (camera) j->camera = *camera;
    j->samples = samples;
    const uint32_t w = settings->window_width ? settings->window_width : settings->full_width;
    const uint32_t h = settings->window_height ? settings->window_height : settings->full_height;
    j->bytes = job_device_bytes(w * h, samples);
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->loop_status != PSY_OK) return fail(PSY_ERROR_STATE, "server: the request loop stopped: " + sv->loop_error);
    j->id = sv->next_id++;
    j->submit_ms = sv->now_ms();
    *job_id = j->id;
    sv->fifo.push_back(Request{j->id, nullptr});
    sv->jobs.emplace(j->id, std::move(j));
    ++sv->jobs_submitted;
    sv->wake.notify_all();
    return PSY_OK;
}

psy_status psy_server_rebind_parameters(psy_server *sv, psy_scene *scene, uint32_t material, const float *scalars,
                                        uint32_t scalar_count, const float *vectors, uint32_t vector_count) {
    if (!sv || !scene) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    if ((scalar_count && !scalars) || (vector_count && !vectors)) return fail(PSY_ERROR_INVALID_ARGUMENT, "null parameters");
    if (material >= scene->materials.size()) return fail(PSY_ERROR_INVALID_ARGUMENT, "material out of range");
    auto e = std::make_shared<Edit>();
    e->scene = scene;
    e->material = material;
    e->scalars.assign(scalars, scalars + scalar_count);
    e->vectors.assign(vectors, vectors + 3ull * vector_count);
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->fifo.push_back(Request{0u, e});
    sv->wake.notify_all();
    return PSY_OK;
}

psy_status psy_server_poll(psy_server *sv, uint64_t job_id, psy_job_info *out) {
    if (!sv || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: unknown job");
    const Job &j = *it->second;
    out->state = j.state;
    out->status = j.status;
    out->samples_done = j.state == PSY_JOB_DONE ? j.samples : 0u;
    out->samples_total = j.samples;
    out->submit_ms = j.submit_ms;
    out->admit_ms = j.admit_ms;
    out->done_ms = j.done_ms;
    return PSY_OK;
}

psy_status psy_server_wait(psy_server *sv, uint64_t job_id, uint32_t timeout_ms) {
    if (!sv) return fail(PSY_ERROR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lock(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: unknown job");
    Job *j = it->second.get();
    const bool ended = sv->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), [j] {
        return j->state == PSY_JOB_DONE || j->state == PSY_JOB_FAILED || j->state == PSY_JOB_CANCELLED;
    });
    if (!ended) return fail(PSY_ERROR_TIMEOUT, "server: job not finished within the timeout");
    if (j->state == PSY_JOB_FAILED) return fail(j->status, "server: job failed");
    if (j->state == PSY_JOB_CANCELLED) return fail(PSY_ERROR_CANCELLED, "server: job cancelled");
    return PSY_OK;
}

psy_status psy_server_read_pass(psy_server *sv, uint64_t job_id, uint32_t pass_kind, float *out, uint64_t capacity,
                                uint32_t *channels) {
    if (!sv) return fail(PSY_ERROR_INVALID_ARGUMENT, "null server");
    psy_session *s = nullptr;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        auto it = sv->jobs.find(job_id);
        if (it == sv->jobs.end()) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: unknown job");
        if (it->second->state != PSY_JOB_DONE) return fail(PSY_ERROR_STATE, "server: job not done");
        s = it->second->session;
    }
    return psy_session_read_pass(s, pass_kind, out, capacity, channels);
}

psy_status psy_server_release(psy_server *sv, uint64_t job_id) {
    if (!sv) return fail(PSY_ERROR_INVALID_ARGUMENT, "null server");
    std::unique_ptr<Job> j;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        auto it = sv->jobs.find(job_id);
        if (it == sv->jobs.end()) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: unknown job");
        const uint32_t st = it->second->state;
        if (st == PSY_JOB_QUEUED || st == PSY_JOB_RUNNING) return fail(PSY_ERROR_STATE, "server: job still in flight");
        j = std::move(it->second);
        sv->jobs.erase(it);
        if (j->session) sv->bytes_in_use -= j->bytes;
    }
    if (j->session) psy_session_destroy(j->session);
    sv->wake.notify_all();
    return PSY_OK;
}

psy_status psy_server_cancel(psy_server *sv, uint64_t job_id) {
    if (!sv) return fail(PSY_ERROR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return fail(PSY_ERROR_INVALID_ARGUMENT, "server: unknown job");
    it->second->cancel = true;
    sv->wake.notify_all();
    return PSY_OK;
}

psy_status psy_server_get_stats(psy_server *sv, psy_server_stats *out) {
    if (!sv || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    const std::vector<double> &lat = sv->latencies;
    *out = psy_server_stats{};
    out->jobs_submitted = sv->jobs_submitted;
    out->jobs_done = sv->jobs_done;
    out->jobs_failed = sv->jobs_failed;
    out->samples = sv->samples_done;
    out->wavefronts = sv->wavefronts;
    out->bytes_in_use = sv->bytes_in_use;
    out->bytes_peak = sv->bytes_peak;
    out->busy_ms = sv->busy_ms;
    out->device_ms = sv->device_ms;
    out->latency_p50_ms = percentile(lat, 0.5);
    out->latency_p99_ms = percentile(lat, 0.99);
    out->latency_jobs = uint32_t(lat.size());
    return PSY_OK;
}

}  // extern "C"
