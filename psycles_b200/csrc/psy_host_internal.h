// Host objects shared by the translation units of libpsycles_cuda.so: the
// opaque handles of the C ABI (context, compiled scene, session), device
// buffers, the wavefront path-state arena and error reporting.
#pragma once

#include "../../include/psycles_cuda.h"
#include "psy_kernels.h"
#include "psy_scene.h"

#include <cuda_runtime.h>

struct psy_session;

#include <algorithm>
#include <atomic>
#include <memory>
#include <mutex>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace psy::host {

// Records `message` as psy_last_error() of this thread and returns `status`.
psy_status fail(psy_status status, const std::string &message);

// Validates a SampleRange against a session (path_tracer_session.cpp:275-292),
// uploads the Sobol table sized from `total` and returns the render
// parameters of the range.
psy_status prepare_render(psy_session *s, uint32_t first, uint32_t count, uint32_t offset, uint32_t total,
                          RenderParams *out);

// Device bytes a compiled scene holds (geometry, BVH, materials, lights, tree).
uint64_t scene_device_bytes(const psy_scene *s);

// Builds the scene's many-light tree unless it is built already (it is built
// on first use, not by psy_scene_compile).
psy_status ensure_light_tree(psy_scene *s);

// Parameter-only material edit that leaves the device data of work already
// queued intact: the parameter block (and a rebuilt light tree) go to new
// device buffers and the scene's view points at them; the old buffers are
// kept until release_retired.  Work planned afterwards sees the edit.
psy_status rebind_parameters_versioned(psy_scene *s, uint32_t material, const float *scalars, uint32_t scalar_count,
                                       const float *vectors, uint32_t vector_count);
// Frees the buffers earlier edits retired; no queued work may read them.
void release_retired(psy_scene *s);

// The job record of a session for a multi-job wavefront.
JobGpu session_job(const psy_session *s, const RenderParams &p);

// psy_session_create (+ psy_session_set_camera when `camera` is set) for a
// render server: the session's buffers are stream-ordered and nothing waits
// for the context's stream, so admitting a job does not stall wavefronts in
// flight.
psy_status create_server_session(psy_scene *scene, const psy_render_settings &settings, const psy_camera_desc *camera,
                                 psy_session **out);

// Device memory.  A buffer bound to a stream (`ordered`) is allocated and
// freed in that stream's order (cudaMallocAsync / cudaFreeAsync), so
// freeing it neither waits for nor disturbs work queued on other buffers;
// otherwise cudaMalloc / cudaFree.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t ordered = nullptr;
    DeviceBuffer() = default;
    explicit DeviceBuffer(cudaStream_t st) : ordered(st) {}
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) {
            if (ordered) cudaFreeAsync(ptr, ordered);
            else cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        bytes = n;
        if (n == 0) return cudaSuccess;
        return ordered ? cudaMallocAsync(&ptr, n, ordered) : cudaMalloc(&ptr, n);
    }
    template <typename T>
    cudaError_t upload(const std::vector<T> &v, cudaStream_t st) {
        cudaError_t e = alloc(std::max<size_t>(v.size() * sizeof(T), 16));
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    }
    template <typename T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
    void swap(DeviceBuffer &o) noexcept {
        std::swap(ptr, o.ptr);
        std::swap(bytes, o.bytes);
        std::swap(ordered, o.ordered);
    }
};

// Wavefront path state over `capacity` paths: the 128-byte per-path
// records and the arrays of the other fields; the per-path job array only
// for batched wavefronts.
struct PathArena {
    uint32_t capacity = 0;
    DeviceBuffer records, rad_final, sample, aov_n, aov_a, mis_n, sh_o, sh_d, sh_c, sh_ids, sh_path, qa, qb, sq, job,
        sort_keys,
        queue_sorted, sort_hist, counters, stats;
    PathBuffers view{};
    psy_status ensure(uint32_t n, bool with_job);
    static size_t bytes_per_path(bool with_job);
};

// Points the record fields of `b` into the records starting at `records`.
void bind_records(PathBuffers &b, unsigned char *records);

}  // namespace psy::host

#define PSY_CUDA_TRY(expr)                                                                          \
    do {                                                                                            \
        const cudaError_t err_ = (expr);                                                            \
        if (err_ != cudaSuccess) {                                                                  \
            return psy::host::fail(PSY_ERROR_CUDA, std::string(#expr ": ") + cudaGetErrorString(err_)); \
        }                                                                                           \
    } while (0)

struct psy_context {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    psy::LaunchConfig launch;      // psy_context_set_tuning
    uint32_t path_capacity = 1u << 24;  // 16 Mi paths, about 3.9 GB of path state
    // Path state shared by every session of the context: their renders run
    // on the context's one stream and render_samples is synchronous, so
    // they never overlap; the mutex orders renders from different threads.
    psy::host::PathArena arena;
    std::mutex render_mutex;
    // pass readback: its own stream (films are complete when read, so it
    // need not wait for renders queued on `stream`), a device buffer for the
    // resolved pass and pinned host staging
    cudaStream_t readback = nullptr;
    psy::host::DeviceBuffer readback_pass, readback_flag;
    void *readback_host = nullptr;
    size_t readback_host_bytes = 0;
    std::mutex readback_mutex;
};

struct psy_scene {
    psy_context *context = nullptr;
    uint64_t revision = 0;
    psy_camera_desc camera{};
    std::vector<psy::MaterialGpu> materials;
    std::vector<float> scalars, vectors;
    psy::host::DeviceBuffer tlas, blas, tlas8, blas8, tlas_ids, tris, instances, meshes, positions, normals, indices, tri_materials, material_buf, code,
        value_buf, scalar_buf, vector_buf, emitters, distribution, ggx_tables, lights, lamp_consts, lamp_bounds, lamp_ids, lt_nodes, lt_emitters,
        lt_mapping, lt_lookup;
    psy::SceneView view{};
    uint64_t triangle_count = 0;
    psy_scene_build_stats stats{};
    // What the light tree is built from, kept on the host: it is built on
    // first use (a session with use_light_tree) and rebuilt when a
    // parameter edit changes an emissive material's estimate.
    std::vector<psy::EmitterGpu> emitters_host;
    std::vector<psy_light_desc> lights_host;
    std::vector<psy_closure_instruction> code_host;
    std::vector<psy_value_instruction> values_host;
    std::vector<uint8_t> instance_mirrored;  // object-to-world determinant < 0
    std::mutex light_tree_mutex;
    bool light_tree_built = false;
    // device buffers replaced by edits while work still read them
    std::vector<std::unique_ptr<psy::host::DeviceBuffer>> retired;
    std::vector<std::shared_ptr<const void>> retired_host;  // host sources of uploads not yet waited for
    cudaEvent_t uploads_done = nullptr;                      // recorded after the latest edit's uploads
};

struct psy_session {
    psy_scene *scene = nullptr;
    psy_render_settings settings{};
    psy::RenderParams params{};
    bool has_camera = false;      // psy_session_set_camera override
    psy_camera_desc camera{};
    uint32_t pixels = 0;
    uint32_t total = 0;
    uint32_t sobol_size = 0;
    uint32_t rendered = 0;
    std::atomic<bool> cancelled{false};
    psy::host::DeviceBuffer sobol, filter, combined, normal, albedo, sample_count;
    // path state: the context's shared arena (psy_context::arena)
    // trace
    psy::host::DeviceBuffer trace_buf;
    bool trace_requested = false;
    uint32_t trace_x = 0, trace_y = 0, trace_sample = 0;
    psy_path_trace trace_host{};
    psy_render_stats last_stats{};
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    bool profiling = false;
    psy_kernel_profile profile{};
    cudaEvent_t ev_k[2] = {nullptr, nullptr};
};

