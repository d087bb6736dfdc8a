// Static device scratch for psy_session_render_samples_static.
//
// Some callers cannot allocate device memory at render time: a plugin that
// runs inside an application's fixed device-memory budget, or a real-time
// viewport thread where an allocation's implicit synchronisation stalls the
// frame.  For them the wavefront path state lives in the file-scope arrays
// below instead of session-owned buffers.  Every GPU that loads
// libpsycles_cuda.so holds these ~17 MiB until the process exits.
//
// In host code `g_static_paths` / `g_static_sobol` name host-side stand-ins,
// not device addresses; the device addresses come from
// cudaGetSymbolAddress, taken once per device with that device current
// (static_scratch below) and cached.
#include <cuda_runtime.h>

#include <mutex>

#include "psy_static.h"

namespace psy {

static __device__ __align__(256) unsigned char g_static_paths[kStaticPathBytes];
static __device__ __align__(256) float4 g_static_sobol[kStaticSobolRows];

namespace {
struct StaticSlot {
    bool ready = false;
    void *paths = nullptr;
    float4 *sobol = nullptr;
};
std::mutex g_static_mutex;
StaticSlot g_static_slots[kStaticMaxDevices];
}  // namespace

cudaError_t static_scratch(int device, cudaStream_t stream, StaticSobolFill fill, void **paths, float4 **sobol) {
    if (device < 0 || device >= kStaticMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticSlot &slot = g_static_slots[device];
    if (!slot.ready) {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return e;
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_paths);
        if (e != cudaSuccess) return e;
        void *t = nullptr;
        e = cudaGetSymbolAddress(&t, g_static_sobol);
        if (e != cudaSuccess) return e;
        float4 *table = static_cast<float4 *>(t);
        // one 4 KiB pattern at a time from the stack (no heap); a copy from
        // pageable memory returns once its source is staged, so the buffer
        // can be refilled, and the copies are ordered on `stream`
        float pattern[kStaticSobolSize * 4u];
        for (uint32_t k = 0; k < 256u; ++k) {
            fill(pattern, kStaticSobolSize, k);
            e = cudaMemcpyAsync(table + size_t(k) * kStaticSobolSize, pattern, sizeof(pattern),
                                cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) return e;
        }
        // the table is complete on the device before any caller, on any
        // stream, sees the device as ready
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        slot.paths = p;
        slot.sobol = table;
        slot.ready = true;
    }
    *paths = slot.paths;
    *sobol = slot.sobol;
    return cudaSuccess;
}

}  // namespace psy
