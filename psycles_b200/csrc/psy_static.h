// Limits and set-up of the static scratch used by
// psy_session_render_samples_static (psy_static.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace psy {

// Paths per batch the static path state holds (window pixels x samples).
constexpr uint32_t kStaticMaxPaths = 1u << 16;
// Bytes of wavefront state per path: the 128-byte path record, eight
// float4 / uint4 fields (128 B) and five 32-bit words (queues, sample,
// shadow owner: 20 B), each array starting on a 256-byte boundary, plus
// 256 B of counters.
constexpr size_t kStaticPerPathBytes = 128u + 8u * 16u + 5u * 4u;
constexpr size_t kStaticPathBytes = size_t(kStaticMaxPaths) * kStaticPerPathBytes + 14u * 256u + 256u;
// The 256-pattern x 256-point Sobol table (renders of at most 256 samples).
constexpr uint32_t kStaticSobolSize = 256u;
constexpr size_t kStaticSobolRows = size_t(kStaticSobolSize) * 256u;
constexpr int kStaticMaxDevices = 64;

// Writes the `size` 4-D points of Sobol pattern `pattern` (4 floats each).
using StaticSobolFill = void (*)(float *points, uint32_t size, uint32_t pattern);

// Device addresses of the static arrays on `device`.  The first call for a
// device, with the set-up lock held, makes `device` current, takes the
// arrays' addresses with cudaGetSymbolAddress, writes the 256 Sobol patterns
// into the static table through `fill` (copies ordered on `stream`, then a
// synchronisation of `stream`), and only then marks the device ready; a
// failing step leaves it not ready, so the next call repeats the set-up.
// Later calls return the cached addresses.
cudaError_t static_scratch(int device, cudaStream_t stream, StaticSobolFill fill, void **paths, float4 **sobol);

}  // namespace psy
