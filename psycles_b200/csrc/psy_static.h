// Limits and set-up of the static scratch used by
// psy_session_render_samples_static (psy_static.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace psy {

// Paths per batch the static path state holds (window pixels x samples).
constexpr uint32_t kStaticMaxPaths = 1u << 16;
// Bytes of wavefront state per path: the 128-byte path record, seven
// float4 / uint4 fields (112 B) and five 32-bit words (queues, sample,
// shadow owner: 20 B), each array starting on a 256-byte boundary, plus
// 256 B of counters.
constexpr size_t kStaticPerPathBytes = 128u + 7u * 16u + 5u * 4u;
constexpr size_t kStaticPathBytes = size_t(kStaticMaxPaths) * kStaticPerPathBytes + 13u * 256u + 256u;
// The 256-pattern x 256-point Sobol table (renders of at most 256 samples).
constexpr uint32_t kStaticSobolSize = 256u;
constexpr size_t kStaticSobolRows = size_t(kStaticSobolSize) * 256u;
constexpr int kStaticMaxDevices = 64;

// Device addresses of the static arrays on `device` (taken with that device
// current on first use and cached).  `first_use` reports whether this call
// did the set-up.
cudaError_t static_scratch(int device, void **paths, float4 **sobol, bool *first_use);

}  // namespace psy
