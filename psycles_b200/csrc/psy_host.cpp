// Host side of libpsycles_cuda.so: the C ABI of include/psycles_cuda.h.
//
//   * host precompute: tabulated-Sobol LUT (src/sampling/tabulated_sobol.cpp),
//     pixel-filter inverse CDF (src/sampling/pixel_filter.cpp), flat light
//     distribution (src/sampling/light_distribution.cpp)
//   * scene compile (LuisaPathTracerBackend::compile_scene,
//     src/luisa/path_tracer_scene.cpp:50): flattening, binned-SAH BVH build
//     per mesh plus an instance TLAS, emitter table, upload
//   * sessions (LuisaRenderSession, src/luisa/path_tracer_session.cpp):
//     film buffers, SampleRange validation, the wavefront render loop and
//     pass readback
// Compiled without FP contraction so the host tables are bit-identical to
// the reference's construction.
#include "psy_host_internal.h"
#include "psy_kernels.h"
#include "psy_light_tree.h"
#include "psy_scene.h"
#include "psy_static.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <exception>
#include <thread>
#include <vector>

namespace psy::host {

thread_local std::string g_last_error;

psy_status fail(psy_status status, const std::string &message) {
    g_last_error = message;
    return status;
}

void bind_records(PathBuffers &b, unsigned char *records) {
    b.ray_o.base = records + psy::kRecRayO;
    b.ray_d.base = records + psy::kRecRayD;
    b.st.base = records + psy::kRecSt;
    b.st2.base = records + psy::kRecSt2;
    b.tp.base = records + psy::kRecTp;
    b.rad.base = records + psy::kRecRad;
    b.hit.base = records + psy::kRecHit;
    b.hit_prim.base = records + psy::kRecHitPrim;
}

psy_status PathArena::ensure(uint32_t n, bool with_job) {
    if (capacity >= n && (!with_job || job.ptr)) return PSY_OK;
    const uint32_t c = std::max(n, capacity);
    const size_t f4 = sizeof(float4) * size_t(c), u4 = sizeof(uint4) * size_t(c), u1 = sizeof(uint32_t) * size_t(c);
    PSY_CUDA_TRY(records.alloc(psy::kPathRecordBytes * size_t(c)));
    // the kernels move record sectors with 32-byte accesses
    if (reinterpret_cast<uintptr_t>(records.ptr) % psy::kPathRecordBytes != 0u)
        return fail(PSY_ERROR_CUDA, "path records are not 128-byte aligned");
    PSY_CUDA_TRY(rad_final.alloc(f4));
    PSY_CUDA_TRY(sample.alloc(u1));
    PSY_CUDA_TRY(aov_n.alloc(f4));
    PSY_CUDA_TRY(aov_a.alloc(f4));
    PSY_CUDA_TRY(mis_n.alloc(f4));
    PSY_CUDA_TRY(sh_o.alloc(f4));
    PSY_CUDA_TRY(sh_d.alloc(f4));
    PSY_CUDA_TRY(sh_c.alloc(f4));
    PSY_CUDA_TRY(sh_ids.alloc(u4));
    PSY_CUDA_TRY(sh_path.alloc(u1));
    PSY_CUDA_TRY(qa.alloc(u1));
    PSY_CUDA_TRY(qb.alloc(u1));
    PSY_CUDA_TRY(sq.alloc(u1));
    if (with_job) PSY_CUDA_TRY(job.alloc(u1));
    PSY_CUDA_TRY(sort_keys.alloc(u1));
    PSY_CUDA_TRY(queue_sorted.alloc(u1));
    if (!sort_hist.ptr) {
        PSY_CUDA_TRY(sort_hist.alloc(2u * psy::kSortBuckets * sizeof(uint32_t)));
        PSY_CUDA_TRY(cudaMemset(sort_hist.ptr, 0, 2u * psy::kSortBuckets * sizeof(uint32_t)));
    }
    if (!counters.ptr) PSY_CUDA_TRY(counters.alloc(64));
    if (!stats.ptr) PSY_CUDA_TRY(stats.alloc(64));
    capacity = c;
    PathBuffers &b = view;
    bind_records(b, records.as<unsigned char>());
    b.rad_final = rad_final.as<float4>();
    b.sample = sample.as<uint32_t>();
    b.aov_n = aov_n.as<float4>();
    b.aov_a = aov_a.as<float4>();
    b.mis_n = mis_n.as<float4>();
    b.sh_o = sh_o.as<float4>();
    b.sh_d = sh_d.as<float4>();
    b.sh_c = sh_c.as<float4>();
    b.sh_ids = sh_ids.as<uint4>();
    b.sh_path = sh_path.as<uint32_t>();
    b.queue_in = qa.as<uint32_t>();
    b.queue_out = qb.as<uint32_t>();
    b.shadow_queue = sq.as<uint32_t>();
    b.counters = counters.as<uint32_t>();
    b.job = job.ptr ? job.as<uint32_t>() : nullptr;
    b.sort_keys = sort_keys.as<uint32_t>();
    b.queue_sorted = queue_sorted.as<uint32_t>();
    b.sort_hist = sort_hist.as<uint32_t>();
    b.sort_offsets = b.sort_hist + psy::kSortBuckets;
    return PSY_OK;
}

size_t PathArena::bytes_per_path(bool with_job) {
    return psy::kPathRecordBytes + 6u * sizeof(float4) + 1u * sizeof(uint4) +
           (8u + (with_job ? 1u : 0u)) * sizeof(uint32_t);
}

}  // namespace psy::host

using namespace psy::host;

namespace {

// ------------------------------------------------------------ Sobol LUT
// Cycles' progressive multi-jittered 4-D table (tabulated_sobol.cpp:75-200).

const uint32_t kXors[4][32] = {
    {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u,
     0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u},
    {0x00000000u, 0x00000001u, 0x00000001u, 0x00000007u, 0x00000001u, 0x00000013u, 0x00000015u, 0x0000007fu,
     0x00000001u, 0x00000103u, 0x00000105u, 0x0000070fu, 0x00000111u, 0x00001333u, 0x00001555u, 0x00007fffu,
     0x00000001u, 0x00010003u, 0x00010005u, 0x0007000fu, 0x00010011u, 0x00130033u, 0x00150055u, 0x007f00ffu,
     0x00010101u, 0x01030303u, 0x01050505u, 0x070f0f0fu, 0x01111111u, 0x13333333u, 0x15555555u, 0x7fffffffu},
    {0x00000000u, 0x00000001u, 0x00000003u, 0x00000001u, 0x00000005u, 0x0000001fu, 0x0000002bu, 0x0000003du,
     0x00000011u, 0x00000133u, 0x00000377u, 0x00000199u, 0x00000445u, 0x00001ccfu, 0x00002ddbu, 0x0000366du,
     0x00000101u, 0x00010303u, 0x00030707u, 0x00010909u, 0x00051515u, 0x001f3f3fu, 0x002b6b6bu, 0x003dbdbdu,
     0x00101011u, 0x01303033u, 0x03707077u, 0x01909099u, 0x04515145u, 0x1cf3f3cfu, 0x2db6b6dbu, 0x36dbdb6du},
    {0x00000000u, 0x00000001u, 0x00000000u, 0x00000003u, 0x0000000du, 0x0000000cu, 0x00000005u, 0x0000004fu,
     0x00000014u, 0x000000e7u, 0x00000329u, 0x0000039cu, 0x00000011u, 0x00001033u, 0x00000044u, 0x000030bbu,
     0x0000d1cdu, 0x0000c2ecu, 0x00005415u, 0x0004fc3fu, 0x00015054u, 0x000e5c97u, 0x0032e5b9u, 0x0039725cu,
     0x00000101u, 0x01000303u, 0x00000404u, 0x03000b0bu, 0x0d001d1du, 0x0c002c2cu, 0x05004545u, 0x4f00cfcfu},
};

uint32_t hp_hash(uint32_t v) {
    v ^= v >> 16u;
    v *= 0x21f0aaadu;
    v ^= v >> 15u;
    v *= 0xd35a2d97u;
    v ^= v >> 15u;
    return v ^ 0xe6fe3bebu;
}
float hp_float(uint32_t v) { return static_cast<float>(hp_hash(v)) * (1.0f / 4294967808.0f); }

void sobol_pattern(float *pts, uint32_t size, uint32_t seed) {
    uint32_t s = 0x44605a73u;
    s ^= s << 19u;
    uint32_t idx = hp_hash(seed ^ s);
    for (int c = 0; c < 4; ++c) pts[c] = hp_float(idx++);
    uint32_t log_n = 0u;
    for (uint32_t n = 1u; n < size; ++log_n, n *= 2u) {
        const float strata = static_cast<float>(n * 2u);
        for (uint32_t i = 0u; i < n && n + i < size; ++i) {
            uint32_t occ[4];
            for (int c = 0; c < 4; ++c) occ[c] = static_cast<uint32_t>(pts[4 * (i ^ kXors[c][log_n]) + c] * strata);
            for (int c = 0; c < 4; ++c)
                pts[4 * (n + i) + c] = (static_cast<float>(occ[c] ^ 1u) + hp_float(idx++)) / strata;
        }
    }
}

bool sobol_size_valid(uint32_t s) { return s >= 256u && s <= 8192u && (s & (s - 1u)) == 0u; }

// ------------------------------------------------------- pixel filter

std::array<float, 1024> filter_table(uint32_t filter, float width) {
    width = std::max(width, 1.0e-5f);
    int kind = 0;
    if (filter == PSY_FILTER_GAUSSIAN) {
        kind = 1;
        width *= 3.0f;
    } else if (filter == PSY_FILTER_BLACKMAN_HARRIS) {
        kind = 2;
        width *= 2.0f;
    }
    auto f = [&](float v, float w) -> float {
        if (kind == 1) {
            v *= 6.0f / w;
            return std::exp(-2.0f * v * v);
        }
        if (kind == 2) {
            constexpr float two_pi = 6.28318530717958647692f;
            v = two_pi * (v / w + 0.5f);
            return 0.35875f - 0.48829f * std::cos(v) + 0.14128f * std::cos(2.0f * v) - 0.01168f * std::cos(3.0f * v);
        }
        return 1.0f;
    };
    constexpr size_t n = 1024u, res = n - 1u, half = (n - 1u) / 2u;
    std::array<float, n> cdf{};
    const float range = width * 0.5f;
    for (size_t i = 0; i < res; ++i) {
        const float v = range * static_cast<float>(i) / static_cast<float>(res - 1u);
        cdf[i + 1u] = cdf[i] + std::fabs(f(v, width));
    }
    const float norm = cdf[res] == 0.0f ? 0.0f : 1.0f / cdf[res];
    for (auto &v : cdf) v *= norm;
    cdf[res] = 1.0f;
    std::array<float, n> inv{};
    for (size_t i = 0; i <= half; ++i) {
        const float x = static_cast<float>(i) / static_cast<float>(half);
        size_t index = static_cast<size_t>(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
        float t = 0.0f;
        if (index < res) t = (x - cdf[index]) / (cdf[index + 1u] - cdf[index]);
        else index = res;
        const float y = (static_cast<float>(index) + t) / static_cast<float>(n - 1u) * (2.0f * range);
        inv[half + i] = 0.5f * (1.0f + y);
        inv[half - i] = 0.5f * (1.0f - y);
    }
    return inv;
}

// ------------------------------------------------------------- geometry

struct V3 {
    float x, y, z;
};
V3 v3(float x, float y, float z) { return {x, y, z}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 crs(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float dt(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct M34 {
    V3 c0, c1, c2, c3;
};
M34 m34(const float *e) { return {{e[0], e[1], e[2]}, {e[4], e[5], e[6]}, {e[8], e[9], e[10]}, {e[12], e[13], e[14]}}; }
V3 xaff(const M34 &m, V3 v, bool t) {
    const float tx = t ? m.c3.x : 0.0f, ty = t ? m.c3.y : 0.0f, tz = t ? m.c3.z : 0.0f;
    return {std::fma(v.x, m.c0.x, std::fma(v.y, m.c1.x, std::fma(v.z, m.c2.x, tx))),
            std::fma(v.x, m.c0.y, std::fma(v.y, m.c1.y, std::fma(v.z, m.c2.y, ty))),
            std::fma(v.x, m.c0.z, std::fma(v.y, m.c1.z, std::fma(v.z, m.c2.z, tz)))};
}
// Affine inverse in double precision with one rounding to float.
M34 inverse34(const M34 &m) {
    const double a00 = m.c0.x, a10 = m.c0.y, a20 = m.c0.z, a01 = m.c1.x, a11 = m.c1.y, a21 = m.c1.z;
    const double a02 = m.c2.x, a12 = m.c2.y, a22 = m.c2.z, t0 = m.c3.x, t1 = m.c3.y, t2 = m.c3.z;
    const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double inv = det != 0.0 ? 1.0 / det : 0.0;
    const double i00 = c00 * inv, i01 = (a02 * a21 - a01 * a22) * inv, i02 = (a01 * a12 - a02 * a11) * inv;
    const double i10 = c01 * inv, i11 = (a00 * a22 - a02 * a20) * inv, i12 = (a02 * a10 - a00 * a12) * inv;
    const double i20 = c02 * inv, i21 = (a01 * a20 - a00 * a21) * inv, i22 = (a00 * a11 - a01 * a10) * inv;
    const double u0 = -(i00 * t0 + i01 * t1 + i02 * t2);
    const double u1 = -(i10 * t0 + i11 * t1 + i12 * t2);
    const double u2 = -(i20 * t0 + i21 * t1 + i22 * t2);
    M34 r;
    r.c0 = {float(i00), float(i10), float(i20)};
    r.c1 = {float(i01), float(i11), float(i21)};
    r.c2 = {float(i02), float(i12), float(i22)};
    r.c3 = {float(u0), float(u1), float(u2)};
    return r;
}
void store34(float *dst, const M34 &m) {
    const V3 cols[4] = {m.c0, m.c1, m.c2, m.c3};
    for (int c = 0; c < 4; ++c) {
        dst[3 * c + 0] = cols[c].x;
        dst[3 * c + 1] = cols[c].y;
        dst[3 * c + 2] = cols[c].z;
    }
}

// ------------------------------------------------------------ BVH build

struct Box {
    double lo[3] = {1e300, 1e300, 1e300};
    double hi[3] = {-1e300, -1e300, -1e300};
    void grow(const Box &b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(double x, double y, double z) {
        const double p[3] = {x, y, z};
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    bool empty() const { return lo[0] > hi[0]; }
    double area() const {
        if (empty()) return 0.0;
        const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct Prim {
    Box box;
    double c[3];
    uint32_t id;
};

// Pads a child box so that float slab tests never cull a triangle the
// Pluecker predicate accepts: relative 1e-5 of the extent plus 1e-6 of the
// coordinate magnitude, rounded outward.
void padded(const Box &b, float lo[3], float hi[3]) {
    for (int a = 0; a < 3; ++a) {
        if (b.empty()) {
            lo[a] = 1.0f;
            hi[a] = -1.0f;
            continue;
        }
        const double pad = 1e-5 * (b.hi[a] - b.lo[a]) + 1e-6 * std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])) + 1e-30;
        lo[a] = std::nextafter(float(b.lo[a] - pad), -INFINITY);
        hi[a] = std::nextafter(float(b.hi[a] + pad), INFINITY);
    }
}

#ifndef PSY_LEAF_SIZE
#define PSY_LEAF_SIZE 1u
#endif
#ifndef PSY_SAH_BINS
#define PSY_SAH_BINS 32
#endif
#ifndef PSY_SAH_AXES
#define PSY_SAH_AXES 3
#endif

struct Builder {
    std::vector<psy::BvhNodeGpu> nodes;
    std::vector<Prim> prims;
    uint32_t leaf_size = PSY_LEAF_SIZE;
    bool leaf_is_id = false;  // TLAS: leaf link = ~prim id, count 1
    bool parallel = true;     // large subtrees on threads of their own
    // binary depth below which splits are chosen by SAH; deeper ranges split
    // at the centroid median of the widest axis (0: median splits only, the
    // balanced tree the traversal-stack check falls back to)
    int sah_depth_limit = 60;

    struct Child {
        Box box;
        int link;
        int count;
    };

    Child leaf(uint32_t begin, uint32_t end, const Box &box) {
        if (leaf_is_id) return {box, ~int(prims[begin].id), 1};
        return {box, ~int(begin), int(end - begin)};
    }

    static void grow_side(const Prim &p, Box &box, Box &cbox) {
        box.grow(p.box);
        cbox.grow(p.c[0], p.c[1], p.c[2]);
    }

    // Binary SAH build of prims [begin, end) into `out` (pre-order node
    // list).  Large ranges near the root build their right half on a thread
    // of its own into a separate list that is spliced in after the left
    // half, so the tree and its node order equal the sequential build's
    // (the two halves touch disjoint prim ranges).
    Child build(uint32_t begin, uint32_t end, int depth) {
        Box box, cbox;
        bounds(begin, end, box, cbox);
        return build_into(nodes, begin, end, depth, box, cbox);
    }

    // Box of the prims [begin, end) and of their centroids.
    void bounds(uint32_t begin, uint32_t end, Box &box, Box &cbox) const {
        for (uint32_t i = begin; i < end; ++i) {
            box.grow(prims[i].box);
            cbox.grow(prims[i].c[0], prims[i].c[1], prims[i].c[2]);
        }
    }

    // `box` / `cbox` bound the prims [begin, end) and their centroids.
    Child build_into(std::vector<psy::BvhNodeGpu> &out, uint32_t begin, uint32_t end, int depth, const Box &box,
                     const Box &cbox) {
        const uint32_t count = end - begin;
        if (count <= leaf_size) return leaf(begin, end, box);
        // binned SAH: PSY_SAH_BINS bins on every axis with a centroid extent
        // (PSY_SAH_AXES 1: the widest axis only)
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (cbox.hi[a] - cbox.lo[a] > cbox.hi[axis] - cbox.lo[axis]) axis = a;
        uint32_t mid = begin + count / 2u;
        bool done = false;
        Box lbox, lcbox, rbox, rcbox;
        if (depth < sah_depth_limit) {
            // one pass bins the centroids on every axis; the sweep then visits
            // only the boundaries right after non-empty bins (a boundary after
            // an empty bin costs the same as the one before it, and the first
            // of equal costs wins, so the chosen split is the one a sweep over
            // every boundary finds)
            constexpr int kBins = PSY_SAH_BINS;
            struct BinBox {
                double lo[3], hi[3];
            };
            BinBox bins[3][kBins];
            uint32_t counts[3][kBins] = {};
            double scale[3];
            bool use[3];
            for (int a = 0; a < 3; ++a) {
                const double extent = cbox.hi[a] - cbox.lo[a];
                use[a] = (PSY_SAH_AXES != 1 || a == axis) && extent > 0.0;
                scale[a] = use[a] ? kBins / extent : 0.0;
            }
            for (uint32_t i = begin; i < end; ++i) {
                const Prim &p = prims[i];
                for (int a = 0; a < 3; ++a) {
                    if (!use[a]) continue;
                    const int bn = std::min(std::max(int((p.c[a] - cbox.lo[a]) * scale[a]), 0), kBins - 1);
                    BinBox &bb = bins[a][bn];
                    if (counts[a][bn]++ == 0u) {
                        for (int e = 0; e < 3; ++e) {
                            bb.lo[e] = p.box.lo[e];
                            bb.hi[e] = p.box.hi[e];
                        }
                    } else {
                        for (int e = 0; e < 3; ++e) {
                            bb.lo[e] = std::min(bb.lo[e], p.box.lo[e]);
                            bb.hi[e] = std::max(bb.hi[e], p.box.hi[e]);
                        }
                    }
                }
            }
            double best = 1e300;
            int best_split = -1, best_axis = -1;
            for (int a = 0; a < 3; ++a) {
                if (!use[a]) continue;
                int filled[kBins];
                int m = 0;
                for (int bn = 0; bn < kBins; ++bn)
                    if (counts[a][bn] != 0u) filled[m++] = bn;
                if (m < 2) continue;
                double right_area[kBins];
                uint32_t right_count[kBins];
                Box acc;
                uint32_t acc_n = 0u;
                for (int j = m - 1; j > 0; --j) {
                    const BinBox &bb = bins[a][filled[j]];
                    for (int e = 0; e < 3; ++e) {
                        acc.lo[e] = std::min(acc.lo[e], bb.lo[e]);
                        acc.hi[e] = std::max(acc.hi[e], bb.hi[e]);
                    }
                    acc_n += counts[a][filled[j]];
                    right_area[j] = acc.area();
                    right_count[j] = acc_n;
                }
                Box left;
                uint32_t left_n = 0u;
                for (int j = 1; j < m; ++j) {
                    const BinBox &bb = bins[a][filled[j - 1]];
                    for (int e = 0; e < 3; ++e) {
                        left.lo[e] = std::min(left.lo[e], bb.lo[e]);
                        left.hi[e] = std::max(left.hi[e], bb.hi[e]);
                    }
                    left_n += counts[a][filled[j - 1]];
                    const double cost = left.area() * left_n + right_area[j] * right_count[j];
                    if (cost < best) {
                        best = cost;
                        best_split = filled[j - 1] + 1;
                        best_axis = a;
                    }
                }
            }
            if (best_split > 0) {
                const int a = best_axis;
                const double scale_a = scale[a];
                const auto left_side = [&](const Prim &p) {
                    return std::min(std::max(int((p.c[a] - cbox.lo[a]) * scale_a), 0), kBins - 1) < best_split;
                };
                // two-ended partition (the classic exchange order, so the
                // permutation is the one std::partition gives on these
                // iterators) that also bounds both sides for the children
                uint32_t first = begin, last = end;
                for (;;) {
                    while (first != last && left_side(prims[first])) {
                        grow_side(prims[first], lbox, lcbox);
                        ++first;
                    }
                    if (first == last) break;
                    --last;
                    while (first != last && !left_side(prims[last])) {
                        grow_side(prims[last], rbox, rcbox);
                        --last;
                    }
                    if (first == last) {
                        grow_side(prims[last], rbox, rcbox);
                        break;
                    }
                    std::swap(prims[first], prims[last]);
                    grow_side(prims[first], lbox, lcbox);
                    grow_side(prims[last], rbox, rcbox);
                    ++first;
                }
                mid = first;
                done = mid > begin && mid < end;
            }
        }
        if (!done) {
            mid = begin + count / 2u;
            std::nth_element(prims.begin() + begin, prims.begin() + mid, prims.begin() + end,
                             [&](const Prim &a, const Prim &b) {
                                 return a.c[axis] < b.c[axis] || (a.c[axis] == b.c[axis] && a.id < b.id);
                             });
            lbox = lcbox = rbox = rcbox = Box{};
            bounds(begin, mid, lbox, lcbox);
            bounds(mid, end, rbox, rcbox);
        }
        const int index = int(out.size());
        out.push_back({});
        Child l, r;
        if (parallel && depth < 8 && count >= 2048u) {
            std::vector<psy::BvhNodeGpu> right_nodes;
            std::exception_ptr error;
            std::thread worker([&]() {
                try {
                    r = build_into(right_nodes, mid, end, depth + 1, rbox, rcbox);
                } catch (...) {
                    error = std::current_exception();
                }
            });
            try {
                l = build_into(out, begin, mid, depth + 1, lbox, lcbox);
            } catch (...) {
                worker.join();
                throw;
            }
            worker.join();
            if (error) std::rethrow_exception(error);
            const int offset = int(out.size());
            for (psy::BvhNodeGpu &n : right_nodes) {
                if (n.child.x >= 0) n.child.x += offset;
                if (n.child.y >= 0) n.child.y += offset;
            }
            out.insert(out.end(), right_nodes.begin(), right_nodes.end());
            if (r.link >= 0) r.link += offset;
        } else {
            l = build_into(out, begin, mid, depth + 1, lbox, lcbox);
            r = build_into(out, mid, end, depth + 1, rbox, rcbox);
        }
        write(out, index, l, r);
        return {box, index, 0};
    }

    void write(int index, const Child &l, const Child &r) { write(nodes, index, l, r); }

    void write(std::vector<psy::BvhNodeGpu> &out, int index, const Child &l, const Child &r) {
        float llo[3], lhi[3], rlo[3], rhi[3];
        padded(l.box, llo, lhi);
        padded(r.box, rlo, rhi);
        psy::BvhNodeGpu &n = out[size_t(index)];
        n.x = make_float4(llo[0], lhi[0], rlo[0], rhi[0]);
        n.y = make_float4(llo[1], lhi[1], rlo[1], rhi[1]);
        n.z = make_float4(llo[2], lhi[2], rlo[2], rhi[2]);
        n.child = make_int4(l.link, r.link, l.count, r.count);
    }

    // The 4-wide BVH of the binary nodes: starting from a binary node's two
    // children, the inner child of largest surface area is replaced by its
    // own two children until four children (or only leaves) remain; then
    // every inner child is collapsed the same way.  Child boxes are the
    // binary build's padded boxes, so the slab test stays conservative.
    std::vector<psy::WideNodeGpu> widen() const {
        std::vector<psy::WideNodeGpu> wide;
        wide.reserve(nodes.size() / 2u + 1u);
        collapse(0, wide);
        return wide;
    }

    struct WideChild {
        float lo[3], hi[3];
        int link, count;
        double area() const {
            if (lo[0] > hi[0]) return -1.0;
            const double dx = double(hi[0]) - lo[0], dy = double(hi[1]) - lo[1], dz = double(hi[2]) - lo[2];
            return dx * dy + dy * dz + dz * dx;
        }
    };

    WideChild child_of(int node, int side) const {
        const psy::BvhNodeGpu &n = nodes[size_t(node)];
        WideChild c;
        if (side == 0) {
            c.lo[0] = n.x.x, c.hi[0] = n.x.y, c.lo[1] = n.y.x, c.hi[1] = n.y.y, c.lo[2] = n.z.x, c.hi[2] = n.z.y;
            c.link = n.child.x, c.count = n.child.z;
        } else {
            c.lo[0] = n.x.z, c.hi[0] = n.x.w, c.lo[1] = n.y.z, c.hi[1] = n.y.w, c.lo[2] = n.z.z, c.hi[2] = n.z.w;
            c.link = n.child.y, c.count = n.child.w;
        }
        return c;
    }

    int collapse(int node, std::vector<psy::WideNodeGpu> &wide) const {
        WideChild kids[4] = {child_of(node, 0), child_of(node, 1), {}, {}};
        int n = 2;
        while (n < 4) {
            int best = -1;
            double best_area = -2.0;
            for (int k = 0; k < n; ++k)
                if (kids[k].link >= 0 && kids[k].area() > best_area) {
                    best = k;
                    best_area = kids[k].area();
                }
            if (best < 0) break;
            const int inner = kids[best].link;
            kids[best] = child_of(inner, 0);
            kids[n++] = child_of(inner, 1);
        }
        const int index = int(wide.size());
        wide.push_back({});
        int links[4], counts[4];
        float lo[3][4], hi[3][4];
        // empty slots (and empty leaves) get +inf planes on every axis: the
        // traversal's slab test then misses them for any ray direction
        for (int k = 0; k < 4; ++k) {
            if (k < n && (kids[k].link >= 0 || kids[k].count > 0)) {
                for (int a = 0; a < 3; ++a) {
                    lo[a][k] = kids[k].lo[a];
                    hi[a][k] = kids[k].hi[a];
                }
                // the traversal pushes a count-0 slot's link as it is: a
                // tagged node index (BLAS indices are made global when the
                // meshes are concatenated) or a tagged instance; a leaf of
                // triangles keeps its first primitive (made global likewise)
                if (kids[k].link >= 0) {
                    links[k] = int((leaf_is_id ? psy::kTagTlas : psy::kTagBlas) | uint32_t(collapse(kids[k].link, wide)));
                    counts[k] = 0;
                } else if (leaf_is_id) {
                    links[k] = int(psy::kTagInstance | uint32_t(~kids[k].link));
                    counts[k] = 0;
                } else {
                    links[k] = ~kids[k].link;
                    counts[k] = kids[k].count;
                }
            } else {
                for (int a = 0; a < 3; ++a) {
                    lo[a][k] = INFINITY;
                    hi[a][k] = INFINITY;
                }
                links[k] = int(psy::kInvalidId);
                counts[k] = 0;
            }
        }
        psy::WideNodeGpu &w = wide[size_t(index)];
        w.lox = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
        w.hix = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
        w.loy = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
        w.hiy = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
        w.loz = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
        w.hiz = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
        w.link = make_int4(links[0], links[1], links[2], links[3]);
        w.count = make_int4(counts[0], counts[1], counts[2], counts[3]);
        return index;
    }

    // The compressed 8-wide BVH of the binary nodes: each node takes up to
    // eight children by opening the inner child of largest area (as
    // collapse does for four), assigns them to slots by octant, and
    // quantises their padded boxes outward onto a per-node byte grid.  Nodes
    // are emitted breadth first, so a node's inner children are contiguous;
    // `leaves` receives each node's leaf entries (binary leaf: prim index;
    // TLAS: instance id) in slot order, which is the order their records
    // must be laid out in.  Indices are relative to the tree.
    std::vector<psy::CwNodeGpu> widen8(std::vector<uint32_t> &leaves) const {
        std::vector<psy::CwNodeGpu> out(1);
        leaves.clear();
        std::vector<std::pair<int, uint32_t>> queue{{0, 0u}};  // (binary node, output node)
        for (size_t j = 0; j < queue.size(); ++j) {
            WideChild kids[8] = {child_of(queue[j].first, 0), child_of(queue[j].first, 1)};
            int n = 2;
            while (n < 8) {
                int best = -1;
                double best_area = -2.0;
                for (int k = 0; k < n; ++k)
                    if (kids[k].link >= 0 && kids[k].area() > best_area) {
                        best = k;
                        best_area = kids[k].area();
                    }
                if (best < 0) break;
                const int inner = kids[best].link;
                kids[best] = child_of(inner, 0);
                kids[n++] = child_of(inner, 1);
            }
            // drop empty children (no link, no triangles)
            int m = 0;
            for (int k = 0; k < n; ++k)
                if (kids[k].link >= 0 || kids[k].count > 0) kids[m++] = kids[k];
            n = m;
            // node box and slot assignment: slot s takes the child whose
            // centre lies furthest against direction octant s, greedily by
            // the most negative projection first
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int k = 0; k < n; ++k)
                for (int a = 0; a < 3; ++a) {
                    lo[a] = std::min(lo[a], double(kids[k].lo[a]));
                    hi[a] = std::max(hi[a], double(kids[k].hi[a]));
                }
            int slot_of[8];
            {
                bool used_child[8] = {}, used_slot[8] = {};
                double cost[8][8];
                for (int k = 0; k < n; ++k)
                    for (int s = 0; s < 8; ++s) {
                        double c = 0.0;
                        for (int a = 0; a < 3; ++a) {
                            const double d = 0.5 * (double(kids[k].lo[a]) + kids[k].hi[a]) - 0.5 * (lo[a] + hi[a]);
                            c += ((s >> a) & 1) ? -d : d;
                        }
                        cost[k][s] = c;
                    }
                for (int step = 0; step < n; ++step) {
                    int bk = -1, bs = -1;
                    for (int k = 0; k < n; ++k)
                        for (int s = 0; s < 8; ++s)
                            if (!used_child[k] && !used_slot[s] && (bk < 0 || cost[k][s] < cost[bk][bs])) {
                                bk = k;
                                bs = s;
                            }
                    used_child[bk] = used_slot[bs] = true;
                    slot_of[bk] = bs;
                }
            }
            int child_in_slot[8];
            for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
            for (int k = 0; k < n; ++k) child_in_slot[slot_of[k]] = k;
            // quantisation grid: origin below the node box by a margin that
            // covers the slab test's float rounding (relative to the node's
            // extent and magnitude), power-of-two cells of 255 steps
            psy::CwNodeGpu node{};
            double origin[3], cell[3], margin[3];
            uint32_t exps = 0u;
            for (int a = 0; a < 3; ++a) {
                if (n == 0) {
                    lo[a] = hi[a] = 0.0;
                }
                margin[a] = 4e-6 * (hi[a] - lo[a]) + 4e-6 * std::max(std::fabs(lo[a]), std::fabs(hi[a])) + 1e-30;
                const float p = std::nextafter(float(lo[a] - margin[a]), -INFINITY);
                origin[a] = double(p);
                const double span = (hi[a] + margin[a]) - origin[a];
                int e = int(std::ceil(std::log2(std::max(span, 1e-300) / 255.0)));
                e = std::max(e, -126);
                while (std::ldexp(255.0, e) < span) ++e;
                cell[a] = std::ldexp(1.0, e);
                exps |= uint32_t(e + 127) << (8 * a);
            }
            node.px = float(origin[0]);
            node.py = float(origin[1]);
            node.pz = float(origin[2]);
            uint32_t imask = 0u, leafmask = 0u;
            for (int s = 0; s < 8; ++s) {
                const int k = child_in_slot[s];
                if (k < 0) continue;
                if (kids[k].link >= 0) imask |= 1u << s;
                else leafmask |= 1u << s;
                for (int a = 0; a < 3; ++a) {
                    const double ql = std::floor(((double(kids[k].lo[a]) - margin[a]) - origin[a]) / cell[a]);
                    const double qh = std::ceil(((double(kids[k].hi[a]) + margin[a]) - origin[a]) / cell[a]);
                    const uint32_t bl = uint32_t(std::min(std::max(ql, 0.0), 255.0));
                    const uint32_t bh = uint32_t(std::min(std::max(qh, 0.0), 255.0));
                    node.q[2 * a + (s >> 2)] |= bl << (8 * (s & 3));
                    node.q[6 + 2 * a + (s >> 2)] |= bh << (8 * (s & 3));
                }
            }
            node.exps_imask = exps | (imask << 24);
            node.leafmask = leafmask;
            node.child_base = uint32_t(out.size());
            node.leaf_base = uint32_t(leaves.size());
            for (int s = 0; s < 8; ++s) {
                const int k = child_in_slot[s];
                if (k < 0) continue;
                if (kids[k].link >= 0) {
                    queue.push_back({kids[k].link, uint32_t(out.size())});
                    out.push_back({});
                } else {
                    leaves.push_back(uint32_t(~kids[k].link));
                }
            }
            out[queue[j].second] = node;
        }
        return out;
    }

    // Root node: a single leaf still gets a two-child root (empty right).
    Box build_root() {
        nodes.clear();
        Box box;
        for (const auto &p : prims) box.grow(p.box);
        if (prims.empty()) {
            nodes.push_back({});
            write(0, Child{Box{}, ~0, 0}, Child{Box{}, ~0, 0});
            return box;
        }
        if (prims.size() <= leaf_size && !leaf_is_id) {
            nodes.push_back({});
            write(0, leaf(0u, uint32_t(prims.size()), box), Child{Box{}, ~0, 0});
            return box;
        }
        if (prims.size() == 1u) {
            nodes.push_back({});
            write(0, leaf(0u, 1u, box), Child{Box{}, ~0, 0});
            return box;
        }
        const Child root = build(0u, uint32_t(prims.size()), 0);
        (void)root;
        return box;
    }
};

// Traversal-stack bound.  A visit of a wide node pushes every hit child it
// does not descend into (inner nodes; instances in the TLAS) and continues
// with one of them, so while a child's subtree is walked at most (n - 1) of
// the node's n pushable children wait on the stack, whichever order the ray
// takes.  Entering an instance pushes one more entry (the return to the
// world ray) before the BLAS root.  The bounds below are therefore the
// largest stack any ray can build, and the compile step keeps them within
// the device stack (psy::kTraversalStackSize).

// Pushable children (count-0 slots with a link) of a wide node.
int wide_pushable(const psy::WideNodeGpu &w, uint32_t links[4]) {
    const int *lk = &w.link.x;
    const int *ct = &w.count.x;
    int n = 0;
    for (int k = 0; k < 4; ++k)
        if (ct[k] == 0 && uint32_t(lk[k]) != psy::kInvalidId) links[n++] = uint32_t(lk[k]);
    return n;
}

// Entries a BLAS walk adds above those waiting when its root is entered
// (mesh-local node indices; a parent precedes its children).
uint32_t blas_stack_need(const std::vector<psy::WideNodeGpu> &w) {
    std::vector<uint32_t> need(w.size(), 0u);
    for (size_t i = w.size(); i-- > 0;) {
        uint32_t links[4];
        const int n = wide_pushable(w[i], links);
        uint32_t deepest = 0u;
        for (int k = 0; k < n; ++k) deepest = std::max(deepest, need[links[k] & ~psy::kTagMask]);
        need[i] = n > 0 ? uint32_t(n - 1) + deepest : 0u;
    }
    return w.empty() ? 0u : need[0];
}

// The same bounds for the compressed 8-wide trees, whose traversal keeps
// one stack entry per node group: a visit that continues into one of n hit
// inner children leaves the other n - 1 as one entry (so one entry when
// n >= 2).  In the TLAS a node with hit instances first stacks its inner
// hits (one entry when it has any), then the other hit instances (one entry
// when there are two or more) and the return to the world ray.
[[maybe_unused]] uint32_t blas_stack_need8(const std::vector<psy::CwNodeGpu> &w) {
    std::vector<uint32_t> need(w.size(), 0u);
    for (size_t i = w.size(); i-- > 0;) {
        const uint32_t imask = w[i].exps_imask >> 24;
        const uint32_t n = uint32_t(__builtin_popcount(imask));
        uint32_t deepest = 0u;
        for (uint32_t k = 0; k < n; ++k) deepest = std::max(deepest, need[w[i].child_base + k]);
        need[i] = n > 0 ? (n >= 2 ? 1u : 0u) + deepest : 0u;
    }
    return w.empty() ? 0u : need[0];
}

[[maybe_unused]] std::vector<uint32_t> tlas_instance_depths8(const std::vector<psy::CwNodeGpu> &w, const std::vector<uint32_t> &leaves,
                                            uint32_t instance_count) {
    std::vector<uint32_t> depth(w.size(), 0u), inst(instance_count, 0u);
    for (size_t i = 0; i < w.size(); ++i) {
        const uint32_t imask = w[i].exps_imask >> 24, leafmask = w[i].leafmask;
        const uint32_t ni = uint32_t(__builtin_popcount(imask)), nl = uint32_t(__builtin_popcount(leafmask));
        for (uint32_t k = 0; k < ni; ++k) depth[w[i].child_base + k] = depth[i] + (ni >= 2 ? 1u : 0u);
        const uint32_t entered = depth[i] + (ni > 0 ? 1u : 0u) + (nl >= 2 ? 1u : 0u);
        for (uint32_t k = 0; k < nl; ++k) {
            const uint32_t id = leaves[w[i].leaf_base + k];
            if (id < instance_count) inst[id] = entered;
        }
    }
    return inst;
}

// Entries waiting on the stack when each instance of the TLAS is entered
// (0 for instances the TLAS does not reference).
std::vector<uint32_t> tlas_instance_depths(const std::vector<psy::WideNodeGpu> &w, uint32_t instance_count) {
    std::vector<uint32_t> depth(w.size(), 0u), inst(instance_count, 0u);
    for (size_t i = 0; i < w.size(); ++i) {
        uint32_t links[4];
        const int n = wide_pushable(w[i], links);
        for (int k = 0; k < n; ++k) {
            const uint32_t below = depth[i] + uint32_t(n - 1);
            const uint32_t idx = links[k] & ~psy::kTagMask;
            if ((links[k] & psy::kTagMask) == psy::kTagInstance) {
                if (idx < instance_count) inst[idx] = below;
            } else if (idx < w.size()) {
                depth[idx] = below;
            }
        }
    }
    return inst;
}


}  // namespace


namespace {

// Light selection of a render from the scene's current tables: the tree is
// used only where the scene has one; NEE runs only when a light can be
// picked and the mode is not forward path tracing, and without NEE every
// emitter is weighted as forward path tracing
// (src/luisa/path_tracer_kernel.cpp:206-223).  Re-applied before every
// render, so a tree rebuilt by a parameter edit is picked up.
void apply_light_selection(psy::RenderParams &p, const psy_render_settings &r, const psy::SceneView &sv) {
    p.use_light_tree = (r.use_light_tree && sv.lt_node_count > 0u && sv.lt_emitter_count > 0u) ? 1u : 0u;
    const bool available = p.use_light_tree ? sv.lt_emitter_count > 0u : sv.emitter_count > 0u;
    const bool nee = r.next_event_estimation != 0u && r.direct_light_sampling != PSY_DIRECT_LIGHT_FORWARD && available;
    p.nee = nee ? 1u : 0u;
    p.direct_mode = nee ? r.direct_light_sampling : PSY_DIRECT_LIGHT_FORWARD;
}

psy_status derive_params(psy_session *s, const psy_render_settings &r) {
    if (r.full_width == 0u || r.full_height == 0u)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "render extent must be non-empty");
    const uint32_t ww = r.window_width ? r.window_width : r.full_width;
    const uint32_t wh = r.window_height ? r.window_height : r.full_height;
    if (uint64_t(r.window_x) + ww > r.full_width || uint64_t(r.window_y) + wh > r.full_height)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "render window lies outside the full extent");
    if (r.transparent_max_bounces > 255u || r.max_bounces > 250u || r.diffuse_bounces > 250u ||
        r.glossy_bounces > 250u || r.transmission_bounces > 250u)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "bounce limits above 250 are not supported");
    if (r.direct_light_sampling > PSY_DIRECT_LIGHT_NEE)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "unknown direct light sampling mode");
    psy::RenderParams &p = s->params;
    p.full_w = r.full_width;
    p.full_h = r.full_height;
    p.win_x = r.window_x;
    p.win_y = r.window_y;
    p.win_w = ww;
    p.win_h = wh;
    p.seed = r.seed;
    p.transparent_background = r.transparent_background;
    p.pass_alpha_threshold = r.pass_alpha_threshold;
    // cycles_kernel_bounce_limits (src/luisa/cycles_integrator_limits.h:62-85)
    p.maximum = r.max_bounces + 1u;
    p.minimum = r.min_bounces + 1u;
    p.max_diffuse = r.diffuse_bounces + 1u;
    p.max_glossy = r.glossy_bounces + 1u;
    p.max_transmission = r.transmission_bounces + 1u;
    p.transparent_min = r.transparent_min_bounces + 1u;
    p.transparent_max = r.transparent_max_bounces;
    p.steps = std::min<uint32_t>(2u * p.maximum + std::max(p.transparent_max, 1u) + 1u, 1024u);
    p.clamp_direct = r.sample_clamp_direct;
    p.clamp_indirect = r.sample_clamp_indirect;
    p.inv_rr_threshold = (!r.use_light_tree && r.light_sampling_threshold > 0.0f)
                             ? r.film_exposure / r.light_sampling_threshold : 0.0f;
    if (r.use_light_tree) {
        const psy_status built = ensure_light_tree(s->scene);
        if (built != PSY_OK) return built;
    }
    apply_light_selection(p, r, s->scene->view);
    // camera parameters (src/luisa/path_tracer_kernel.cpp:225-280)
    const psy_camera_desc &c = s->has_camera ? s->camera : s->scene->camera;
    const float aspect = static_cast<float>(std::max(r.full_width, 1u)) / static_cast<float>(std::max(r.full_height, 1u));
    const bool hfit = c.sensor_fit == 1u || (c.sensor_fit == 0u && aspect >= 1.0f);
    p.vtan = hfit ? std::tan(c.horizontal_field_of_view * 0.5f) / aspect : std::tan(c.field_of_view * 0.5f);
    p.htan = p.vtan * aspect;
    p.shift_x = c.lens_shift_x * (hfit ? 1.0f : 1.0f / aspect);
    p.shift_y = c.lens_shift_y * (hfit ? aspect : 1.0f);
    p.near_clip = c.near_clip;
    p.far_clip = c.far_clip;
    // orthographic_viewplane_span (include/psycles/luisa/camera_sampling.h:47-53)
    // and the depth-of-field switch (src/luisa/path_tracer_kernel.cpp:246-278)
    if (c.projection > PSY_CAMERA_PANORAMA) return fail(PSY_ERROR_INVALID_ARGUMENT, "unknown camera projection");
    p.projection = c.projection;
    p.ortho_span = hfit ? c.orthographic_scale / aspect : c.orthographic_scale;
    p.aperture_radius = c.aperture_radius;
    p.focal_distance = c.focal_distance;
    p.aperture_ratio = c.aperture_ratio;
    p.aperture_blades = c.aperture_blades;
    p.aperture_rotation = c.aperture_rotation;
    p.depth_of_field =
        (c.projection == PSY_CAMERA_PERSPECTIVE && c.aperture_radius > 0.0f && c.focal_distance > 0.0f) ? 1u : 0u;
    store34(p.cam, m34(c.camera_to_world));
    s->pixels = ww * wh;
    return PSY_OK;
}

psy_status ensure_capacity(psy_session *s, uint32_t n) {
    return s->scene->context->arena.ensure(n, false);
}

psy_status clear_film(psy_session *s, bool sync = true) {
    cudaStream_t st = s->scene->context->stream;
    const size_t n = s->pixels;
    PSY_CUDA_TRY(s->combined.alloc(sizeof(float4) * n));
    PSY_CUDA_TRY(s->normal.alloc(sizeof(float4) * n));
    PSY_CUDA_TRY(s->albedo.alloc(sizeof(float4) * n));
    PSY_CUDA_TRY(s->sample_count.alloc(sizeof(uint32_t) * n));
    PSY_CUDA_TRY(cudaMemsetAsync(s->combined.ptr, 0, sizeof(float4) * n, st));
    PSY_CUDA_TRY(cudaMemsetAsync(s->normal.ptr, 0, sizeof(float4) * n, st));
    PSY_CUDA_TRY(cudaMemsetAsync(s->albedo.ptr, 0, sizeof(float4) * n, st));
    PSY_CUDA_TRY(cudaMemsetAsync(s->sample_count.ptr, 0, sizeof(uint32_t) * n, st));
    if (sync) PSY_CUDA_TRY(cudaStreamSynchronize(st));
    s->rendered = 0;
    s->total = 0;
    return PSY_OK;
}


// Checks a compiled SurfaceProgram against what the kernels interpret: the
// in-scope closure and value operations, operands that name earlier value
// instructions of the right type, parameter slots inside the block, and
// closure inputs of the type their socket takes.
psy_status validate_material(const psy_material_desc &m) {
    if (m.closure_count == 0u || !m.closures || m.root >= m.closure_count)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "material without a valid closure root");
    if (m.value_count > psy::kMaxValues)
        return fail(PSY_ERROR_UNSUPPORTED, "value stream longer than " + std::to_string(psy::kMaxValues) +
                                               " instructions");
    if (m.value_count != 0u && !m.values) return fail(PSY_ERROR_INVALID_ARGUMENT, "value stream without instructions");
    constexpr uint32_t S = PSY_VALUE_TYPE_SCALAR, V = PSY_VALUE_TYPE_VECTOR, X = 0xffffffffu;
    for (uint32_t k = 0; k < m.value_count; ++k) {
        const psy_value_instruction &in = m.values[k];
        // result type and operand types (X: operand unused) per operation
        uint32_t result = S, ta = X, tb = X, tc = X;
        switch (in.op) {
        case PSY_VALUE_PARAMETER: result = in.type; break;
        case PSY_VALUE_PASSTHROUGH: result = in.type; ta = in.type; break;
        case PSY_VALUE_SCALAR_TO_COLOR: result = V; ta = S; break;
        case PSY_VALUE_SCALAR_TO_BOOLEAN: ta = S; break;
        case PSY_VALUE_COLOR_TO_SCALAR:
        case PSY_VALUE_VECTOR_TO_SCALAR: ta = V; break;
        case PSY_VALUE_ADD: case PSY_VALUE_SUBTRACT: case PSY_VALUE_MULTIPLY: case PSY_VALUE_DIVIDE:
        case PSY_VALUE_MINIMUM: case PSY_VALUE_MAXIMUM: case PSY_VALUE_POWER: ta = tb = S; break;
        case PSY_VALUE_ABSOLUTE: case PSY_VALUE_CLAMP01: ta = S; break;
        case PSY_VALUE_CLAMP_RANGE: case PSY_VALUE_MIX_FLOAT: ta = tb = tc = S; break;
        case PSY_VALUE_MIX_VECTOR: result = V; ta = tb = V; tc = in.static_u0 != 0u ? V : S; break;
        case PSY_VALUE_MIX:
            if (in.static_u0 != PSY_BLEND_MIX && in.static_u0 != PSY_BLEND_DARKEN && in.static_u0 != PSY_BLEND_MULTIPLY &&
                in.static_u0 != PSY_BLEND_LIGHTEN && in.static_u0 != PSY_BLEND_SCREEN && in.static_u0 != PSY_BLEND_ADD &&
                in.static_u0 != PSY_BLEND_DIFFERENCE && in.static_u0 != PSY_BLEND_SUBTRACT)
                return fail(PSY_ERROR_UNSUPPORTED, "colour blend mode outside the supported set");
            result = V; ta = tb = V; tc = S;
            break;
        case PSY_VALUE_MULTIPLY_COLOR: result = V; ta = tb = V; tc = S; break;
        case PSY_VALUE_INVERT: result = V; ta = V; tb = S; break;
        case PSY_VALUE_SEPARATE_R: case PSY_VALUE_SEPARATE_G: case PSY_VALUE_SEPARATE_B:
            if (in.static_u0 != 0u) return fail(PSY_ERROR_UNSUPPORTED, "separate colour outside RGB mode");
            ta = V;
            break;
        case PSY_VALUE_COMBINE_COLOR:
            if (in.static_u0 != 0u) return fail(PSY_ERROR_UNSUPPORTED, "combine colour outside RGB mode");
            result = V; ta = tb = tc = S;
            break;
        default:
            return fail(PSY_ERROR_UNSUPPORTED, "value operation " + std::to_string(in.op) + " outside the supported set");
        }
        if (in.type != result) return fail(PSY_ERROR_INVALID_ARGUMENT, "value instruction of the wrong result type");
        if (in.op == PSY_VALUE_PARAMETER && in.parameter >= (in.type == S ? m.scalar_count : m.vector_count))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "value parameter slot out of range");
        const uint32_t ops[3] = {in.a, in.b, in.c}, types[3] = {ta, tb, tc};
        for (int o = 0; o < 3; ++o) {
            if (types[o] == X) continue;
            if (ops[o] >= k) return fail(PSY_ERROR_INVALID_ARGUMENT, "value operand is not an earlier instruction");
            if (m.values[ops[o]].type != types[o])
                return fail(PSY_ERROR_INVALID_ARGUMENT, "value operand of the wrong type");
        }
    }
    // a closure input of type `type`; `optional` admits PSY_INPUT_NONE
    auto input_ok = [&](uint32_t ref, uint32_t type, bool optional) {
        if (ref == PSY_INPUT_NONE) return optional;
        if (ref & PSY_INPUT_VALUE) {
            const uint32_t id = ref & ~PSY_INPUT_VALUE;
            return id < m.value_count && m.values[id].type == type;
        }
        return ref < (type == S ? m.scalar_count : m.vector_count);
    };
    for (uint32_t k = 0; k < m.closure_count; ++k) {
        const psy_closure_instruction &c = m.closures[k];
        if (c.op > PSY_CLOSURE_REFRACTION)
            return fail(PSY_ERROR_UNSUPPORTED, "closure operation outside the supported set");
        const bool microfacet = c.op == PSY_CLOSURE_GLOSSY || c.op == PSY_CLOSURE_GLASS || c.op == PSY_CLOSURE_REFRACTION;
        if ((c.op == PSY_CLOSURE_ADD || c.op == PSY_CLOSURE_MIX) && (c.a >= m.closure_count || c.b >= m.closure_count))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "closure child out of range");
        if ((c.op == PSY_CLOSURE_DIFFUSE || c.op == PSY_CLOSURE_EMISSION || c.op == PSY_CLOSURE_TRANSPARENT ||
             microfacet) &&
            !input_ok(c.color, V, false))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "closure colour input out of range");
        if ((c.op == PSY_CLOSURE_EMISSION || c.op == PSY_CLOSURE_MIX || c.op == PSY_CLOSURE_GLASS ||
             c.op == PSY_CLOSURE_REFRACTION) &&
            !input_ok(c.scalar, S, false))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "closure scalar input out of range");
        if ((c.op == PSY_CLOSURE_DIFFUSE || microfacet) && !input_ok(c.roughness, S, true))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "closure roughness input out of range");
        if (microfacet && c.a != PSY_GLOSSY_GGX && c.a != PSY_GLOSSY_BECKMANN &&
            !(c.op == PSY_CLOSURE_GLOSSY && c.a == PSY_GLOSSY_MULTI_GGX))
            return fail(PSY_ERROR_UNSUPPORTED, "microfacet distribution outside GGX, Beckmann and (glossy) MULTI_GGX");
    }
    // The device walks the tree with a 32-entry stack and keeps at most 16
    // BSDF closures per shading point (the reference's capacity is Cycles'
    // MAX_CLOSURE, 64): a material that would overflow either is refused
    // rather than rendered with closures dropped.  The walk is replayed here.
    uint32_t stack[32];
    uint32_t sp = 0u, leaves = 0u, visits = 0u;
    bool transparent = false, glass = false;
    stack[sp++] = m.root;
    while (sp > 0u) {
        const uint32_t id = stack[--sp];
        if (++visits > 4096u) return fail(PSY_ERROR_UNSUPPORTED, "closure tree too large");
        const psy_closure_instruction &c = m.closures[id];
        if (c.op == PSY_CLOSURE_ADD || c.op == PSY_CLOSURE_MIX) {
            if (sp + 2u > 32u) return fail(PSY_ERROR_UNSUPPORTED, "closure tree deeper than the device walk's stack");
            stack[sp++] = c.b;
            stack[sp++] = c.a;
        } else if (c.op == PSY_CLOSURE_DIFFUSE || c.op == PSY_CLOSURE_GLOSSY || c.op == PSY_CLOSURE_GLASS ||
                   c.op == PSY_CLOSURE_REFRACTION) {
            ++leaves;
            glass = glass || c.op == PSY_CLOSURE_GLASS;
        } else if (c.op == PSY_CLOSURE_TRANSPARENT) {
            transparent = true;  // every transparent closure merges into one
        }
    }
    if (leaves + (transparent ? 1u : 0u) > 16u)
        return fail(PSY_ERROR_UNSUPPORTED, "more than 16 BSDF closures in one material");
    // a glass closure's selection weight among other closures is Cycles'
    // tabulated Fresnel albedo, which this build does not carry
    if (glass && leaves + (transparent ? 1u : 0u) > 1u)
        return fail(PSY_ERROR_UNSUPPORTED, "a glass closure must be the only BSDF closure of its material");
    return PSY_OK;
}

// Emission estimate of a closure program for the light tree
// (estimate_surface_emission, src/compiler/surface_program.cpp:244-330): one
// estimate per instruction in program order -- emission colour x strength,
// add a + b, mix a (1 - f) + b f with the unclamped factor -- where an
// operand that is not an earlier instruction counts as one.  Only an
// unlinked socket of the closure node itself is read as a literal
// (direct_parameter_value, surface_program.cpp:170-186); a linked colour or
// strength counts as one, and a mix with a linked factor sums its branches.
void emission_estimate(const psy_material_desc &m, float out[3]) {
    std::vector<std::array<float, 3>> est;
    est.reserve(m.closure_count);
    auto dep = [&](uint32_t id) { return id < est.size() ? est[id] : std::array<float, 3>{1.0f, 1.0f, 1.0f}; };
    auto literal = [](uint32_t ref) { return (ref & PSY_INPUT_VALUE) == 0u; };
    for (uint32_t i = 0; i < m.closure_count; ++i) {
        const psy_closure_instruction &c = m.closures[i];
        std::array<float, 3> e{0.0f, 0.0f, 0.0f};
        if (c.op == PSY_CLOSURE_EMISSION) {
            const float strength = literal(c.scalar) ? m.scalars[c.scalar] : 1.0f;
            for (int k = 0; k < 3; ++k) e[k] = (literal(c.color) ? m.vectors[3u * c.color + k] : 1.0f) * strength;
        } else if (c.op == PSY_CLOSURE_ADD) {
            const auto a = dep(c.a), b = dep(c.b);
            for (int k = 0; k < 3; ++k) e[k] = a[k] + b[k];
        } else if (c.op == PSY_CLOSURE_MIX) {
            const auto a = dep(c.a), b = dep(c.b);
            if (literal(c.scalar)) {
                const float f = m.scalars[c.scalar];
                for (int k = 0; k < 3; ++k) e[k] = a[k] * (1.0f - f) + b[k] * f;
            } else {
                for (int k = 0; k < 3; ++k) e[k] = a[k] + b[k];
            }
        }
        est.push_back(e);
    }
    for (int k = 0; k < 3; ++k) out[k] = m.root < est.size() ? est[m.root][k] : 0.0f;
}

// The per-lamp constants of the sampling kernels, in the kernels' float
// expressions and operation order (the library is compiled without FP
// contraction); transcendentals are evaluated in double and rounded once,
// as the kernels' own are (analytic_light_sampling.h:84-108, 309-376,
// 880-896).
psy::LampConstGpu lamp_constants(const psy_light_desc &l) {
    constexpr float kPiF = 3.1415926535897932f, kInvPiF = 0.31830988618379067154f;
    auto rounded = [](double v) { return static_cast<float>(v); };
    auto maxf = [](float a, float b) { return a > b ? a : b; };
    psy::LampConstGpu c{};
    float ax[3], ay[3], az[3];
    for (int k = 0; k < 3; ++k) {
        ax[k] = l.axis_x[k] * l.axis_scale[0];
        ay[k] = l.axis_y[k] * l.axis_scale[1];
        az[k] = l.axis_z[k] * l.axis_scale[2];
    }
    auto cross = [](const float a[3], const float b[3], float o[3]) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    float adj_x[3], adj_y[3], adj_z[3];
    cross(ay, az, adj_x);
    cross(az, ax, adj_y);
    cross(ax, ay, adj_z);
    const float det = ax[0] * adj_x[0] + ax[1] * adj_x[1] + ax[2] * adj_x[2];
    const float inv_det = 1.0f / (std::fabs(det) > 1.0e-20f ? det : 1.0f);
    const float cos_half = rounded(std::cos(static_cast<double>(0.5f * l.spot_angle)));
    const float blend = (1.0f - cos_half) * l.spot_smooth;
    const float t = rounded(std::tan(static_cast<double>(0.5f * l.spot_angle)));
    const float ts2 = maxf(l.axis_scale[0] * l.axis_scale[0], l.axis_scale[1] * l.axis_scale[1]);
    const float as2 = l.axis_scale[2] * l.axis_scale[2];
    const float spread_cap = 1.0f - 1.0f / std::sqrt(1.0f + t * t * ts2 / maxf(as2, 1.0e-30f));
    c.spot_rx = make_float4(adj_x[0] * inv_det, adj_x[1] * inv_det, adj_x[2] * inv_det, cos_half);
    c.spot_ry = make_float4(adj_y[0] * inv_det, adj_y[1] * inv_det, adj_y[2] * inv_det, blend);
    c.spot_rz = make_float4(adj_z[0] * inv_det, adj_z[1] * inv_det, adj_z[2] * inv_det, spread_cap);
    const bool normalize_power = (l.flags & PSY_LIGHT_FLAG_NORMALIZE) != 0u;
    const float r2 = l.radius * l.radius;
    const float area = r2 > 0.0f ? 4.0f * kPiF * r2 : 4.0f;
    c.factors.x = (normalize_power ? 1.0f / maxf(area, 1.0e-20f) : 1.0f) * kInvPiF;
    const float half_angle = 0.5f * maxf(l.angle, 0.0f);
    const float sq = rounded(std::sin(static_cast<double>(0.5f * half_angle)));
    c.factors.y = 2.0f * sq * sq;
    const float sh = rounded(std::sin(static_cast<double>(half_angle)));
    const float disk_area = kPiF * sh * sh;
    c.factors.z = (normalize_power && half_angle > 0.0f) ? 1.0f / maxf(disk_area, 1.0e-20f) : 1.0f;
    return c;
}

// Argument checks of a parameter-only edit: the material exists and the
// new block has the compiled block's layout.
psy_status check_rebind(const psy_scene *s, uint32_t material, const float *scalars, uint32_t scalar_count,
                        const float *vectors, uint32_t vector_count) {
    if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "null scene");
    if (material >= s->materials.size()) return fail(PSY_ERROR_INVALID_ARGUMENT, "material out of range");
    const psy::MaterialGpu &m = s->materials[material];
    const uint32_t next_scalar =
        material + 1 < s->materials.size() ? s->materials[material + 1].scalar_offset : uint32_t(s->scalars.size());
    const uint32_t next_vector = material + 1 < s->materials.size() ? s->materials[material + 1].vector_offset
                                                                    : uint32_t(s->vectors.size() / 3u);
    if (scalar_count != next_scalar - m.scalar_offset || vector_count != next_vector - m.vector_offset)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "parameter block layout differs from the compiled program");
    if ((scalar_count && !scalars) || (vector_count && !vectors)) return fail(PSY_ERROR_INVALID_ARGUMENT, "null parameters");
    return PSY_OK;
}

// Runs body(i) for every i in [0, n) on up to 32 host threads that pull
// indices from a shared counter; `threads` receives the count used.  An
// exception in a body (out of host memory) becomes PSY_ERROR_OUT_OF_MEMORY.
template <typename F>
psy_status parallel_for(uint32_t n, uint32_t *threads, F &&body) {
    const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint32_t count = std::max(1u, std::min({hw, n, 32u}));
    std::atomic<uint32_t> next{0u};
    std::atomic<bool> failed{false};
    auto worker = [&]() {
        for (uint32_t i; !failed.load() && (i = next.fetch_add(1u)) < n;) {
            try {
                body(i);
            } catch (...) {
                failed.store(true);
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < count; ++t) pool.emplace_back(worker);
    worker();
    for (std::thread &t : pool) t.join();
    if (threads) *threads = count;
    return failed.load() ? fail(PSY_ERROR_OUT_OF_MEMORY, "host memory exhausted while building the scene") : PSY_OK;
}

// Uploads `v` into a new device buffer that takes the place of `slot`; the
// buffer it replaces joins the scene's retired list.
// The new buffer is stream-ordered on the context's stream, and the host
// copy it is uploaded from stays alive with the retired list, so the caller
// need not wait for the upload.
template <typename T>
cudaError_t replace_buffer(psy_scene *sc, DeviceBuffer &slot, const std::vector<T> &v) {
    auto source = std::make_shared<const std::vector<T>>(v);
    auto fresh = std::make_unique<DeviceBuffer>(sc->context->stream);
    const cudaError_t e = fresh->upload(*source, sc->context->stream);
    if (e != cudaSuccess) return e;
    slot.swap(*fresh);
    if (fresh->ptr) sc->retired.push_back(std::move(fresh));
    sc->retired_host.push_back(std::move(source));
    return cudaSuccess;
}

// The many-light tree over the scene's emitter population -- emissive
// triangles in emitter order, then the analytic lights -- built from the
// host copies and uploaded (src/luisa/path_tracer_light_sampling_scene.cpp:
// 160-240).  A tree whose root carries no energy is left empty, and
// sessions then select lights from the flat distribution.
psy_status build_light_tree(psy_scene *sc, bool sync = true) {
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<psy::LtNodeGpu> lt_nodes;
    std::vector<psy::LtEmitterGpu> lt_emitters;
    std::vector<uint2> lt_mapping;
    std::vector<uint4> lt_lookup;
    uint32_t lt_root = 0u;
    const std::vector<psy::EmitterGpu> &emitters = sc->emitters_host;
    const uint32_t tri_n = uint32_t(emitters.size()), light_n = uint32_t(sc->lights_host.size());
    // estimate_surface_emission per material (a property of the program and
    // its parameter block)
    std::vector<std::array<float, 3>> estimates(sc->materials.size());
    for (size_t i = 0; i < sc->materials.size(); ++i) {
        const psy::MaterialGpu &g = sc->materials[i];
        psy_material_desc m{};
        m.closures = sc->code_host.data() + g.code_offset;
        m.closure_count = g.code_count;
        m.root = g.root;
        m.scalars = sc->scalars.data() + g.scalar_offset;
        m.vectors = sc->vectors.data() + 3ull * g.vector_offset;
        m.values = sc->values_host.data() + g.value_offset;
        m.value_count = g.value_count;
        if (g.has_emission) emission_estimate(m, estimates[i].data());
        else estimates[i] = {0.0f, 0.0f, 0.0f};
    }
    std::vector<psy::LtEmitter> source;
    source.reserve(tri_n + light_n);
    for (uint32_t i = 0; i < tri_n; ++i) {
        const psy::EmitterGpu &e = emitters[i];
        source.push_back(psy::lt_triangle_emitter(i, e.p0, e.p1, e.p2, estimates[e.material].data(), e.emission_sampling,
                                                  sc->instance_mirrored[e.object] != 0u));
    }
    for (uint32_t i = 0; i < light_n; ++i) source.push_back(psy::lt_analytic_emitter(tri_n + i, &sc->lights_host[i]));
    if (!source.empty()) {
        const psy::LightTree tree = psy::lt_build(source, 8u);
        const bool usable = tree.root < tree.nodes.size() && tree.emitter_to_tree.size() == tree.emitters.size() &&
                            tree.nodes[tree.root].measure.energy > 0.0f;
        if (usable) {
            auto flags = [](const psy::LtMeasure &m, bool distant) {
                return (!m.bounds.empty ? psy::kLtFlagBounds : 0u) | (!m.orientation.empty ? psy::kLtFlagOrientation : 0u) |
                       (distant ? psy::kLtFlagDistant : 0u);
            };
            auto pack = [](const psy::LtMeasure &m, float4 &a, float4 &b, float4 &c) {
                a = make_float4(m.bounds.lo[0], m.bounds.lo[1], m.bounds.lo[2], m.energy);
                b = make_float4(m.bounds.hi[0], m.bounds.hi[1], m.bounds.hi[2], m.orientation.theta_o);
                c = make_float4(m.orientation.axis[0], m.orientation.axis[1], m.orientation.axis[2], m.orientation.theta_e);
            };
            // the cone's trigonometry, double-rounded as the kernels' own
            auto cone = [](const psy::LtMeasure &m) {
                const float to = m.orientation.theta_o, te = m.orientation.theta_e;
                auto rc = [](float v) { return static_cast<float>(std::cos(static_cast<double>(v))); };
                return make_float4(rc(to), static_cast<float>(std::sin(static_cast<double>(to))), rc(to + te),
                                   rc(te - to));
            };
            lt_nodes.reserve(tree.nodes.size());
            for (const psy::LtNode &n : tree.nodes) {
                psy::LtNodeGpu g{};
                pack(n.measure, g.min_energy, g.max_theta_o, g.axis_theta_e);
                g.cone = cone(n.measure);
                g.topology = make_uint4(n.parent, n.left, n.right, n.kind);
                g.emitters = make_uint4(n.first, n.count, flags(n.measure, n.kind == psy::kLtDistant), 0u);
                lt_nodes.push_back(g);
            }
            lt_emitters.reserve(tree.emitters.size());
            for (const psy::LtEmitter &e : tree.emitters) {
                psy::LtEmitterGpu g{};
                pack(e.measure, g.min_energy, g.max_theta_o, g.axis_theta_e);
                g.cone = cone(e.measure);
                g.identity = make_uint4(e.emitter_id, flags(e.measure, e.distant), 0u, 0u);
                lt_emitters.push_back(g);
            }
            for (size_t id = 0; id < tree.emitters.size(); ++id)
                lt_mapping.push_back(make_uint2(tree.emitter_to_tree[id], tree.emitter_to_leaf[id]));
            for (uint32_t i = 0; i < tri_n; ++i)
                lt_lookup.push_back(make_uint4(emitters[i].object, emitters[i].cycles_prim, i, 0u));
            std::sort(lt_lookup.begin(), lt_lookup.end(), [](const uint4 &a, const uint4 &b) {
                return a.x < b.x || (a.x == b.x && (a.y < b.y || (a.y == b.y && a.z < b.z)));
            });
            lt_root = tree.root;
        }
    }
    cudaStream_t st = sc->context->stream;
    PSY_CUDA_TRY(cudaSetDevice(sc->context->device));
    // new buffers; a tree built before is retired, not freed, as queued
    // work may still read it
    PSY_CUDA_TRY(replace_buffer(sc, sc->lt_nodes, lt_nodes));
    PSY_CUDA_TRY(replace_buffer(sc, sc->lt_emitters, lt_emitters));
    PSY_CUDA_TRY(replace_buffer(sc, sc->lt_mapping, lt_mapping));
    PSY_CUDA_TRY(replace_buffer(sc, sc->lt_lookup, lt_lookup));
    if (sync) PSY_CUDA_TRY(cudaStreamSynchronize(st));
    psy::SceneView &v = sc->view;
    v.lt_nodes = sc->lt_nodes.as<psy::LtNodeGpu>();
    v.lt_emitters = sc->lt_emitters.as<psy::LtEmitterGpu>();
    v.lt_mapping = sc->lt_mapping.as<uint2>();
    v.lt_lookup = sc->lt_lookup.as<uint4>();
    v.lt_node_count = uint32_t(lt_nodes.size());
    v.lt_emitter_count = uint32_t(lt_emitters.size());
    v.lt_lookup_count = uint32_t(lt_lookup.size());
    v.lt_root = lt_root;
    sc->light_tree_built = true;
    sc->stats.light_tree_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    sc->stats.light_tree_builds++;
    return PSY_OK;
}

}  // namespace

psy_status psy::host::rebind_parameters_versioned(psy_scene *s, uint32_t material, const float *scalars,
                                                  uint32_t scalar_count, const float *vectors, uint32_t vector_count) {
    const psy_status valid = check_rebind(s, material, scalars, scalar_count, vectors, vector_count);
    if (valid != PSY_OK) return valid;
    const psy::MaterialGpu &m = s->materials[material];
    PSY_CUDA_TRY(cudaSetDevice(s->context->device));
    if (scalar_count) std::memcpy(s->scalars.data() + m.scalar_offset, scalars, sizeof(float) * scalar_count);
    if (vector_count) std::memcpy(s->vectors.data() + 3ull * m.vector_offset, vectors, sizeof(float) * 3u * vector_count);
    PSY_CUDA_TRY(replace_buffer(s, s->scalar_buf, s->scalars));
    PSY_CUDA_TRY(replace_buffer(s, s->vector_buf, s->vectors));
    s->view.scalars = s->scalar_buf.as<float>();
    s->view.vectors = s->vector_buf.as<float>();
    if (m.has_emission) {
        std::lock_guard<std::mutex> lock(s->light_tree_mutex);
        if (s->light_tree_built) {
            const psy_status r = build_light_tree(s, false);
            if (r != PSY_OK) return r;
        }
    }
    if (!s->uploads_done) PSY_CUDA_TRY(cudaEventCreateWithFlags(&s->uploads_done, cudaEventDisableTiming));
    PSY_CUDA_TRY(cudaEventRecord(s->uploads_done, s->context->stream));
    return PSY_OK;
}

void psy::host::release_retired(psy_scene *s) {
    if (!s || (s->retired.empty() && s->retired_host.empty())) return;
    cudaSetDevice(s->context->device);
    s->retired.clear();  // stream-ordered frees: after all work queued so far
    // host sources go once their uploads have run
    if (!s->uploads_done || cudaEventQuery(s->uploads_done) == cudaSuccess) s->retired_host.clear();
}

psy_status psy::host::ensure_light_tree(psy_scene *sc) {
    std::lock_guard<std::mutex> lock(sc->light_tree_mutex);
    return sc->light_tree_built ? PSY_OK : build_light_tree(sc);
}

// ================================================================== C ABI

extern "C" {

const char *psy_last_error(void) { return g_last_error.c_str(); }
uint32_t psy_abi_version(void) { return PSY_ABI_VERSION; }

void psy_render_settings_default(psy_render_settings *r) {
    if (!r) return;
    std::memset(r, 0, sizeof(*r));
    r->filter_width = 1.0f;
    r->pass_alpha_threshold = 0.5f;
    r->max_bounces = 12u;
    r->diffuse_bounces = 4u;
    r->glossy_bounces = 4u;
    r->transmission_bounces = 12u;
    r->transparent_max_bounces = 8u;
    r->film_exposure = 1.0f;
    r->light_sampling_threshold = 0.01f;
    r->direct_light_sampling = PSY_DIRECT_LIGHT_MIS;
    r->next_event_estimation = 1u;
}

uint32_t psy_sobol_sequence_size_for_samples(uint32_t samples) {
    const uint32_t c = std::clamp(samples, 1u, 8192u);
    uint32_t u = 1u;
    if (c != 1u) u = 1u << (32u - static_cast<uint32_t>(__builtin_clz(c - 1u)));
    return std::clamp(u, 256u, 8192u);
}

psy_status psy_sobol_generate_table(uint32_t size, float *out) {
    if (!out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null output");
    if (!sobol_size_valid(size))
        return fail(PSY_ERROR_INVALID_ARGUMENT, "tabulated Sobol sequence size must be a power of two between 256 and 8192");
    for (uint32_t pattern = 0; pattern < 256u; ++pattern) sobol_pattern(out + size_t(pattern) * size * 4u, size, pattern);
    return PSY_OK;
}

psy_status psy_pixel_filter_table(uint32_t filter, float width, float *out) {
    if (!out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null output");
    if (filter > PSY_FILTER_BLACKMAN_HARRIS) return fail(PSY_ERROR_INVALID_ARGUMENT, "unknown pixel filter");
    const auto t = filter_table(filter, width);
    std::memcpy(out, t.data(), sizeof(float) * t.size());
    return PSY_OK;
}

psy_status psy_context_create(int device, psy_context **out) {
    if (!out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    int count = 0;
    PSY_CUDA_TRY(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(PSY_ERROR_INVALID_ARGUMENT, "no such CUDA device");
    PSY_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop{};
    PSY_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(PSY_ERROR_UNSUPPORTED, "libpsycles_cuda is built for sm_100a (B200)");
    // stream-ordered buffers (render-server sessions, edited parameter
    // blocks) come from the device's default pool; freed memory stays in the
    // pool for the next job instead of going back to the driver
    cudaMemPool_t pool = nullptr;
    PSY_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    PSY_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    auto c = std::make_unique<psy_context>();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    c->launch.sms = c->sms;
    PSY_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    PSY_CUDA_TRY(cudaStreamCreateWithFlags(&c->readback, cudaStreamNonBlocking));
    *out = c.release();
    return PSY_OK;
}

psy_status psy_context_set_tuning(psy_context *c, const psy_tuning *t) {
    if (!c || !t) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    if (t->stream_blocks_per_sm > 64u || t->traversal_blocks_per_sm > 64u || t->shade_blocks_per_sm > 64u)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "at most 64 blocks per SM");
    if (t->path_capacity > (1u << 26)) return fail(PSY_ERROR_INVALID_ARGUMENT, "path capacity above 64 Mi");
    if (t->stream_block_size && t->stream_block_size != 128u && t->stream_block_size != 256u &&
        t->stream_block_size != 512u)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "stream block size must be 128, 256 or 512");
    const psy::LaunchConfig defaults;
    c->path_capacity = t->path_capacity ? t->path_capacity : (1u << 24);
    c->launch.stream_blocks_per_sm = t->stream_blocks_per_sm ? t->stream_blocks_per_sm : defaults.stream_blocks_per_sm;
    c->launch.traversal_blocks_per_sm =
        t->traversal_blocks_per_sm ? t->traversal_blocks_per_sm : defaults.traversal_blocks_per_sm;
    c->launch.shade_blocks_per_sm = t->shade_blocks_per_sm ? t->shade_blocks_per_sm : defaults.shade_blocks_per_sm;
    c->launch.sort_threshold = t->sort_threshold == 0xffffffffu ? defaults.sort_threshold : t->sort_threshold;
    c->launch.shadow_sort_threshold =
        t->shadow_sort_threshold == 0xffffffffu ? defaults.shadow_sort_threshold : t->shadow_sort_threshold;
    c->launch.ray_sort_threshold =
        t->ray_sort_threshold == 0xffffffffu ? defaults.ray_sort_threshold : t->ray_sort_threshold;
    c->launch.stream_block = t->stream_block_size ? t->stream_block_size : defaults.stream_block;
    return PSY_OK;
}

psy_status psy_context_get_tuning(const psy_context *c, psy_tuning *t) {
    if (!c || !t) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    t->path_capacity = c->path_capacity;
    t->stream_blocks_per_sm = c->launch.stream_blocks_per_sm;
    t->traversal_blocks_per_sm = c->launch.traversal_blocks_per_sm;
    t->shade_blocks_per_sm = c->launch.shade_blocks_per_sm;
    t->sort_threshold = c->launch.sort_threshold;
    t->shadow_sort_threshold = c->launch.shadow_sort_threshold;
    t->ray_sort_threshold = c->launch.ray_sort_threshold;
    t->stream_block_size = c->launch.stream_block;
    return PSY_OK;
}

void psy_context_destroy(psy_context *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    if (c->readback) cudaStreamDestroy(c->readback);
    if (c->readback_host) cudaFreeHost(c->readback_host);
    delete c;
}

psy_status psy_scene_compile(psy_context *ctx, const psy_scene_desc *d, psy_scene **out) {
    if (!ctx || !d || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    const auto t_begin = std::chrono::steady_clock::now();
    PSY_CUDA_TRY(cudaSetDevice(ctx->device));
    // ---- validation (SceneDatabase commits only valid snapshots)
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        if (d->instances[i].mesh >= d->mesh_count) return fail(PSY_ERROR_INVALID_ARGUMENT, "instance mesh out of range");
        if (d->instances[i].material >= d->material_count)
            return fail(PSY_ERROR_INVALID_ARGUMENT, "instance material out of range");
    }
    for (uint32_t i = 0; i < d->mesh_count; ++i) {
        const psy_mesh_desc &m = d->meshes[i];
        if (m.triangle_count && (!m.indices || !m.positions))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "mesh without indices or positions");
        for (uint64_t k = 0; k < 3ull * m.triangle_count; ++k)
            if (m.indices[k] >= m.vertex_count) return fail(PSY_ERROR_INVALID_ARGUMENT, "mesh index out of range");
        if (m.materials)
            for (uint32_t k = 0; k < m.triangle_count; ++k)
                if (m.materials[k] >= d->material_count)
                    return fail(PSY_ERROR_INVALID_ARGUMENT, "triangle material out of range");
        if (m.smooth && !m.normals) return fail(PSY_ERROR_INVALID_ARGUMENT, "smooth mesh without normals");
    }
    for (uint32_t i = 0; i < d->material_count; ++i) {
        const psy_status valid = validate_material(d->materials[i]);
        if (valid != PSY_OK) return valid;
    }
    for (uint32_t i = 0; i < d->light_count; ++i) {
        const psy_light_desc &l = d->lights[i];
        if (l.type == PSY_LIGHT_AREA && !(l.spread >= 3.14159165f))
            return fail(PSY_ERROR_UNSUPPORTED, "area lights with a spread below pi are not available in this build");
        if (l.type == PSY_LIGHT_AREA && !(l.size_u > 0.0f && l.size_v > 0.0f))
            return fail(PSY_ERROR_INVALID_ARGUMENT, "area light with an empty size");
        if (l.type > PSY_LIGHT_DISTANT) return fail(PSY_ERROR_INVALID_ARGUMENT, "unknown light type");
        if ((l.flags >> 16) != 0u) return fail(PSY_ERROR_INVALID_ARGUMENT, "reserved light flag bits are set");
    }
    auto sc = std::make_unique<psy_scene>();
    sc->context = ctx;
    sc->revision = d->revision;
    sc->camera = d->camera;
    cudaStream_t st = ctx->stream;
    auto t_phase = std::chrono::steady_clock::now();
    auto lap = [&t_phase]() {
        const auto now = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(now - t_phase).count();
        t_phase = now;
        return ms;
    };
    sc->stats.validate_ms = lap();

    // ---- meshes: flatten, then one BLAS per mesh (meshes build in parallel;
    // each build is sequential and deterministic, so the result does not
    // depend on the thread count)
    std::vector<psy::MeshGpu> meshes(d->mesh_count);
    std::vector<float> positions, normals;
    std::vector<uint32_t> indices, tri_materials;
    std::vector<psy::WideNodeGpu> blas;
    std::vector<float4> tris;
    std::vector<Box> mesh_boxes(d->mesh_count);
    std::vector<std::vector<psy::WideNodeGpu>> mesh_wide(d->mesh_count);
    std::vector<std::vector<psy::CwNodeGpu>> mesh_cw(d->mesh_count);
    std::vector<psy::CwNodeGpu> blas8;
    // triangle records in BVH leaf order, written by each mesh's build at
    // the mesh's offset (meshes in input order)
    std::vector<uint64_t> mesh_tri_first(d->mesh_count + 1u, 0u);
    for (uint32_t i = 0; i < d->mesh_count; ++i) mesh_tri_first[i + 1u] = mesh_tri_first[i] + d->meshes[i].triangle_count;
    tris.resize(3u * mesh_tri_first[d->mesh_count]);
    // one mesh's BLAS, its triangle records in leaf order and its stack need
    std::vector<uint32_t> mesh_need(d->mesh_count, 0u);
    auto build_mesh = [&](uint32_t i, int sah_depth_limit) {
        const psy_mesh_desc &m = d->meshes[i];
        Builder bld;
        bld.sah_depth_limit = sah_depth_limit;
        bld.prims.resize(m.triangle_count);
        for (uint32_t k = 0; k < m.triangle_count; ++k) {
            Prim &p = bld.prims[k];
            for (int c = 0; c < 3; ++c) {
                const float *v = m.positions + 3ull * m.indices[3ull * k + c];
                p.box.grow(v[0], v[1], v[2]);
            }
            for (int a = 0; a < 3; ++a) p.c[a] = 0.5 * (p.box.lo[a] + p.box.hi[a]);
            p.id = k;
        }
        mesh_boxes[i] = bld.build_root();
        float4 *out = tris.data() + 3u * mesh_tri_first[i];
        auto put = [&](uint32_t id) {
            for (int c = 0; c < 3; ++c) {
                const float *v = m.positions + 3ull * m.indices[3ull * id + c];
                float w = 0.0f;
                if (c == 0) std::memcpy(&w, &id, 4);
                *out++ = make_float4(v[0], v[1], v[2], w);
            }
        };
#if PSY_BVH_WIDTH == 8
        // triangle records in the slot order of the 8-wide leaves
        std::vector<uint32_t> leaves;
        mesh_cw[i] = bld.widen8(leaves);
        mesh_need[i] = blas_stack_need8(mesh_cw[i]);
        for (const uint32_t leaf : leaves) put(bld.prims[leaf].id);
#else
        mesh_wide[i] = bld.widen();
        mesh_need[i] = blas_stack_need(mesh_wide[i]);
        for (const Prim &p : bld.prims) put(p.id);
#endif
    };
    {
        std::vector<uint32_t> by_size(d->mesh_count);
        for (uint32_t i = 0; i < d->mesh_count; ++i) by_size[i] = i;
        std::stable_sort(by_size.begin(), by_size.end(), [d](uint32_t a, uint32_t b) {
            return d->meshes[a].triangle_count > d->meshes[b].triangle_count;
        });
        const psy_status built = parallel_for(d->mesh_count, &sc->stats.build_threads,
                                              [&](uint32_t job) { build_mesh(by_size[job], Builder{}.sah_depth_limit); });
        if (built != PSY_OK) return built;
    }
    sc->stats.blas_ms = lap();

    // ---- instances + TLAS
    std::vector<psy::InstanceGpu> instances(d->instance_count);
    Builder tl;
    tl.leaf_size = 1u;
    tl.leaf_is_id = true;
    std::vector<M34> o2w(d->instance_count);
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const psy_instance_desc &id = d->instances[i];
        psy::InstanceGpu &g = instances[i];
        o2w[i] = m34(id.object_to_world);
        const M34 w2o = inverse34(o2w[i]);
        M34 nrm;
        nrm.c0 = {w2o.c0.x, w2o.c1.x, w2o.c2.x};
        nrm.c1 = {w2o.c0.y, w2o.c1.y, w2o.c2.y};
        nrm.c2 = {w2o.c0.z, w2o.c1.z, w2o.c2.z};
        nrm.c3 = {0.0f, 0.0f, 0.0f};
        store34(g.o2w, o2w[i]);
        store34(g.w2o, w2o);
        store34(g.nrm, nrm);
        g.mesh = id.mesh;
        g.material = id.material;
        g.visibility = id.visibility;
    }
    // Instance boxes: the world-space bounds of the instance's transformed
    // vertices (the mesh box's transformed corners would be up to about 1.7
    // times wider per axis under rotation), computed in double per instance
    // in parallel, then widened for the float transform of the ray by ten
    // times the mesh boxes' relative padding.
    {
        std::vector<Box> instance_boxes(d->instance_count);
        uint32_t box_threads = 0u;
        const psy_status boxed = parallel_for(d->instance_count, &box_threads, [&](uint32_t i) {
            const psy_mesh_desc &m = d->meshes[d->instances[i].mesh];
            if (mesh_boxes[d->instances[i].mesh].empty()) return;
            const M34 &t = o2w[i];
            Box &b = instance_boxes[i];
            for (uint64_t v = 0; v < m.vertex_count; ++v) {
                const double x = m.positions[3 * v], y = m.positions[3 * v + 1], z = m.positions[3 * v + 2];
                b.grow(x * t.c0.x + y * t.c1.x + z * t.c2.x + t.c3.x, x * t.c0.y + y * t.c1.y + z * t.c2.y + t.c3.y,
                       x * t.c0.z + y * t.c1.z + z * t.c2.z + t.c3.z);
            }
        });
        if (boxed != PSY_OK) return boxed;
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            if (instance_boxes[i].empty()) continue;
            Prim p;
            p.box = instance_boxes[i];
            for (int a = 0; a < 3; ++a) {
                const double pad = 1e-4 * (p.box.hi[a] - p.box.lo[a]) +
                                   1e-5 * std::max(std::fabs(p.box.lo[a]), std::fabs(p.box.hi[a]));
                p.box.lo[a] -= pad;
                p.box.hi[a] += pad;
                p.c[a] = 0.5 * (p.box.lo[a] + p.box.hi[a]);
            }
            p.id = i;
            tl.prims.push_back(p);
        }
    }
    tl.build_root();
    Box world;
    for (const Prim &p : tl.prims) world.grow(p.box);
    sc->instance_mirrored.resize(d->instance_count);
    for (uint32_t i = 0; i < d->instance_count; ++i)
        sc->instance_mirrored[i] = dt(o2w[i].c0, crs(o2w[i].c1, o2w[i].c2)) < 0.0f ? 1u : 0u;
    sc->stats.tlas_ms = lap();

    // ---- traversal-stack bound: every ray's stack must fit the device's
    // kTraversalStackSize entries.  A tree that could exceed it is rebuilt
    // with median splits only (balanced: about 3 entries per two binary
    // levels); a scene that still exceeds it is rejected, so no traversal
    // ever drops a subtree.
#if PSY_BVH_WIDTH == 8
    const uint32_t stack_cap = psy::kTraversalStackSize8;
    std::vector<psy::WideNodeGpu> tl_wide(1);
    std::vector<uint32_t> tl_leaves;
    std::vector<psy::CwNodeGpu> tl_cw = tl.widen8(tl_leaves);
    auto instance_depths = [&]() {
        tl_cw = tl.widen8(tl_leaves);
        return tlas_instance_depths8(tl_cw, tl_leaves, d->instance_count);
    };
#else
    const uint32_t stack_cap = psy::kTraversalStackSize;
    std::vector<psy::WideNodeGpu> tl_wide = tl.widen();
    auto instance_depths = [&]() {
        tl_wide = tl.widen();
        return tlas_instance_depths(tl_wide, d->instance_count);
    };
#endif
    std::vector<uint32_t> inst_depth = instance_depths();
    auto tlas_depth = [&]() {
        uint32_t deepest = 0u;
        for (const Prim &p : tl.prims) deepest = std::max(deepest, inst_depth[p.id]);
        return deepest;
    };
    if (!tl.prims.empty() && tlas_depth() + 1u > stack_cap / 2u) {
        tl.sah_depth_limit = 0;
        tl.build_root();
        inst_depth = instance_depths();
    }
    auto mesh_budgets = [&]() {
        std::vector<uint32_t> budget(d->mesh_count, stack_cap);
        for (const Prim &p : tl.prims) {
            const uint32_t mesh = d->instances[p.id].mesh;
            const uint32_t used = inst_depth[p.id] + 1u;
            budget[mesh] = std::min(budget[mesh], used >= stack_cap ? 0u : stack_cap - used);
        }
        return budget;
    };
    {
        const std::vector<uint32_t> budget = mesh_budgets();
        for (uint32_t i = 0; i < d->mesh_count; ++i) {
            if (mesh_need[i] <= budget[i]) continue;
            build_mesh(i, 0);
            sc->stats.median_rebuilds += 1u;
            if (mesh_need[i] > budget[i])
                return fail(PSY_ERROR_UNSUPPORTED, "mesh " + std::to_string(i) + ": its BVH needs " +
                                                       std::to_string(mesh_need[i]) + " traversal stack entries below " +
                                                       "its instances, more than the " + std::to_string(budget[i]) +
                                                       " left of " + std::to_string(stack_cap));
        }
        uint32_t need = 0u;
        for (const Prim &p : tl.prims)
            need = std::max(need, inst_depth[p.id] + 1u + mesh_need[d->instances[p.id].mesh]);
        sc->stats.stack_need = need;
        sc->stats.stack_capacity = stack_cap;
    }

    uint32_t prim_offset = 0;
    for (uint32_t i = 0; i < d->mesh_count; ++i) {
        const psy_mesh_desc &m = d->meshes[i];
        psy::MeshGpu &g = meshes[i];
        g.vertex_offset = uint32_t(positions.size() / 3u);
        g.index_offset = uint32_t(indices.size());
        g.triangle_count = m.triangle_count;
        g.prim_offset = prim_offset;
        g.smooth = m.smooth ? 1u : 0u;
        prim_offset += m.triangle_count;
        positions.insert(positions.end(), m.positions, m.positions + 3ull * m.vertex_count);
        if (m.smooth) normals.insert(normals.end(), m.normals, m.normals + 3ull * m.vertex_count);
        else normals.resize(positions.size(), 0.0f);
        indices.insert(indices.end(), m.indices, m.indices + 3ull * m.triangle_count);
        if (m.materials) {
            g.material_offset = uint32_t(tri_materials.size());
            tri_materials.insert(tri_materials.end(), m.materials, m.materials + m.triangle_count);
        } else {
            g.material_offset = psy::kInvalidId;
        }
        g.tri_offset = uint32_t(mesh_tri_first[i]);
#if PSY_BVH_WIDTH == 8
        g.node_offset = uint32_t(blas8.size());
        for (psy::CwNodeGpu &w : mesh_cw[i]) {
            w.child_base += g.node_offset;
            w.leaf_base += g.tri_offset;
        }
        blas8.insert(blas8.end(), mesh_cw[i].begin(), mesh_cw[i].end());
        std::vector<psy::CwNodeGpu>().swap(mesh_cw[i]);
#endif
        g.node_offset = PSY_BVH_WIDTH == 8 ? g.node_offset : uint32_t(blas.size());
        // global node and triangle indices of the mesh's links
        for (psy::WideNodeGpu &w : mesh_wide[i]) {
            int *lk = &w.link.x;
            const int *ct = &w.count.x;
            for (int k = 0; k < 4; ++k) {
                const uint32_t v = uint32_t(lk[k]);
                if (ct[k] > 0) lk[k] = int(v + g.tri_offset);
                else if (v != psy::kInvalidId && (v & psy::kTagMask) == psy::kTagBlas)
                    lk[k] = int(psy::kTagBlas | ((v & ~psy::kTagMask) + g.node_offset));
            }
        }
        blas.insert(blas.end(), mesh_wide[i].begin(), mesh_wide[i].end());
        std::vector<psy::WideNodeGpu>().swap(mesh_wide[i]);
        sc->triangle_count += m.triangle_count;
    }
    if (blas.empty()) blas.push_back({});
    if (blas8.empty()) blas8.push_back({});

    // ---- materials and parameter blocks
    std::vector<psy_closure_instruction> code;
    std::vector<psy_value_instruction> values;
    bool any_transparent = false, any_glossy = false;
    for (uint32_t i = 0; i < d->material_count; ++i) {
        const psy_material_desc &m = d->materials[i];
        psy::MaterialGpu g{};
        g.code_offset = uint32_t(code.size());
        g.code_count = m.closure_count;
        g.value_offset = uint32_t(values.size());
        g.value_count = m.value_count;
        values.insert(values.end(), m.values, m.values + m.value_count);
        g.root = m.root;
        g.scalar_offset = uint32_t(sc->scalars.size());
        g.vector_offset = uint32_t(sc->vectors.size() / 3u);
        g.emission_sampling = m.emission_sampling;
        g.bump_correction = (m.flags & PSY_MATERIAL_NO_BUMP_MAP_CORRECTION) == 0u ? 1u : 0u;
        for (uint32_t k = 0; k < m.closure_count; ++k) {
            if (m.closures[k].op == PSY_CLOSURE_EMISSION) g.has_emission = 1u;
            if (m.closures[k].op == PSY_CLOSURE_TRANSPARENT) g.has_transparent = 1u;
        }
        any_transparent = any_transparent || g.has_transparent;
        for (uint32_t k = 0; k < m.closure_count; ++k)
            if (m.closures[k].op == PSY_CLOSURE_GLOSSY || m.closures[k].op == PSY_CLOSURE_GLASS ||
                m.closures[k].op == PSY_CLOSURE_REFRACTION)
                any_glossy = true;
        code.insert(code.end(), m.closures, m.closures + m.closure_count);
        sc->scalars.insert(sc->scalars.end(), m.scalars, m.scalars + m.scalar_count);
        sc->vectors.insert(sc->vectors.end(), m.vectors, m.vectors + 3ull * m.vector_count);
        sc->materials.push_back(g);
    }

    // ---- Cycles' GGX albedo tables, for MULTI_GGX glossy closures
    bool any_multi_ggx = false;
    for (const psy_closure_instruction &c : code)
        if (c.op == PSY_CLOSURE_GLOSSY && c.a == PSY_GLOSSY_MULTI_GGX) any_multi_ggx = true;
    if (any_multi_ggx && (d->ggx_e == nullptr || d->ggx_eavg == nullptr))
        return fail(PSY_ERROR_INVALID_ARGUMENT, "MULTI_GGX glossy closures need the scene's GGX albedo tables");
    std::vector<float> ggx_tables;
    if (any_multi_ggx) {
        ggx_tables.assign(d->ggx_e, d->ggx_e + psy::kGgxETableSize);
        ggx_tables.insert(ggx_tables.end(), d->ggx_eavg, d->ggx_eavg + psy::kGgxEavgTableSize);
    }

    // ---- emissive triangles + flat light distribution
    // (src/sampling/light_distribution.cpp:25-150; emitter geometry as in
    // src/luisa/path_kernel_emissive_triangle.cpp:80-150)
    // in parallel over chunks of an instance's triangles, concatenated in
    // (instance, triangle) order
    constexpr uint32_t kEmitterChunk = 4096u;
    struct EmitterJob {
        uint32_t instance, first, end;
    };
    std::vector<EmitterJob> emitter_jobs;
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const uint32_t n = d->meshes[d->instances[i].mesh].triangle_count;
        for (uint32_t f = 0; f < n; f += kEmitterChunk) emitter_jobs.push_back({i, f, std::min(n, f + kEmitterChunk)});
    }
    std::vector<std::vector<psy::EmitterGpu>> instance_emitters(emitter_jobs.size());
    uint32_t emitter_threads = 0u;
    const psy_status emit_status = parallel_for(uint32_t(emitter_jobs.size()), &emitter_threads, [&](uint32_t job) {
        const uint32_t i = emitter_jobs[job].instance;
        std::vector<psy::EmitterGpu> &out_e = instance_emitters[job];
        const psy_instance_desc &id = d->instances[i];
        const psy_mesh_desc &m = d->meshes[id.mesh];
        const psy::InstanceGpu &g = instances[i];
        M34 nrm;
        nrm.c0 = {g.nrm[0], g.nrm[1], g.nrm[2]};
        nrm.c1 = {g.nrm[3], g.nrm[4], g.nrm[5]};
        nrm.c2 = {g.nrm[6], g.nrm[7], g.nrm[8]};
        nrm.c3 = {0, 0, 0};
        for (uint32_t k = emitter_jobs[job].first; k < emitter_jobs[job].end; ++k) {
            const uint32_t mi = m.materials ? m.materials[k] : id.material;
            const psy::MaterialGpu &mat = sc->materials[mi];
            if (!mat.has_emission || mat.emission_sampling == 0u) continue;
            auto vert = [&](int c) {
                const float *v = m.positions + 3ull * m.indices[3ull * k + c];
                return v3(v[0], v[1], v[2]);
            };
            const V3 l0 = vert(0), l1 = vert(1), l2 = vert(2);
            const V3 p0 = xaff(o2w[i], l0, true), p1 = xaff(o2w[i], l1, true), p2 = xaff(o2w[i], l2, true);
            V3 ln = crs(sub(l1, l0), sub(l2, l0));
            const float l2n = dt(ln, ln);
            ln = l2n > 1.0e-20f ? V3{ln.x / std::sqrt(std::max(l2n, 1.0e-20f)), ln.y / std::sqrt(std::max(l2n, 1.0e-20f)),
                                     ln.z / std::sqrt(std::max(l2n, 1.0e-20f))}
                                : v3(0.0f, 0.0f, 1.0f);
            V3 ng = xaff(nrm, ln, false);
            const float g2 = dt(ng, ng);
            ng = g2 > 1.0e-20f ? V3{ng.x / std::sqrt(std::max(g2, 1.0e-20f)), ng.y / std::sqrt(std::max(g2, 1.0e-20f)),
                                    ng.z / std::sqrt(std::max(g2, 1.0e-20f))}
                               : v3(0.0f, 0.0f, 1.0f);
            const V3 cr = crs(sub(p1, p0), sub(p2, p0));
            psy::EmitterGpu e{};
            e.p0[0] = p0.x; e.p0[1] = p0.y; e.p0[2] = p0.z;
            e.p1[0] = p1.x; e.p1[1] = p1.y; e.p1[2] = p1.z;
            e.p2[0] = p2.x; e.p2[1] = p2.y; e.p2[2] = p2.z;
            e.ng[0] = ng.x; e.ng[1] = ng.y; e.ng[2] = ng.z;
            e.area = 0.5f * std::sqrt(dt(cr, cr));
            e.material = mi;
            e.object = i;
            e.cycles_prim = meshes[id.mesh].prim_offset + k;
            e.emission_sampling = mat.emission_sampling;
            out_e.push_back(e);
        }
    });
    if (emit_status != PSY_OK) return emit_status;
    // the chunks' emitters concatenated in chunk order, each chunk copied on
    // a thread of its own
    std::vector<size_t> chunk_first(instance_emitters.size() + 1u, 0u);
    for (size_t j = 0; j < instance_emitters.size(); ++j)
        chunk_first[j + 1u] = chunk_first[j] + instance_emitters[j].size();
    std::vector<psy::EmitterGpu> emitters(chunk_first.back());
    std::vector<float> areas(chunk_first.back());
    const psy_status gathered = parallel_for(uint32_t(instance_emitters.size()), nullptr, [&](uint32_t job) {
        const std::vector<psy::EmitterGpu> &v = instance_emitters[job];
        for (size_t k = 0; k < v.size(); ++k) {
            emitters[chunk_first[job] + k] = v[k];
            areas[chunk_first[job] + k] = v[k].area;
        }
    });
    if (gathered != PSY_OK) return gathered;
    std::vector<std::vector<psy::EmitterGpu>>().swap(instance_emitters);
    std::vector<psy::DistEntryGpu> dist;
    const uint32_t tri_n = uint32_t(areas.size()), light_n = d->light_count;
    dist.reserve(size_t(tri_n) + light_n + 1u);
    auto valid_area = [](float a) { return std::isfinite(a) && a > 0.0f ? a : 0.0f; };
    float total = 0.0f;
    for (uint32_t i = 0; i < tri_n; ++i) {
        dist.push_back({total, 0.0f, 0u, i});
        total += valid_area(areas[i]);
    }
    const float triangle_area = total;
    const float light_area = light_n > 0u ? (total > 0.0f ? total / float(light_n) : 1.0f) : 0.0f;
    for (uint32_t i = 0; i < light_n; ++i) {
        dist.push_back({total, 0.0f, 1u, i});
        total += light_area;
    }
    dist.push_back({total, 0.0f, 3u, 0u});
    float triangle_area_pdf = 0.0f, light_selection_pdf = 0.0f;
    if (triangle_area > 0.0f) {
        triangle_area_pdf = 1.0f / triangle_area;
        if (light_n > 0u) triangle_area_pdf *= 0.5f;
    }
    if (light_n > 0u) {
        light_selection_pdf = 1.0f / float(light_n);
        if (triangle_area > 0.0f) light_selection_pdf *= 0.5f;
    }
    for (uint32_t i = 0; i < tri_n; ++i) dist[i].selection_pdf = valid_area(areas[i]) * triangle_area_pdf;
    for (uint32_t i = tri_n; i < tri_n + light_n; ++i) dist[i].selection_pdf = light_selection_pdf;
    if (total > 0.0f) {
        const float inv = 1.0f / total;
        for (uint32_t i = 0; i < tri_n + light_n; ++i) dist[i].cumulative *= inv;
        dist.back().cumulative = 1.0f;
    }
    std::vector<psy_light_desc> lights(d->lights, d->lights + d->light_count);
    // effective use_mis and forward intersectability (path_tracer_scene.cpp:1787-1830)
    for (psy_light_desc &l : lights) {
        bool extent = true;
        if (l.type == PSY_LIGHT_POINT || l.type == PSY_LIGHT_SPOT) extent = l.radius > 0.0f;
        else if (l.type == PSY_LIGHT_AREA) extent = l.size_u != 0.0f && l.size_v != 0.0f && l.spread > 0.0f;
        else if (l.type == PSY_LIGHT_DISTANT) extent = l.angle > 0.0f;
        const bool mis = (l.flags & PSY_LIGHT_FLAG_USE_MIS) != 0u && extent;
        if (mis) l.flags |= psy::kLightFlagUseMis;
        if (mis && l.type != PSY_LIGHT_DISTANT) l.flags |= psy::kLightFlagForward;
    }

    sc->code_host = code;
    sc->values_host = values;
    sc->emitters_host = std::move(emitters);
    sc->lights_host = lights;
    sc->stats.emitters_ms = lap();

    // ---- upload.  Every scene array is a stream-ordered allocation from the
    // device pool: a later compile reuses the memory a destroyed scene gave
    // back, and parameter blocks replaced by edits are retired without
    // waiting on the device.
    for (DeviceBuffer *b : {&sc->tlas, &sc->blas, &sc->tlas8, &sc->blas8, &sc->tlas_ids, &sc->tris, &sc->instances, &sc->meshes, &sc->positions, &sc->normals,
                            &sc->indices, &sc->tri_materials, &sc->material_buf, &sc->code, &sc->value_buf, &sc->scalar_buf,
                            &sc->vector_buf, &sc->emitters, &sc->distribution, &sc->ggx_tables, &sc->lights, &sc->lamp_consts,
                            &sc->lamp_bounds, &sc->lamp_ids})
        b->ordered = st;
    PSY_CUDA_TRY(sc->tlas.upload(tl_wide, st));
    PSY_CUDA_TRY(sc->blas.upload(blas, st));
#if PSY_BVH_WIDTH == 8
    if (tl_leaves.empty()) tl_leaves.push_back(0u);
    PSY_CUDA_TRY(sc->tlas8.upload(tl_cw, st));
    PSY_CUDA_TRY(sc->blas8.upload(blas8, st));
    PSY_CUDA_TRY(sc->tlas_ids.upload(tl_leaves, st));
#endif
    PSY_CUDA_TRY(sc->tris.upload(tris, st));
    PSY_CUDA_TRY(sc->instances.upload(instances, st));
    PSY_CUDA_TRY(sc->meshes.upload(meshes, st));
    PSY_CUDA_TRY(sc->positions.upload(positions, st));
    PSY_CUDA_TRY(sc->normals.upload(normals, st));
    PSY_CUDA_TRY(sc->indices.upload(indices, st));
    PSY_CUDA_TRY(sc->tri_materials.upload(tri_materials, st));
    PSY_CUDA_TRY(sc->material_buf.upload(sc->materials, st));
    PSY_CUDA_TRY(sc->code.upload(code, st));
    PSY_CUDA_TRY(sc->value_buf.upload(values, st));
    PSY_CUDA_TRY(sc->scalar_buf.upload(sc->scalars, st));
    PSY_CUDA_TRY(sc->vector_buf.upload(sc->vectors, st));
    PSY_CUDA_TRY(sc->emitters.upload(sc->emitters_host, st));
    PSY_CUDA_TRY(sc->distribution.upload(dist, st));
    if (!ggx_tables.empty()) PSY_CUDA_TRY(sc->ggx_tables.upload(ggx_tables, st));
    PSY_CUDA_TRY(sc->lights.upload(lights, st));
    std::vector<psy::LampConstGpu> lamp_consts;
    lamp_consts.reserve(lights.size());
    for (const psy_light_desc &l : lights) lamp_consts.push_back(lamp_constants(l));
    PSY_CUDA_TRY(sc->lamp_consts.upload(lamp_consts, st));
    // lamps a ray can hit, in light order, with a bounding sphere each
    std::vector<float4> lamp_bounds;
    std::vector<uint32_t> lamp_ids;
    for (uint32_t i = 0; i < light_n; ++i) {
        const psy_light_desc &l = lights[i];
        double r2 = -1.0;
        if (l.type == PSY_LIGHT_AREA && l.size_u * l.size_v != 0.0f) {
            double hu2 = 0.0, hv2 = 0.0, huv = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double hu = 0.5 * double(l.size_u) * double(l.axis_x[k]);
                const double hv = 0.5 * double(l.size_v) * double(l.axis_y[k]);
                hu2 += hu * hu;
                hv2 += hv * hv;
                huv += hu * hv;
            }
            r2 = hu2 + hv2 + 2.0 * std::fabs(huv);
        } else if ((l.type == PSY_LIGHT_POINT || l.type == PSY_LIGHT_SPOT) && l.radius > 0.0f) {
            r2 = double(l.radius) * double(l.radius);
        }
        if (r2 < 0.0) continue;
        lamp_bounds.push_back(make_float4(l.position[0], l.position[1], l.position[2], float(r2 * (1.0 + 1.0e-6))));
        lamp_ids.push_back(i);
    }
    PSY_CUDA_TRY(sc->lamp_bounds.upload(lamp_bounds, st));
    PSY_CUDA_TRY(sc->lamp_ids.upload(lamp_ids, st));
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    sc->stats.upload_bytes = 0u;
    for (const DeviceBuffer *b : {&sc->tlas, &sc->blas, &sc->tlas8, &sc->blas8, &sc->tlas_ids, &sc->tris, &sc->instances, &sc->meshes, &sc->positions,
                                  &sc->normals, &sc->indices, &sc->tri_materials, &sc->material_buf, &sc->code,
                                  &sc->value_buf, &sc->scalar_buf, &sc->vector_buf, &sc->emitters, &sc->distribution, &sc->ggx_tables, &sc->lights,
                                  &sc->lamp_consts, &sc->lamp_bounds, &sc->lamp_ids})
        sc->stats.upload_bytes += b->bytes;
    psy::SceneView &v = sc->view;
    v.tlas = sc->tlas.as<psy::WideNodeGpu>();
    v.blas = sc->blas.as<psy::WideNodeGpu>();
    v.tlas8 = sc->tlas8.as<psy::CwNodeGpu>();
    v.blas8 = sc->blas8.as<psy::CwNodeGpu>();
    v.tlas_ids = sc->tlas_ids.as<uint32_t>();
    v.tris = sc->tris.as<float4>();
    v.instances = sc->instances.as<psy::InstanceGpu>();
    v.meshes = sc->meshes.as<psy::MeshGpu>();
    v.positions = sc->positions.as<float>();
    v.normals = sc->normals.as<float>();
    v.indices = sc->indices.as<uint32_t>();
    v.tri_materials = sc->tri_materials.as<uint32_t>();
    v.materials = sc->material_buf.as<psy::MaterialGpu>();
    v.code = sc->code.as<psy_closure_instruction>();
    v.values = sc->value_buf.as<psy_value_instruction>();
    v.scalars = sc->scalar_buf.as<float>();
    v.vectors = sc->vector_buf.as<float>();
    v.emitters = sc->emitters.as<psy::EmitterGpu>();
    v.distribution = sc->distribution.as<psy::DistEntryGpu>();
    v.ggx_e = ggx_tables.empty() ? nullptr : sc->ggx_tables.as<float>();
    v.ggx_eavg = ggx_tables.empty() ? nullptr : sc->ggx_tables.as<float>() + psy::kGgxETableSize;
    v.lights = sc->lights.as<psy_light_desc>();
    v.lamp_bounds = sc->lamp_bounds.as<float4>();
    v.lamp_consts = sc->lamp_consts.as<psy::LampConstGpu>();
    if (!world.empty())
        for (int a = 0; a < 3; ++a) {
            (&v.world_lo.x)[a] = float(world.lo[a]);
            (&v.world_hi.x)[a] = float(world.hi[a]);
        }
    v.lamp_ids = sc->lamp_ids.as<uint32_t>();
    v.lamp_count = uint32_t(lamp_ids.size());
    v.instance_count = tl.prims.empty() ? 0u : d->instance_count;
    v.emitter_count = tri_n + light_n;
    v.triangle_emitters = tri_n;
    v.light_count = light_n;
    v.triangle_area_pdf = triangle_area_pdf;
    v.light_selection_pdf = light_selection_pdf;
    v.background[0] = d->background[0];
    v.background[1] = d->background[1];
    v.background[2] = d->background[2];
    v.world_visibility = d->world_visibility;
    v.any_transparent = any_transparent ? 1u : 0u;
    v.has_glossy = any_glossy ? 1u : 0u;
    // the light tree is built on first use (ensure_light_tree)
    sc->stats.upload_ms = lap();
    sc->stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
    *out = sc.release();
    return PSY_OK;
}

void psy_scene_destroy(psy_scene *s) {
    if (!s) return;
    cudaSetDevice(s->context->device);
    if (s->uploads_done) {
        cudaEventSynchronize(s->uploads_done);
        cudaEventDestroy(s->uploads_done);
    }
    delete s;
}

uint64_t psy_scene_source_revision(const psy_scene *s) { return s ? s->revision : 0u; }

psy_status psy_scene_rebind_parameters(psy_scene *s, uint32_t material, const float *scalars, uint32_t scalar_count,
                                       const float *vectors, uint32_t vector_count) {
    const psy_status valid = check_rebind(s, material, scalars, scalar_count, vectors, vector_count);
    if (valid != PSY_OK) return valid;
    const psy::MaterialGpu &m = s->materials[material];
    cudaStream_t st = s->context->stream;
    PSY_CUDA_TRY(cudaSetDevice(s->context->device));
    if (scalar_count) {
        std::memcpy(s->scalars.data() + m.scalar_offset, scalars, sizeof(float) * scalar_count);
        PSY_CUDA_TRY(cudaMemcpyAsync(s->scalar_buf.as<float>() + m.scalar_offset, scalars, sizeof(float) * scalar_count,
                                     cudaMemcpyHostToDevice, st));
    }
    if (vector_count) {
        std::memcpy(s->vectors.data() + 3ull * m.vector_offset, vectors, sizeof(float) * 3u * vector_count);
        PSY_CUDA_TRY(cudaMemcpyAsync(s->vector_buf.as<float>() + 3ull * m.vector_offset, vectors,
                                     sizeof(float) * 3u * vector_count, cudaMemcpyHostToDevice, st));
    }
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    // the light tree's energies follow the emission estimates: rebuild a
    // built tree when an emissive material changes, as a recompile would
    if (m.has_emission) {
        std::lock_guard<std::mutex> lock(s->light_tree_mutex);
        if (s->light_tree_built) {
            const psy_status r = build_light_tree(s);
            if (r != PSY_OK) return r;
        }
    }
    // renders through a session are synchronous: nothing queued reads the
    // replaced tree any more
    release_retired(s);
    return PSY_OK;
}

psy_status psy_scene_get_build_stats(const psy_scene *s, psy_scene_build_stats *out) {
    if (!s || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = s->stats;
    return PSY_OK;
}

psy_status psy_session_create(psy_scene *scene, const psy_render_settings *settings, psy_session **out) {
    if (!scene || !settings || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    PSY_CUDA_TRY(cudaSetDevice(scene->context->device));
    auto s = std::make_unique<psy_session>();
    s->scene = scene;
    s->settings = *settings;
    psy_status r = derive_params(s.get(), *settings);
    if (r != PSY_OK) return r;
    const auto table = filter_table(settings->pixel_filter, settings->filter_width);
    std::vector<float> tv(table.begin(), table.end());
    PSY_CUDA_TRY(s->filter.upload(tv, scene->context->stream));
    s->params.filter = s->filter.as<float>();
    if ((r = clear_film(s.get())) != PSY_OK) return r;
    PSY_CUDA_TRY(s->trace_buf.alloc(sizeof(psy_path_trace)));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_begin));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_end));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_k[0]));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_k[1]));
    *out = s.release();
    return PSY_OK;
}

}  // extern "C"

psy_status psy::host::create_server_session(psy_scene *scene, const psy_render_settings &settings,
                                            const psy_camera_desc *camera, psy_session **out) {
    *out = nullptr;
    PSY_CUDA_TRY(cudaSetDevice(scene->context->device));
    cudaStream_t st = scene->context->stream;
    auto s = std::make_unique<psy_session>();
    s->scene = scene;
    s->settings = settings;
    for (DeviceBuffer *b : {&s->sobol, &s->filter, &s->combined, &s->normal, &s->albedo, &s->sample_count, &s->trace_buf})
        b->ordered = st;
    s->has_camera = camera != nullptr;
    if (camera) s->camera = *camera;
    psy_status r = derive_params(s.get(), settings);
    if (r != PSY_OK) return r;
    // (copies from pageable host memory are staged before the call returns,
    // so the temporary tables may go at once)
    const auto table = filter_table(settings.pixel_filter, settings.filter_width);
    const std::vector<float> tv(table.begin(), table.end());
    PSY_CUDA_TRY(s->filter.upload(tv, st));
    s->params.filter = s->filter.as<float>();
    if ((r = clear_film(s.get(), false)) != PSY_OK) return r;
    PSY_CUDA_TRY(s->trace_buf.alloc(sizeof(psy_path_trace)));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_begin));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_end));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_k[0]));
    PSY_CUDA_TRY(cudaEventCreate(&s->ev_k[1]));
    *out = s.release();
    return PSY_OK;
}

extern "C" {

void psy_session_destroy(psy_session *s) {
    if (!s) return;
    cudaSetDevice(s->scene->context->device);
    if (s->ev_begin) cudaEventDestroy(s->ev_begin);
    if (s->ev_end) cudaEventDestroy(s->ev_end);
    for (cudaEvent_t e : s->ev_k)
        if (e) cudaEventDestroy(e);
    delete s;
}

psy_status psy_session_reset(psy_session *s, const psy_render_settings *settings) {
    if (!s || !settings) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    PSY_CUDA_TRY(cudaSetDevice(s->scene->context->device));
    s->settings = *settings;
    psy_status r = derive_params(s, *settings);
    if (r != PSY_OK) return r;
    const auto table = filter_table(settings->pixel_filter, settings->filter_width);
    std::vector<float> tv(table.begin(), table.end());
    PSY_CUDA_TRY(s->filter.upload(tv, s->scene->context->stream));
    s->params.filter = s->filter.as<float>();
    s->cancelled.store(false);
    return clear_film(s);
}

psy_status psy_session_set_camera(psy_session *s, const psy_camera_desc *camera) {
    if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "null session");
    PSY_CUDA_TRY(cudaSetDevice(s->scene->context->device));
    s->has_camera = camera != nullptr;
    if (camera) s->camera = *camera;
    psy_status r = derive_params(s, s->settings);
    if (r != PSY_OK) return r;
    s->params.filter = s->filter.as<float>();
    return clear_film(s);
}

void psy_session_cancel(psy_session *s) {
    if (s) s->cancelled.store(true);
}

uint32_t psy_session_rendered_samples(const psy_session *s) { return s ? s->rendered : 0u; }

psy_status psy_session_request_trace(psy_session *s, uint32_t x, uint32_t y, uint32_t sample) {
    if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "null session");
    if (x >= s->params.full_w || y >= s->params.full_h) return fail(PSY_ERROR_INVALID_ARGUMENT, "trace pixel outside the film");
    s->trace_requested = true;
    s->trace_x = x;
    s->trace_y = y;
    s->trace_sample = sample;
    std::memset(&s->trace_host, 0, sizeof(s->trace_host));
    PSY_CUDA_TRY(cudaMemset(s->trace_buf.ptr, 0, sizeof(psy_path_trace)));
    return PSY_OK;
}

psy_status psy_session_read_trace(psy_session *s, psy_path_trace *out) {
    if (!s || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = s->trace_host;
    return PSY_OK;
}

}  // extern "C"

uint64_t psy::host::scene_device_bytes(const psy_scene *s) {
    uint64_t n = 0u;
    for (const DeviceBuffer *b : {&s->tlas, &s->blas, &s->tlas8, &s->blas8, &s->tlas_ids, &s->tris, &s->instances, &s->meshes, &s->positions, &s->normals,
                                  &s->indices, &s->tri_materials, &s->material_buf, &s->code, &s->value_buf, &s->scalar_buf,
                                  &s->vector_buf, &s->emitters, &s->distribution, &s->ggx_tables, &s->lights, &s->lamp_consts, &s->lamp_bounds,
                                  &s->lamp_ids, &s->lt_nodes, &s->lt_emitters, &s->lt_mapping, &s->lt_lookup})
        n += b->bytes;
    return n;
}

psy::JobGpu psy::host::session_job(const psy_session *s, const psy::RenderParams &p) {
    psy::JobGpu j{};
    j.p = p;
    j.s = s->scene->view;
    j.combined = s->combined.as<float4>();
    j.normal = s->normal.as<float4>();
    j.albedo = s->albedo.as<float4>();
    j.sample_count = s->sample_count.as<uint32_t>();
    return j;
}

psy_status psy::host::prepare_render(psy_session *s, uint32_t first, uint32_t count, uint32_t offset, uint32_t total,
                                      psy::RenderParams *out) {
    if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "null session");
    if (s->cancelled.load()) return fail(PSY_ERROR_CANCELLED, "session cancelled");
    if (count == 0u) return fail(PSY_ERROR_RANGE, "empty sample range");
    const uint64_t begin = uint64_t(first) + offset, end = begin + count;
    if (total == 0u || end > total) return fail(PSY_ERROR_RANGE, "sample range beyond the render's total");
    if (s->total != 0u && s->total != total) return fail(PSY_ERROR_STATE, "total sample count changed within the session");
    psy_context *ctx = s->scene->context;
    PSY_CUDA_TRY(cudaSetDevice(ctx->device));
    // Sobol table sized from the render's total (path_tracer_session.cpp:41-69)
    const uint32_t size = psy_sobol_sequence_size_for_samples(total);
    if (s->sobol_size != size) {
        std::vector<float> table(size_t(size) * 256u * 4u);
        psy_sobol_generate_table(size, table.data());
        PSY_CUDA_TRY(s->sobol.upload(table, ctx->stream));
        s->sobol_size = size;
    }
    s->total = total;
    *out = s->params;
    apply_light_selection(*out, s->settings, s->scene->view);
    out->sobol = s->sobol.as<float4>();
    out->sobol_size = s->sobol_size;
    return PSY_OK;
}

extern "C" {

psy_status psy_session_render_samples(psy_session *s, uint32_t first, uint32_t count, uint32_t offset, uint32_t total) {
    psy::RenderParams p;
    const psy_status prepared = prepare_render(s, first, count, offset, total, &p);
    if (prepared != PSY_OK) return prepared;
    const uint64_t begin = uint64_t(first) + offset, end = begin + count;
    psy_context *ctx = s->scene->context;
    std::lock_guard<std::mutex> render_lock(ctx->render_mutex);
    cudaStream_t st = ctx->stream;
    const uint32_t pixels = s->pixels;
    uint32_t per_batch = std::max(1u, std::min(count, ctx->path_capacity / std::max(pixels, 1u)));
    psy_status r = ensure_capacity(s, pixels * per_batch);
    if (r != PSY_OK) return r;
    psy_path_trace *trace = s->trace_requested ? s->trace_buf.as<psy_path_trace>() : nullptr;
    PSY_CUDA_TRY(cudaMemsetAsync(ctx->arena.stats.ptr, 0, 64, st));
    psy_render_stats stats{};
    PSY_CUDA_TRY(cudaEventRecord(s->ev_begin, st));
    const psy::LaunchConfig &lc = ctx->launch;
    const bool prof = s->profiling;
    if (prof) std::memset(&s->profile, 0, sizeof(s->profile));
    // Times one launch class when profiling: events on both sides, then a
    // synchronisation so the queue sizes the byte model needs are final.
    auto timed = [&](auto &&launch, uint32_t &launches, float &ms) -> psy_status {
        if (!prof) {
            launch();
            return PSY_OK;
        }
        PSY_CUDA_TRY(cudaEventRecord(s->ev_k[0], st));
        launch();
        PSY_CUDA_TRY(cudaEventRecord(s->ev_k[1], st));
        PSY_CUDA_TRY(cudaEventSynchronize(s->ev_k[1]));
        float t = 0.0f;
        PSY_CUDA_TRY(cudaEventElapsedTime(&t, s->ev_k[0], s->ev_k[1]));
        ms += t;
        launches += 1u;
        return PSY_OK;
    };
    auto read_counters = [&](uint32_t *c3) -> psy_status {
        PSY_CUDA_TRY(cudaMemcpyAsync(c3, ctx->arena.view.counters, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        PSY_CUDA_TRY(cudaStreamSynchronize(st));
        return PSY_OK;
    };
    psy_kernel_profile &pf = s->profile;
    psy_status ps = PSY_OK;
    for (uint64_t sample = begin; sample < end;) {
        if (s->cancelled.load()) return fail(PSY_ERROR_CANCELLED, "session cancelled");
        const uint32_t n_samples = uint32_t(std::min<uint64_t>(per_batch, end - sample));
        const uint32_t paths = pixels * n_samples;
        uint32_t trace_path = psy::kInvalidId;
        if (trace && s->trace_sample >= sample && s->trace_sample < sample + n_samples &&
            s->trace_x >= p.win_x && s->trace_x < p.win_x + p.win_w && s->trace_y >= p.win_y &&
            s->trace_y < p.win_y + p.win_h) {
            const uint32_t local = (s->trace_y - p.win_y) * p.win_w + (s->trace_x - p.win_x);
            trace_path = uint32_t(s->trace_sample - sample) * pixels + local;
        }
        psy_path_trace *tr = trace_path != psy::kInvalidId ? trace : nullptr;
        psy::PathBuffers b = ctx->arena.view;
        psy::launch_set_counters(st, b.counters, paths);
        if ((ps = timed([&] { psy::launch_raygen(st, lc, p, b, pixels, paths, uint32_t(sample), trace_path, tr); },
                        pf.raygen_launches, pf.raygen_ms)) != PSY_OK)
            return ps;
        pf.raygen_bytes += 164.0 * paths;
        stats.camera_rays += paths;
        for (uint32_t step = 0; step < p.steps; ++step) {
            uint32_t c3[3] = {0u, 0u, 0u};
            if (prof && (ps = read_counters(c3)) != PSY_OK) return ps;
            if ((ps = timed([&] { psy::launch_intersect(st, lc, s->scene->view, b, paths); }, pf.intersect_launches,
                            pf.intersect_ms)) != PSY_OK)
                return ps;
            pf.intersect_bytes += 88.0 * c3[0];
            if ((ps = timed([&] { psy::launch_shade(st, lc, s->scene->view, p, b, paths, step, trace_path, tr); },
                            pf.shade_launches, pf.shade_ms)) != PSY_OK)
                return ps;
            psy::launch_count_rays(st, b.counters, ctx->arena.stats.as<unsigned long long>());
            if (prof && (ps = read_counters(c3)) != PSY_OK) return ps;
            pf.shade_bytes += 304.0 * c3[0] + 68.0 * c3[2];
            if ((ps = timed([&] { psy::launch_shadow(st, lc, s->scene->view, p, b, paths, step, trace_path, tr); },
                            pf.shadow_launches, pf.shadow_ms)) != PSY_OK)
                return ps;
            pf.shadow_bytes += 100.0 * c3[2];
            psy::launch_swap(st, b.counters);
            std::swap(b.queue_in, b.queue_out);
            stats.kernel_launches += 5u;
            // every 4 steps, stop early once no path is left
            if ((step & 3u) == 3u) {
                uint32_t left = 0u;
                PSY_CUDA_TRY(cudaMemcpyAsync(&left, b.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                PSY_CUDA_TRY(cudaStreamSynchronize(st));
                if (left == 0u) break;
            }
        }
        if ((ps = timed([&] {
                 psy::launch_film(st, lc, b, pixels, n_samples, s->combined.as<float4>(), s->normal.as<float4>(),
                                  s->albedo.as<float4>(), s->sample_count.as<uint32_t>(), trace_path, tr);
             }, pf.film_launches, pf.film_ms)) != PSY_OK)
            return ps;
        pf.film_bytes += 48.0 * paths + 104.0 * pixels;
        stats.kernel_launches += 3u;
        stats.batches += 1u;
        sample += n_samples;
    }
    PSY_CUDA_TRY(cudaEventRecord(s->ev_end, st));
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    uint32_t overflows = 0u;
    PSY_CUDA_TRY(psy::take_stack_overflows(st, &overflows));
    if (overflows != 0u) return fail(PSY_ERROR_UNSUPPORTED, "traversal stack overflow on the device");
    float ms = 0.0f;
    PSY_CUDA_TRY(cudaEventElapsedTime(&ms, s->ev_begin, s->ev_end));
    unsigned long long counts[2] = {0, 0};
    PSY_CUDA_TRY(cudaMemcpy(counts, ctx->arena.stats.ptr, sizeof(counts), cudaMemcpyDeviceToHost));
    stats.closest_rays = counts[0];
    stats.path_segments = counts[0];
    stats.shadow_rays = counts[1];
    stats.ms_total = ms;
    s->last_stats = stats;
    s->rendered += count;
    if (trace) {
        PSY_CUDA_TRY(cudaMemcpy(&s->trace_host, trace, sizeof(psy_path_trace), cudaMemcpyDeviceToHost));
    }
    return PSY_OK;
}

// Allocation-free render for callers that cannot allocate device memory at
// render time.  Same kernels and sample order as psy_session_render_samples;
// the wavefront state and the Sobol table come from static device arrays
// (psy_static.cu).  The first call on a device takes the arrays' addresses
// and fills the table (ordered on the context stream and synchronised before
// the device counts as set up); make that first call before any stream
// capture.  Calls on one context are serialised by the context's render
// lock; calls on different contexts of one device share the arrays and race
// when they overlap on the GPU.
psy_status psy_session_render_samples_static(psy_session *s, uint32_t first, uint32_t count, uint32_t offset,
                                             uint32_t total) {
    if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "null session");
    if (s->cancelled.load()) return fail(PSY_ERROR_CANCELLED, "session cancelled");
    if (count == 0u) return fail(PSY_ERROR_RANGE, "empty sample range");
    const uint64_t begin = uint64_t(first) + offset, end = begin + count;
    if (total == 0u || end > total) return fail(PSY_ERROR_RANGE, "sample range beyond the render's total");
    if (s->total != 0u && s->total != total) return fail(PSY_ERROR_STATE, "total sample count changed within the session");
    if (psy_sobol_sequence_size_for_samples(total) != psy::kStaticSobolSize)
        return fail(PSY_ERROR_RANGE, "the static render supports renders of at most 256 total samples");
    if (s->pixels > psy::kStaticMaxPaths)
        return fail(PSY_ERROR_RANGE, "the static render supports windows of at most 65536 pixels");
    psy_context *ctx = s->scene->context;
    std::lock_guard<std::mutex> render_lock(ctx->render_mutex);
    cudaStream_t st = ctx->stream;
    PSY_CUDA_TRY(cudaSetDevice(ctx->device));
    void *base = nullptr;
    float4 *sobol = nullptr;
    PSY_CUDA_TRY(psy::static_scratch(ctx->device, st, sobol_pattern, &base, &sobol));
    // carve the static bytes into the wavefront arrays
    unsigned char *cursor = static_cast<unsigned char *>(base);
    auto carve = [&](size_t bytes) {
        unsigned char *p = cursor;
        cursor += (bytes + 255u) & ~size_t(255u);
        return p;
    };
    const size_t n = psy::kStaticMaxPaths;
    psy::PathBuffers b{};
    psy::host::bind_records(b, carve(psy::kPathRecordBytes * n));
    b.rad_final = reinterpret_cast<float4 *>(carve(16 * n));
    b.sample = reinterpret_cast<uint32_t *>(carve(4 * n));
    b.aov_n = reinterpret_cast<float4 *>(carve(16 * n));
    b.aov_a = reinterpret_cast<float4 *>(carve(16 * n));
    b.mis_n = reinterpret_cast<float4 *>(carve(16 * n));
    b.sh_o = reinterpret_cast<float4 *>(carve(16 * n));
    b.sh_d = reinterpret_cast<float4 *>(carve(16 * n));
    b.sh_c = reinterpret_cast<float4 *>(carve(16 * n));
    b.sh_ids = reinterpret_cast<uint4 *>(carve(16 * n));
    b.sh_path = reinterpret_cast<uint32_t *>(carve(4 * n));
    b.queue_in = reinterpret_cast<uint32_t *>(carve(4 * n));
    b.queue_out = reinterpret_cast<uint32_t *>(carve(4 * n));
    b.shadow_queue = reinterpret_cast<uint32_t *>(carve(4 * n));
    b.counters = reinterpret_cast<uint32_t *>(carve(64));
    if (cursor > static_cast<unsigned char *>(base) + psy::kStaticPathBytes)
        return fail(PSY_ERROR_STATE, "static path state larger than its array");
    unsigned long long *ray_stats = reinterpret_cast<unsigned long long *>(reinterpret_cast<unsigned char *>(b.counters) + 64);
    // the ray counters accumulate: clear them; every other array is written
    // before it is read within the call
    PSY_CUDA_TRY(cudaMemsetAsync(ray_stats, 0, 2 * sizeof(unsigned long long), st));
    psy::RenderParams p = s->params;
    apply_light_selection(p, s->settings, s->scene->view);
    p.sobol = sobol;
    p.sobol_size = psy::kStaticSobolSize;
    s->total = total;
    const uint32_t pixels = s->pixels;
    const uint32_t per_batch = std::max(1u, std::min(count, psy::kStaticMaxPaths / std::max(pixels, 1u)));
    // the static path state has no sort buffers
    psy::LaunchConfig lc = ctx->launch;
    lc.sort_threshold = 0u;
    lc.shadow_sort_threshold = 0u;
    lc.ray_sort_threshold = 0u;
    psy_render_stats stats{};
    PSY_CUDA_TRY(cudaEventRecord(s->ev_begin, st));
    for (uint64_t sample = begin; sample < end;) {
        if (s->cancelled.load()) return fail(PSY_ERROR_CANCELLED, "session cancelled");
        const uint32_t n_samples = uint32_t(std::min<uint64_t>(per_batch, end - sample));
        const uint32_t paths = pixels * n_samples;
        psy::PathBuffers bb = b;
        psy::launch_set_counters(st, bb.counters, paths);
        psy::launch_raygen(st, lc, p, bb, pixels, paths, uint32_t(sample), psy::kInvalidId, nullptr);
        stats.camera_rays += paths;
        for (uint32_t step = 0; step < p.steps; ++step) {
            psy::launch_intersect(st, lc, s->scene->view, bb, paths);
            psy::launch_shade(st, lc, s->scene->view, p, bb, paths, step, psy::kInvalidId, nullptr);
            psy::launch_count_rays(st, bb.counters, ray_stats);
            psy::launch_shadow(st, lc, s->scene->view, p, bb, paths, step, psy::kInvalidId, nullptr);
            psy::launch_swap(st, bb.counters);
            std::swap(bb.queue_in, bb.queue_out);
            stats.kernel_launches += 5u;
            if ((step & 3u) == 3u) {
                uint32_t left = 0u;
                PSY_CUDA_TRY(cudaMemcpyAsync(&left, bb.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                PSY_CUDA_TRY(cudaStreamSynchronize(st));
                if (left == 0u) break;
            }
        }
        psy::launch_film(st, lc, bb, pixels, n_samples, s->combined.as<float4>(), s->normal.as<float4>(),
                         s->albedo.as<float4>(), s->sample_count.as<uint32_t>(), psy::kInvalidId, nullptr);
        stats.kernel_launches += 3u;
        stats.batches += 1u;
        sample += n_samples;
    }
    PSY_CUDA_TRY(cudaEventRecord(s->ev_end, st));
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    uint32_t overflows = 0u;
    PSY_CUDA_TRY(psy::take_stack_overflows(st, &overflows));
    if (overflows != 0u) return fail(PSY_ERROR_UNSUPPORTED, "traversal stack overflow on the device");
    float ms = 0.0f;
    PSY_CUDA_TRY(cudaEventElapsedTime(&ms, s->ev_begin, s->ev_end));
    unsigned long long counts[2] = {0, 0};
    PSY_CUDA_TRY(cudaMemcpy(counts, ray_stats, sizeof(counts), cudaMemcpyDeviceToHost));
    stats.closest_rays = counts[0];
    stats.path_segments = counts[0];
    stats.shadow_rays = counts[1];
    stats.ms_total = ms;
    s->last_stats = stats;
    s->rendered += count;
    return PSY_OK;
}

psy_status psy_session_read_pass(psy_session *s, uint32_t pass_kind, float *out, uint64_t capacity, uint32_t *channels) {
    if (!s || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    const uint64_t n = s->pixels;
    const uint32_t ch = pass_kind == PSY_PASS_SAMPLE_COUNT ? 1u : 4u;
    if (pass_kind != PSY_PASS_COMBINED && pass_kind != PSY_PASS_NORMAL && pass_kind != PSY_PASS_ALBEDO &&
        pass_kind != PSY_PASS_DENOISING_NORMAL && pass_kind != PSY_PASS_DENOISING_ALBEDO &&
        pass_kind != PSY_PASS_SAMPLE_COUNT)
        return fail(PSY_ERROR_UNSUPPORTED, "pass kind not produced by this backend");
    if (capacity < n * ch) return fail(PSY_ERROR_INVALID_ARGUMENT, "output buffer too small");
    if (channels) *channels = ch;
    psy_context *ctx = s->scene->context;
    PSY_CUDA_TRY(cudaSetDevice(ctx->device));
    std::lock_guard<std::mutex> lock(ctx->readback_mutex);
    cudaStream_t st = ctx->readback;
    const size_t bytes = sizeof(float) * ch * n;
    if (ctx->readback_pass.bytes < std::max<size_t>(bytes, 16)) PSY_CUDA_TRY(ctx->readback_pass.alloc(std::max<size_t>(bytes, 16)));
    if (!ctx->readback_flag.ptr) PSY_CUDA_TRY(ctx->readback_flag.alloc(16));
    if (ctx->readback_host_bytes < std::max<size_t>(bytes, 16)) {
        if (ctx->readback_host) PSY_CUDA_TRY(cudaFreeHost(ctx->readback_host));
        ctx->readback_host = nullptr;
        ctx->readback_host_bytes = 0;
        PSY_CUDA_TRY(cudaMallocHost(&ctx->readback_host, std::max<size_t>(bytes, 16)));
        ctx->readback_host_bytes = std::max<size_t>(bytes, 16);
    }
    // write_passes fails when pixels disagree on the sample count
    // (src/luisa/path_tracer_session.cpp:88-95); checked on the device
    psy::launch_check_counts(st, s->sample_count.as<uint32_t>(), uint32_t(n), s->rendered, ctx->readback_flag.as<uint32_t>());
    uint32_t *flag = static_cast<uint32_t *>(ctx->readback_host);
    PSY_CUDA_TRY(cudaMemcpyAsync(flag, ctx->readback_flag.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    if (*flag != 0u) return fail(PSY_ERROR_STATE, "film sample counts disagree with the session");
    const void *src = pass_kind == PSY_PASS_COMBINED ? s->combined.ptr
                      : (pass_kind == PSY_PASS_NORMAL || pass_kind == PSY_PASS_DENOISING_NORMAL) ? s->normal.ptr
                                                                                                  : s->albedo.ptr;
    const uint32_t kind = pass_kind == PSY_PASS_SAMPLE_COUNT ? 2u : (pass_kind == PSY_PASS_COMBINED ? 0u : 1u);
    psy::launch_resolve_pass(st, static_cast<const float4 *>(src), s->sample_count.as<uint32_t>(), uint32_t(n), kind,
                             s->settings.film_exposure, ctx->readback_pass.as<float>());
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaMemcpyAsync(ctx->readback_host, ctx->readback_pass.ptr, bytes, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    // staging -> caller's buffer, in 8 MiB pieces on several host threads
    constexpr size_t kPiece = size_t(8) << 20;
    const size_t pieces = (bytes + kPiece - 1) / kPiece;
    const unsigned char *from = static_cast<const unsigned char *>(ctx->readback_host);
    unsigned char *to = reinterpret_cast<unsigned char *>(out);
    return parallel_for(uint32_t(pieces), nullptr, [&](uint32_t k) {
        const size_t at = size_t(k) * kPiece;
        std::memcpy(to + at, from + at, std::min(kPiece, bytes - at));
    });
}

psy_status psy_session_set_profiling(psy_session *s, uint32_t enabled) {
    if (!s) return fail(PSY_ERROR_INVALID_ARGUMENT, "null session");
    s->profiling = enabled != 0u;
    return PSY_OK;
}

psy_status psy_session_profile(const psy_session *s, psy_kernel_profile *out) {
    if (!s || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = s->profile;
    return PSY_OK;
}

psy_status psy_session_stats(const psy_session *s, psy_render_stats *out) {
    if (!s || !out) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    *out = s->last_stats;
    return PSY_OK;
}

psy_status psy_debug_sobol_samples(psy_context *ctx, uint32_t size, const uint32_t *queries, uint32_t count,
                                   float *out_samples, uint32_t *out_indices) {
    if (!ctx || !queries || !out_samples || !out_indices) return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    if (!sobol_size_valid(size)) return fail(PSY_ERROR_INVALID_ARGUMENT, "invalid Sobol sequence size");
    if (count == 0u) return PSY_OK;
    PSY_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    std::vector<float> table(size_t(size) * 256u * 4u);
    psy_sobol_generate_table(size, table.data());
    DeviceBuffer dt_, dq, ds, di;
    PSY_CUDA_TRY(dt_.upload(table, st));
    std::vector<uint32_t> q(queries, queries + 5ull * count);
    PSY_CUDA_TRY(dq.upload(q, st));
    PSY_CUDA_TRY(ds.alloc(sizeof(float4) * count));
    PSY_CUDA_TRY(di.alloc(sizeof(uint32_t) * count));
    psy::launch_debug_sobol(st, dt_.as<float4>(), size, dq.as<uint32_t>(), count, ds.as<float4>(), di.as<uint32_t>());
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaMemcpyAsync(out_samples, ds.ptr, sizeof(float4) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(out_indices, di.ptr, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    return PSY_OK;
}

psy_status psy_debug_light_tree(psy_scene *scene, const float *queries, const uint32_t *pdf_emitters, uint32_t count,
                                uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf) {
    if (!scene || !queries || !pdf_emitters || !out_emitters || !out_sample_pdf || !out_reverse_pdf)
        return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    const psy_status built = ensure_light_tree(scene);
    if (built != PSY_OK) return built;
    if (scene->view.lt_node_count == 0u || scene->view.lt_emitter_count == 0u)
        return fail(PSY_ERROR_UNSUPPORTED, "scene has no usable light tree");
    if (count == 0u) return PSY_OK;
    PSY_CUDA_TRY(cudaSetDevice(scene->context->device));
    cudaStream_t st = scene->context->stream;
    DeviceBuffer dq, de, ds, dsp, drp;
    std::vector<float> q(queries, queries + 8ull * count);
    std::vector<uint32_t> e(pdf_emitters, pdf_emitters + count);
    PSY_CUDA_TRY(dq.upload(q, st));
    PSY_CUDA_TRY(de.upload(e, st));
    PSY_CUDA_TRY(ds.alloc(sizeof(uint32_t) * count));
    PSY_CUDA_TRY(dsp.alloc(sizeof(float) * count));
    PSY_CUDA_TRY(drp.alloc(sizeof(float) * count));
    psy::launch_debug_light_tree(st, scene->view, dq.as<float4>(), de.as<uint32_t>(), count, ds.as<uint32_t>(),
                                 dsp.as<float>(), drp.as<float>());
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaMemcpyAsync(out_emitters, ds.ptr, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(out_sample_pdf, dsp.ptr, sizeof(float) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(out_reverse_pdf, drp.ptr, sizeof(float) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    return PSY_OK;
}

psy_status psy_debug_light_distribution(psy_scene *scene, const float *u, uint32_t count, uint32_t *out_kind,
                                        uint32_t *out_index, float *out_pdf) {
    if (!scene || (count > 0u && (!u || !out_kind || !out_index || !out_pdf)))
        return fail(PSY_ERROR_INVALID_ARGUMENT, "null argument");
    if (count == 0u) return PSY_OK;
    PSY_CUDA_TRY(cudaSetDevice(scene->context->device));
    cudaStream_t st = scene->context->stream;
    DeviceBuffer du, dk, di, dp;
    std::vector<float> uh(u, u + count);
    PSY_CUDA_TRY(du.upload(uh, st));
    PSY_CUDA_TRY(dk.alloc(sizeof(uint32_t) * count));
    PSY_CUDA_TRY(di.alloc(sizeof(uint32_t) * count));
    PSY_CUDA_TRY(dp.alloc(sizeof(float) * count));
    psy::launch_debug_light_distribution(st, scene->view, du.as<float>(), count, dk.as<uint32_t>(),
                                         di.as<uint32_t>(), dp.as<float>());
    PSY_CUDA_TRY(cudaGetLastError());
    PSY_CUDA_TRY(cudaMemcpyAsync(out_kind, dk.ptr, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(out_index, di.ptr, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaMemcpyAsync(out_pdf, dp.ptr, sizeof(float) * count, cudaMemcpyDeviceToHost, st));
    PSY_CUDA_TRY(cudaStreamSynchronize(st));
    return PSY_OK;
}

}  // extern "C"
