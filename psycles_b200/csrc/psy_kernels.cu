// Wavefront path-trace kernels for sm_100a.
//
// One render batch holds P window pixels x S samples = N paths whose state
// lives in HBM as structure-of-arrays (PathBuffers).  Per path step:
//   k_intersect  closest hit of every queued path (two-level BVH)
//   k_shade      background / emission + forward MIS / roulette / AOV /
//                NEE sample + BSDF evaluation (writes one shadow ray) /
//                closure sample + path-state transition; survivors are
//                compacted into the next queue with warp-aggregated atomics
//   k_shadow     transmittance of the queued shadow rays, adds NEE radiance
// and after the last step k_film adds each path's sample into the film in
// sample order.  The kernels reproduce the Psycles Luisa megakernel
// (src/luisa/path_kernel_pipeline.cpp:73-183) path by path: the queue order
// never changes a path's result.
#include "psy_device.cuh"
#include "psy_kernels.h"

#include <algorithm>
#include "psy_light_tree.cuh"

namespace psy {

// Warp-aggregated queue append: one atomic per warp, slots in lane order.
// Every lane of the warp must call it (the callers' loops are warp-uniform).
__device__ __forceinline__ uint32_t warp_push(uint32_t *counter, bool pred) {
    const unsigned ballot = __ballot_sync(0xffffffffu, pred);
    const int lane = threadIdx.x & 31;
    uint32_t base = 0u;
    if (lane == 0 && ballot != 0u) base = atomicAdd(counter, uint32_t(__popc(ballot)));
    base = __shfl_sync(0xffffffffu, base, 0);
    return base + uint32_t(__popc(ballot & ((1u << lane) - 1u)));
}

__device__ __forceinline__ Xform xform12(const float *m) { return {ld3(m), ld3(m + 3), ld3(m + 6), ld3(m + 9)}; }

__device__ __forceinline__ void add3(float *d, f3 v) {
    d[0] += v.x;
    d[1] += v.y;
    d[2] += v.z;
}
__device__ __forceinline__ void set3(float *d, f3 v) {
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
}

// ------------------------------------------------------------------ raygen
// begin_path_sample / construct_camera_ray (src/luisa/path_kernel_setup.cpp:485-700,
// src/luisa/path_tracer_camera.cpp:10-246).
// sample_regular_polygon / sample_aperture (include/psycles/luisa/camera_sampling.h:
// 118-152): a corner triangle of the blade polygon, sampled by area.
__device__ __forceinline__ f2 sample_aperture(f2 r, uint32_t blades, float rotation) {
    if (blades == 0u) return sample_uniform_disk(r);
    const float corners = static_cast<float>(blades);
    float u = r.x, v = r.y;
    const float corner = floorf(u * corners);
    u = u * corners - corner;
    u = sqrtf(u);
    v *= u;
    u = 1.0f - u;
    const float half_corner = kPi / corners;
    const f2 point = mk2((u + v) * cos_(half_corner), (u - v) * sin_(half_corner));
    const float angle = rotation + corner * (2.0f * half_corner);
    const float c = cos_(angle), s = sin_(angle);
    return mk2(c * point.x - s * point.y, s * point.x + c * point.y);
}

// construct_camera_ray (src/luisa/path_tracer_camera.cpp:51-246): the camera-space
// ray of the projection (screen coordinates sx, sy in [-1, 1] plus lens
// shift), then the thin-lens update for depth of field.  `clip_cos` is the
// pinhole direction's cosine that scales the clipping range.
__device__ __forceinline__ void camera_local_ray(const RenderParams &p, float sx, float sy, f2 lens_sample, f3 &origin,
                                                 f3 &direction, float &clip_cos) {
    origin = mk3(0.0f);
    direction = mk3(0.0f, 0.0f, -1.0f);
    clip_cos = 1.0f;
    if (p.projection == PSY_CAMERA_PERSPECTIVE) {
        direction = normalize(mk3(sx * p.htan, sy * p.vtan, -1.0f));
        clip_cos = -direction.z;
    } else if (p.projection == PSY_CAMERA_ORTHOGRAPHIC) {
        const float aspect = static_cast<float>(p.full_w) / static_cast<float>(p.full_h);
        origin = mk3(sx * p.ortho_span * aspect * 0.5f, sy * p.ortho_span * 0.5f, 0.0f);
    } else {
        const float longitude = sx * kPi;
        const float latitude = sy * kPi * 0.5f;
        const float cos_lat = cos_(latitude);
        direction = mk3(cos_lat * sin_(longitude), sin_(latitude), -cos_lat * cos_(longitude));
    }
    if (p.depth_of_field) {
        f2 lens = sample_aperture(lens_sample, p.aperture_blades, p.aperture_rotation) * p.aperture_radius;
        lens.x /= maxf_(p.aperture_ratio, 1.0e-5f);
        const float focus_scale = p.focal_distance / maxf_(-direction.z, 1.0e-6f);
        const f3 focus = direction * focus_scale;
        origin = mk3(lens.x, lens.y, 0.0f);
        direction = normalize(focus - origin);
    }
}

__device__ __forceinline__ void raygen_path(const RenderParams &p, const PathBuffers &b, uint32_t i, uint32_t local,
                                            uint32_t sample, uint32_t trace_path, psy_path_trace *trace) {
    const uint32_t x = p.win_x + local % p.win_w;
    const uint32_t y = p.win_y + local / p.win_w;
    const uint32_t cycles_y = p.full_h - 1u - y;
    const uint32_t rng_hash = pixel_hash(x, cycles_y, p.seed);
    const float4 fs = sample_4d(p, sample, rng_hash, 0u);
    const f2 filter = sample == 0u ? mk2(0.5f, 0.5f) : mk2(fs.x, fs.y);
    const float jx = pixel_filter_sample(p.filter, filter.x);
    const float jy = 1.0f - pixel_filter_sample(p.filter, filter.y);
    const float W = static_cast<float>(p.full_w), H = static_cast<float>(p.full_h);
    const float sx = 2.0f * (static_cast<float>(x) + jx) / W - 1.0f + 2.0f * p.shift_x;
    const float sy = 1.0f - 2.0f * (static_cast<float>(y) + jy) / H + 2.0f * p.shift_y;
    f3 local_origin, local_dir;
    float clip_cos;
    f2 lens_sample = mk2(0.0f, 0.0f);
    if (p.depth_of_field) {
        // sample_3d at camera_lens_time_dimension, lens = .yz (path_tracer_camera.cpp:35-45)
        const float4 lt = sample_4d(p, sample, rng_hash, 1u);
        lens_sample = mk2(lt.y, lt.z);
    }
    camera_local_ray(p, sx, sy, lens_sample, local_origin, local_dir, clip_cos);
    const Xform cam = xform12(p.cam);
    f3 origin = xform_point(cam, local_origin);
    const f3 dir = safe_normalize(xform_direction(cam, local_dir), mk3(0.0f, 0.0f, -1.0f));
    const float safe_cos = maxf_(fabsf(clip_cos), 1.0e-20f);
    const float near_t = p.near_clip / safe_cos;
    const float far_t = (p.far_clip - p.near_clip) / safe_cos;
    origin = origin + dir * near_t;
    store_pair(b.ray_o, i, make_float4(origin.x, origin.y, origin.z, 0.0f), make_float4(dir.x, dir.y, dir.z, far_t));
    store_pair(b.tp, i, make_float4(1.0f, 1.0f, 1.0f, 0.0f), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    // initial_state (include/psycles/luisa/cycles_path_state.h:187-199)
    store_pair(b.st, i, make_uint4(128u | 512u, 1u, 16u, 0u), make_uint4(kSt2Delta, kInvalid, kInvalid, local));
    b.sample[i] = sample;
    b.aov_n[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b.aov_a[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b.mis_n[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b.queue_in[i] = i;
    if (i == trace_path && trace) {
        trace->pixel_x = x;
        trace->pixel_y = y;
        trace->sample = sample;
        trace->rng_hash = rng_hash;
        trace->filter[0] = filter.x;
        trace->filter[1] = filter.y;
        set3(trace->ray_origin, origin);
        set3(trace->ray_direction, dir);
        trace->valid = 1u;
        trace->event_count = 0u;
    }
}

__global__ void k_raygen(RenderParams p, PathBuffers b, uint32_t pixels, uint32_t paths, uint32_t sample_base,
                         uint32_t trace_path, psy_path_trace *trace) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < paths; i += gridDim.x * blockDim.x)
        raygen_path(p, b, i, i % pixels, sample_base + i / pixels, trace_path, trace);
}

// The item of a batched wavefront that holds `index` (items sorted by the
// field `begin` selects).
template <typename Begin>
__device__ __forceinline__ uint32_t find_item(const BatchItem *items, uint32_t n, uint32_t index, Begin begin) {
    uint32_t lo = 0u, hi = n;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (begin(items[mid]) <= index) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Camera rays of every item of a batched wavefront; records each path's job.
// The wavefront's shape comes from device memory (round[0] paths, round[2]
// items) so one captured launch serves every wavefront.
__global__ void k_raygen_batch(const JobGpu *jobs, const BatchItem *items, const uint32_t *round, PathBuffers b) {
    const uint32_t paths = round[0], item_count = round[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < paths; i += gridDim.x * blockDim.x) {
        const BatchItem it = items[find_item(items, item_count, i, [](const BatchItem &t) { return t.path_begin; })];
        const uint32_t r = i - it.path_begin;
        b.job[i] = it.job;
        raygen_path(jobs[it.job].p, b, i, r % it.pixels, it.sample_base + r / it.pixels, kInvalid, nullptr);
    }
}

// --------------------------------------------------------------- intersect
// Cycles ray visibility of a path: contract_visibility (cycles_path_state.h:449-491).
__device__ __forceinline__ uint32_t contract_visibility(uint32_t v) {
    const uint32_t tv = (v & 2u) ? (v & ~(4u | 8u)) : v;
    uint32_t r = 0u;
    if (tv & 1u) r |= PSY_VISIBILITY_CAMERA;
    if (tv & 2u) r |= PSY_VISIBILITY_TRANSMISSION;
    if (tv & 4u) r |= PSY_VISIBILITY_DIFFUSE;
    if (tv & 8u) r |= PSY_VISIBILITY_GLOSSY;
    if (tv & 16u) r |= PSY_VISIBILITY_VOLUME_SCATTER;
    return r;
}

// Persistent closest-hit kernel: each lane owns one ray at a time and, when
// it finishes, the warp refills its idle lanes from a global fetch counter
// (one atomic per warp), so lanes do not wait for the warp's longest ray.
#ifndef PSY_TRAVERSAL_BUDGET
#define PSY_TRAVERSAL_BUDGET 24
#endif
#ifndef PSY_INTERSECT_MIN_BLOCKS
#define PSY_INTERSECT_MIN_BLOCKS 6
#endif
#ifndef PSY_SHADE_MIN_BLOCKS
#define PSY_SHADE_MIN_BLOCKS 3
#endif
#ifndef PSY_SHADOW_MIN_BLOCKS
#define PSY_SHADOW_MIN_BLOCKS 4
#endif
// Nodes a lane advances between refills of idle lanes.
constexpr int kTraversalBudget = PSY_TRAVERSAL_BUDGET;
constexpr uint32_t kFullMask = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Hands the next queue slot below `count` to every lane with `need`, or
// kInvalid.  Warp-uniform: every lane calls it, and `exhausted` (uniform
// across the warp) stops further atomics once the queue is used up.
__device__ __forceinline__ uint32_t warp_fetch(uint32_t *fetch_counter, uint32_t count, bool need, bool &exhausted) {
    if (exhausted) return kInvalid;
    const unsigned mask = __ballot_sync(kFullMask, need);
    if (mask == 0u) return kInvalid;
    uint32_t base = 0u;
    if (lane_id() == 0u) base = atomicAdd(fetch_counter, uint32_t(__popc(mask)));
    base = __shfl_sync(kFullMask, base, 0);
    if (base + uint32_t(__popc(mask)) >= count) exhausted = true;
    if (!need) return kInvalid;
    const uint32_t q = base + uint32_t(__popc(mask & ((1u << lane_id()) - 1u)));
    return q < count ? q : kInvalid;
}

// kMulti: paths of a batched wavefront, each traced in its job's scene.
template <bool kMulti>
__global__ void __launch_bounds__(128, PSY_INTERSECT_MIN_BLOCKS)
    k_intersect(const __grid_constant__ SceneView s_arg, const __grid_constant__ PathBuffers b, const JobGpu *jobs,
                uint32_t sort_threshold) {
    const uint32_t count = b.counters[0];
    const bool sorted = sort_threshold != 0u && count >= sort_threshold;
    TraversalState t;
    Hit best;
    bool has = false, active = false, exhausted = false;
    uint32_t path = 0u, job = 0u;
    for (;;) {
        const uint32_t q = warp_fetch(&b.counters[3], count, !active, exhausted);
        if (q != kInvalid) {
            path = sorted ? b.queue_sorted[q] : b.queue_in[q];
            if (kMulti) job = b.job[path];
        }
        const SceneView &s = kMulti ? jobs[job].s : s_arg;
        if (q != kInvalid) {
            float4 o, d;
            uint4 st, st2;
            load_pair(b.ray_o, path, o, d);
            load_pair(b.st, path, st, st2);
            const uint32_t vis = st.y;
            const Ray ray{mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), o.w, d.w};
            traversal_begin(t, s, ray, contract_visibility(vis), st2.y, st2.z, kInvalid, kInvalid);
            has = false;
            best.t = ray.tmax;
            best.u = best.v = 0.0f;
            best.instance = best.prim = best.object = best.cycles_prim = kInvalid;
            active = true;
        }
        if (!__any_sync(kFullMask, active)) break;
        if (active) {
            const bool done = traversal_steps(t, s, kTraversalBudget,
                                              [&](uint32_t ii, uint32_t local, uint32_t cp, float th, float u, float v) {
                const bool later = ii > best.object || (ii == best.object && cp > best.cycles_prim);
                if (has && !(th < best.t || (th == best.t && later))) return false;
                has = true;
                best.t = th;
                best.u = u;
                best.v = v;
                best.instance = ii;
                best.prim = local;
                best.object = ii;
                best.cycles_prim = cp;
                t.tmax = th;
                return false;
            });
            if (done) {
                store_pair(b.hit, path, make_float4(best.t, best.u, best.v, __uint_as_float(best.instance)),
                           make_uint4(has ? best.prim : kInvalid, 0u, 0u, 0u));
                active = false;
            }
        }
    }
}

// ------------------------------------------------------------------- shade

__device__ __forceinline__ float power_heuristic(float a, float c) {
    const float a2 = a * a, c2 = c * c;
    return a2 / maxf_(a2 + c2, 1.0e-20f);
}

// forward_light_weight / nee_light_weight (src/luisa/path_tracer_lighting.cpp:35-72)
// for the effective direct-light mode.
__device__ __forceinline__ float forward_light_weight(uint32_t mode, float forward_pdf, float nee_pdf, bool competing,
                                                      bool nee_available) {
    if (mode == PSY_DIRECT_LIGHT_FORWARD) return 1.0f;
    if (mode == PSY_DIRECT_LIGHT_NEE) return (competing && nee_available) ? 0.0f : 1.0f;
    return (competing && nee_available) ? power_heuristic(forward_pdf, nee_pdf) : 1.0f;
}
__device__ __forceinline__ float nee_light_weight(uint32_t mode, float nee_pdf, float forward_pdf) {
    if (mode == PSY_DIRECT_LIGHT_NEE) return 1.0f;
    if (mode == PSY_DIRECT_LIGHT_FORWARD) return forward_pdf <= 0.0f ? 1.0f : 0.0f;
    return power_heuristic(nee_pdf, forward_pdf);
}

// film_clamp_light (include/psycles/luisa/cycles_film_light.h:15-49).
__device__ __forceinline__ f3 clamp_contribution(f3 c, uint32_t depth, const RenderParams &p) {
    c = mk3(isfinite(c.x) ? c.x : 0.0f, isfinite(c.y) ? c.y : 0.0f, isfinite(c.z) ? c.z : 0.0f);
    const float limit = depth > 0u ? p.clamp_indirect : p.clamp_direct;
    const float mag = fabsf(c.x) + fabsf(c.y) + fabsf(c.z);
    if (limit > 0.0f && mag > limit) return c * (limit / maxf_(mag, 1.0e-20f));
    return c;
}

__device__ __forceinline__ float light_roulette_weight(f3 unshadowed, float random, float inv_threshold) {
    const float m = max_abs_component(unshadowed);
    const float pr = m * inv_threshold;
    const bool roulette = inv_threshold > 0.0f && pr < 1.0f;
    const bool survives = !roulette || random < pr;
    const float inv_p = roulette ? 1.0f / maxf_(pr, 1.0e-20f) : 1.0f;
    return survives ? inv_p : 0.0f;
}

constexpr uint32_t kFlagReflect = 1u, kFlagSingular = 2u, kFlagTransparent = 4u, kFlagImportanceBake = 8u,
                   kFlagDiffuseAncestor = 16u, kFlagMisHadTransmission = 64u, kFlagMisSkip = 128u,
                   kFlagSinglePassDone = 256u, kFlagTransparentBackground = 512u,
                   kFlagTerminateOnNextSurface = 1024u, kFlagTerminateAfterTransparent = 4096u,
                   kFlagSurfacePass = 1u << 18u, kFlagVolumePass = 1u << 19u;

struct PathState {
    uint32_t flag, visibility, bounce, diffuse_bounce, glossy_bounce, transmission_bounce, transparent_bounce,
        rng_offset;
};

// cycles_path_state::next_surface (include/psycles/luisa/cycles_path_state.h:205-338).
__device__ __forceinline__ PathState next_surface(const PathState &before, uint32_t label, uint32_t runtime,
                                                  const RenderParams &p) {
    if ((label & (kLabelTransparent | 512u)) != 0u) {
        PathState t = before;
        t.transparent_bounce += 1u;
        t.rng_offset += 16u;
        t.flag |= kFlagTransparent;
        if (t.transparent_bounce >= p.transparent_max) t.flag |= kFlagTerminateOnNextSurface;
        if ((runtime & 4096u) != 0u) t.flag |= kFlagMisSkip;
        return t;
    }
    PathState s = before;
    s.bounce += 1u;
    s.rng_offset += 16u;
    if (s.bounce >= p.maximum) s.flag |= kFlagTerminateAfterTransparent;
    s.visibility = 0u;
    s.flag &= ~(kFlagReflect | kFlagSingular | kFlagTransparent | kFlagImportanceBake | kFlagMisSkip |
                kFlagMisHadTransmission);
    const bool reflection = (label & kLabelReflect) != 0u;
    const bool diffuse = (label & kLabelDiffuse) != 0u;
    const bool glossy = (label & kLabelGlossy) != 0u;
    const bool transmit_transparent = (label & 128u) != 0u;
    if (reflection) s.flag |= kFlagReflect;
    if (reflection || !transmit_transparent) s.flag &= ~kFlagTransparentBackground;
    const bool diffuse_reflection = reflection && diffuse;
    const bool glossy_reflection = reflection && !diffuse;
    const bool transmission = !reflection;
    if (diffuse_reflection) s.diffuse_bounce += 1u;
    if (glossy_reflection) s.glossy_bounce += 1u;
    if (transmission) s.transmission_bounce += 1u;
    if (diffuse_reflection && s.diffuse_bounce >= p.max_diffuse) s.flag |= kFlagTerminateAfterTransparent;
    if (glossy_reflection && s.glossy_bounce >= p.max_glossy) s.flag |= kFlagTerminateAfterTransparent;
    if (transmission && s.transmission_bounce >= p.max_transmission) s.flag |= kFlagTerminateAfterTransparent;
    if (transmission) s.visibility |= 2u;
    s.visibility |= diffuse ? 4u : 8u;
    if (diffuse) s.flag |= kFlagDiffuseAncestor;
    if (!diffuse && !glossy) s.flag |= kFlagSingular | kFlagMisSkip;
    if ((runtime & kRuntimeBsdfHasTransmission) != 0u) s.flag |= kFlagMisHadTransmission;
    if ((s.flag & (kFlagSurfacePass | kFlagVolumePass)) == 0u && (s.flag & kFlagTransparentBackground) == 0u)
        s.flag |= kFlagSurfacePass;
    return s;
}

__device__ __forceinline__ PathState unpack_state(uint4 st, uint4 st2) {
    return {st.x, st.y, st.w & 0xffu, (st.w >> 8) & 0xffu, (st.w >> 16) & 0xffu, st.w >> 24, st2.x & 0xffu, st.z};
}

__device__ __forceinline__ float next_float_up(float t) {
    return t == 0.0f ? 1.17549435e-38f : __uint_as_float(__float_as_uint(t) + 1u);
}

// ------------------------------------------------------ sort by material
__device__ __forceinline__ uint32_t surface_material(const SceneView &s, uint32_t instance, uint32_t local);

// The kind of lamp a path's next-event sample will take under the flat
// light distribution, estimated from the same random number the shading
// kernel draws (the lamps share the distribution's tail equally): 1
// emissive triangle, 2 sun, 3 / 4 rectangle / ellipse, 5 delta point or
// spot, 6 disk, 7 sphere; 0 without a flat-distribution pick.  Only the
// queue order depends on it, so an estimate at a bin edge costs
// coherence, never a result.
__device__ __forceinline__ uint32_t nee_kind_hint(const SceneView &s, const RenderParams &p, const PathBuffers &b,
                                                  uint32_t i) {
    if (p.use_light_tree || !p.nee || s.emitter_count == 0u) return 0u;
    uint4 st, st2;
    load_pair(b.st, i, st, st2);
    const uint32_t local = st2.w;
    const uint32_t x = p.win_x + local % p.win_w, y = p.win_y + local / p.win_w;
    const uint32_t rng_hash = pixel_hash(x, p.full_h - 1u - y, p.seed);
    const float u = sample_4d(p, b.sample[i], rng_hash, st.z + 1u).z;
    const uint32_t tri_n = s.triangle_emitters, light_n = s.light_count;
    const float c0 = tri_n > 0u ? s.distribution[tri_n].cumulative : 0.0f;
    if (light_n == 0u || u < c0) return 1u;
    const uint32_t li = min(uint32_t((u - c0) / fmaxf(1.0f - c0, 1.0e-20f) * float(light_n)), light_n - 1u);
    const psy_light_desc &l = s.lights[li];
    if (l.type == PSY_LIGHT_DISTANT) return 2u;
    if (l.type == PSY_LIGHT_AREA) return (l.flags & PSY_LIGHT_FLAG_ELLIPSE) != 0u ? 4u : 3u;
    if (!(l.radius > 0.0f)) return 5u;
    return (l.flags & PSY_LIGHT_FLAG_SPHERE) != 0u ? 7u : 6u;
}

// Queues of at least `threshold` paths are grouped before shading by
// material and by the kind of lamp the path's next-event sample takes, so
// a warp mostly runs one closure program and one light-sampling branch: a
// bucket per queue entry (misses in bucket 0, hits by material, lamp kind
// and job hashed into the other buckets), a histogram, its exclusive scan
// and a scatter.  Order inside a bucket is arbitrary; no path's result
// depends on the queue order.
template <bool kMulti>
__global__ void k_sort_count(const __grid_constant__ SceneView s_arg, const __grid_constant__ RenderParams p_arg,
                             const __grid_constant__ PathBuffers b, const JobGpu *jobs, uint32_t threshold) {
    __shared__ uint32_t local[kSortBuckets];
    const uint32_t count = b.counters[0];
    if (count < threshold) return;
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x) local[k] = 0u;
    __syncthreads();
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const uint32_t i = b.queue_in[q];
        float4 h4;
        uint4 hp4;
        load_pair(b.hit, i, h4, hp4);
        const uint32_t prim = hp4.x;
        uint32_t key = 0u;
        if (prim != kInvalid) {
            const uint32_t job = kMulti ? b.job[i] : 0u;
            const SceneView &s = kMulti ? jobs[job].s : s_arg;
            const RenderParams &p = kMulti ? jobs[job].p : p_arg;
            const uint32_t mat = surface_material(s, __float_as_uint(h4.w), prim);
            key = 1u + (mat * 8u + nee_kind_hint(s, p, b, i) + job * 977u) % (kSortBuckets - 1u);
        }
        b.sort_keys[q] = key;
        atomicAdd(&local[key], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x)
        if (local[k]) atomicAdd(&b.sort_hist[k], local[k]);
}

// One block of 1024 threads: offsets = exclusive scan of the histogram,
// which is cleared for the next sort.
// `counter`: 0 sorts the shading queue, 2 the shadow queue.
__global__ void k_sort_scan(const __grid_constant__ PathBuffers b, uint32_t threshold, uint32_t counter) {
    __shared__ uint32_t part[1024];
    if (b.counters[counter] < threshold) return;
    constexpr uint32_t kPer = kSortBuckets / 1024u;
    const uint32_t t = threadIdx.x;
    uint32_t v[kPer], sum = 0u;
    for (uint32_t k = 0; k < kPer; ++k) {
        v[k] = b.sort_hist[t * kPer + k];
        sum += v[k];
    }
    part[t] = sum;
    __syncthreads();
    for (uint32_t d = 1u; d < 1024u; d <<= 1) {  // inclusive Hillis-Steele scan
        const uint32_t add = t >= d ? part[t - d] : 0u;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (uint32_t k = 0; k < kPer; ++k) {
        b.sort_offsets[t * kPer + k] = run;
        run += v[k];
        b.sort_hist[t * kPer + k] = 0u;
    }
}

// Scatter in three passes over each block's contiguous chunk of the queue:
// ranks inside the block from warp-aggregated shared-memory atomics (stored
// beside the 11-bit bucket), one global reservation per non-empty bucket
// per block, then the writes.  Global atomics drop from one per path to one
// per bucket and block.
// The shading queue sorts its path indices; the shadow queue sorts its
// slot numbers (a permutation k_shadow reads its rays through).
__global__ void __launch_bounds__(256) k_sort_scatter(const __grid_constant__ PathBuffers b, uint32_t threshold,
                                                      uint32_t counter) {
    __shared__ uint32_t hist[kSortBuckets];
    const uint32_t count = b.counters[counter];
    if (count < threshold) return;
    const uint32_t chunk = (count + gridDim.x - 1u) / gridDim.x;
    const uint32_t begin = blockIdx.x * chunk;
    const uint32_t end = min(count, begin + chunk);
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x) hist[k] = 0u;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = begin; base < end; base += blockDim.x) {
        const uint32_t q = base + threadIdx.x;
        const bool live = q < end;
        const uint32_t key = live ? b.sort_keys[q] : kSortBuckets;  // sentinel outside the histogram
        const uint32_t peers = __match_any_sync(kFullMask, key);
        const uint32_t leader = __ffs(peers) - 1u;
        const uint32_t rank_in_warp = __popc(peers & ((1u << lane) - 1u));
        uint32_t first = 0u;
        if (live && lane == leader) first = atomicAdd(&hist[key], __popc(peers));
        first = __shfl_sync(peers, first, leader);
        if (live) b.sort_keys[q] = key | ((first + rank_in_warp) << 11);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x)
        if (hist[k]) hist[k] = atomicAdd(&b.sort_offsets[k], hist[k]);
    __syncthreads();
    for (uint32_t q = begin + threadIdx.x; q < end; q += blockDim.x) {
        const uint32_t packed = b.sort_keys[q];
        b.queue_sorted[hist[packed & (kSortBuckets - 1u)] + (packed >> 11)] = counter == 0u ? b.queue_in[q] : q;
    }
}

// Closest-hit rays grouped by where they start and where they head: the
// direction octant and an 8 x 8 x 4 cell of the scene's bounds around the
// origin, so a warp's rays walk the same part of the BVH.  Rays of a
// batched wavefront are grouped per job as well.
template <bool kMulti>
__global__ void k_sort_count_rays(const __grid_constant__ SceneView s_arg, const __grid_constant__ PathBuffers b,
                                  const JobGpu *jobs, uint32_t threshold) {
    __shared__ uint32_t local[kSortBuckets];
    const uint32_t count = b.counters[0];
    if (count < threshold) return;
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x) local[k] = 0u;
    __syncthreads();
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const uint32_t i = b.queue_in[q];
        const uint32_t job = kMulti ? b.job[i] : 0u;
        const SceneView &s = kMulti ? jobs[job].s : s_arg;
        float4 o, d;
        load_pair(b.ray_o, i, o, d);
        auto cell = [](float v, float lo, float hi, float n) {
            const float f = hi > lo ? (v - lo) / (hi - lo) : 0.0f;
            return uint32_t(fminf(fmaxf(f * n, 0.0f), n - 1.0f));
        };
        const uint32_t cx = cell(o.x, s.world_lo.x, s.world_hi.x, 8.0f);
        const uint32_t cy = cell(o.y, s.world_lo.y, s.world_hi.y, 8.0f);
        const uint32_t cz = cell(o.z, s.world_lo.z, s.world_hi.z, 4.0f);
        const uint32_t octant = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
        const uint32_t key = ((octant << 8 | cz << 6 | cy << 3 | cx) + job * 977u) & (kSortBuckets - 1u);
        b.sort_keys[q] = key;
        atomicAdd(&local[key], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x)
        if (local[k]) atomicAdd(&b.sort_hist[k], local[k]);
}

// Shadow rays grouped by direction (octahedral map of the direction into a
// 45 x 45 grid), so a warp's rays head the same way -- mostly towards the
// same light from nearby points.
__global__ void k_sort_count_shadow(const __grid_constant__ PathBuffers b, uint32_t threshold) {
    __shared__ uint32_t local[kSortBuckets];
    const uint32_t count = b.counters[2];
    if (count < threshold) return;
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x) local[k] = 0u;
    __syncthreads();
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const float4 d = b.sh_d[q];
        const float l1 = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
        float u = l1 > 0.0f ? d.x / l1 : 0.0f, v = l1 > 0.0f ? d.y / l1 : 0.0f;
        if (d.z < 0.0f) {
            const float uu = (1.0f - fabsf(v)) * (u >= 0.0f ? 1.0f : -1.0f);
            v = (1.0f - fabsf(u)) * (v >= 0.0f ? 1.0f : -1.0f);
            u = uu;
        }
        const uint32_t iu = min(44u, uint32_t(fmaxf(u * 0.5f + 0.5f, 0.0f) * 45.0f));
        const uint32_t iv = min(44u, uint32_t(fmaxf(v * 0.5f + 0.5f, 0.0f) * 45.0f));
        const uint32_t key = iv * 45u + iu;
        b.sort_keys[q] = key;
        atomicAdd(&local[key], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < kSortBuckets; k += blockDim.x)
        if (local[k]) atomicAdd(&b.sort_hist[k], local[k]);
}

// kTrace selects the variant that records the per-path trace; the render
// variant carries no trace code.
// kMulti: paths of a batched wavefront, each shaded with its job's scene and
// parameters.
template <bool kTrace, bool kMulti, bool kGlossy>
__global__ void __launch_bounds__(128, PSY_SHADE_MIN_BLOCKS)
    k_shade(const __grid_constant__ SceneView s_arg, const __grid_constant__ RenderParams p_arg,
            const __grid_constant__ PathBuffers b, uint32_t step, uint32_t trace_path, psy_path_trace *trace,
            const JobGpu *jobs, uint32_t sort_threshold) {
    // a batched wavefront launches both variants; the one that does not
    // match the wavefront's glossy flag (set by k_begin_round) returns
    if (kMulti && (b.counters[kCounterWaveGlossy] != 0u) != kGlossy) return;
    const uint32_t count = b.counters[0];
    const uint32_t *queue = (sort_threshold != 0u && count >= sort_threshold) ? b.queue_sorted : b.queue_in;
    const uint32_t rounds = (count + gridDim.x * blockDim.x - 1u) / (gridDim.x * blockDim.x);
    // Every lane runs the same number of rounds so the warp-aggregated queue
    // pushes see the whole warp.
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t q = r * gridDim.x * blockDim.x + blockIdx.x * blockDim.x + threadIdx.x;
        const bool active = q < count;
        bool keep = false;
        bool shadow = false;
        bool final = false;  // the path ends here (its radiance and shadow contribution go to rad_final)
        uint32_t i = 0u;
        float4 sh_o, sh_d, sh_c;
        uint4 sh_ids;
        if (active) {
            i = queue[q];
            const uint32_t job = kMulti ? b.job[i] : 0u;
            const SceneView &s = kMulti ? jobs[job].s : s_arg;
            const RenderParams &p = kMulti ? jobs[job].p : p_arg;
            psy_path_event *ev = nullptr;
            if (kTrace && trace && i == trace_path && step < PSY_TRACE_MAX_EVENTS) {
                ev = &trace->events[step];
                trace->event_count = step + 1u;
            }
            float4 ro, rd, tp4, rad4, h4;
            uint4 st, st2, hp4;
            load_pair(b.ray_o, i, ro, rd);
            load_pair(b.tp, i, tp4, rad4);
            load_pair(b.st, i, st, st2);
            load_pair(b.hit, i, h4, hp4);
            Ray ray{mk3(ro.x, ro.y, ro.z), mk3(rd.x, rd.y, rd.z), ro.w, rd.w};
            f3 throughput = mk3(tp4.x, tp4.y, tp4.z);
            float previous_bsdf_pdf = tp4.w;
            f3 radiance = mk3(rad4.x, rad4.y, rad4.z);
            float transparency = rad4.w;
            PathState ps = unpack_state(st, st2);
            bool previous_delta = (st2.x & kSt2Delta) != 0u;
            bool primary_recorded = (st2.x & kSt2Primary) != 0u;
            const bool terminate_on_next_surface = (st2.x & kSt2TermNext) != 0u;
            const bool terminate_after_transparent = (st2.x & kSt2TermAfter) != 0u;
            const uint32_t ray_visibility = contract_visibility(ps.visibility);
            const uint32_t sample = b.sample[i];
            const uint32_t local = st2.w;
            const uint32_t x = p.win_x + local % p.win_w;
            const uint32_t y = p.win_y + local / p.win_w;
            const uint32_t rng_hash = pixel_hash(x, p.full_h - 1u - y, p.seed);
            const float terminate_sample = sample_4d(p, sample, rng_hash, ps.rng_offset + 0u).x;
            const float4 ls4 = sample_4d(p, sample, rng_hash, ps.rng_offset + 1u);
            const f3 light_sample = mk3(ls4.x, ls4.y, ls4.z);
            const float light_terminate = sample_4d(p, sample, rng_hash, ps.rng_offset + 2u).x;
            const float4 bs4 = sample_4d(p, sample, rng_hash, ps.rng_offset + 3u);
            DistEntryGpu selected = p.use_light_tree ? DistEntryGpu{0.0f, 0.0f, 3u, 0u}
                                                     : distribution_sample(s, light_sample.z);
            const uint32_t prim = hp4.x;
            if (ev) {
                ev->rng_offset = ps.rng_offset;
                ev->random_terminate = terminate_sample;
                set3(ev->random_light, light_sample);
                ev->random_light_terminate = light_terminate;
                set3(ev->random_bsdf, mk3(bs4.x, bs4.y, bs4.z));
                ev->light_kind = selected.kind;
                ev->light_index = selected.index;
                const bool missed = prim == kInvalid;
                ev->hit_t = missed ? 0.0f : h4.x;
                ev->hit_u = missed ? 0.0f : h4.y;
                ev->hit_v = missed ? 0.0f : h4.z;
                ev->closure_index = kInvalid;
                ev->hit_object = kInvalid;
                ev->hit_primitive = kInvalid;
            }
            const uint32_t depth = ps.bounce;
            bool alive = true;
            if (s.lamp_count > 0u) {
                // Lamps in front of the mesh event are transparent events that
                // add their emission without a new bounce or new dimensions
                // (src/luisa/path_kernel_pipeline.cpp:78-126,
                // src/luisa/path_kernel_forward_light.cpp:14-118).
                const float event_distance = prim == kInvalid ? ray.tmax : h4.x;
                uint32_t excluded = kInvalid;
                float tmin = ray.tmin;
                for (uint32_t guard = 0; guard <= s.lamp_count && alive; ++guard) {
                    const float4 mn = b.mis_n[i];
                    const LampHit lh = closest_lamp(s, ray.o, ray.d, tmin, event_distance, ray_visibility, excluded,
                                                    mk3(mn.x, mn.y, mn.z), (ps.flag & kFlagMisHadTransmission) != 0u);
                    if (!lh.valid) break;
                    float selection_pdf = s.light_selection_pdf;
                    if (p.use_light_tree)
                        selection_pdf = lt_pdf(s, s.triangle_emitters + lh.index, ray.o, mk3(mn.x, mn.y, mn.z),
                                               (ps.flag & kFlagMisHadTransmission) != 0u);
                    const float light_pdf = lh.pdf * selection_pdf;
                    const bool competing = depth > 0u && !previous_delta;
                    const float w = forward_light_weight(p.direct_mode, previous_bsdf_pdf, light_pdf, competing,
                                                         light_pdf > 0.0f);
                    const psy_light_desc &l = s.lights[lh.index];
                    const f3 lr = ld3(l.color) * (l.power * lh.eval_factor);
                    const f3 c = clamp_contribution(throughput * lr * w, depth, p);
                    radiance = radiance + c;
                    if (ev) add3(ev->emission, c);
                    ps.transparent_bounce += 1u;
                    tmin = next_float_up(lh.distance);
                    excluded = lh.index;
                    if (ps.transparent_bounce >= p.transparent_max) {
                        alive = false;
                        if (ev) ev->terminated = 1u;
                    }
                }
            }
            if (!alive) {
                // a lamp event used up the transparent budget
            } else if (prim == kInvalid) {
                // BackgroundEventStage (src/luisa/path_kernel_background_event.cpp:14-160)
                const f3 bg = ld3(s.background);
                const f3 c = clamp_contribution(throughput * bg * 1.0f, depth, p);
                const bool world_visible = (s.world_visibility & ray_visibility) != 0u;
                const bool transparent_bg = p.transparent_background != 0u && (ps.flag & kFlagTransparentBackground) != 0u;
                if (transparent_bg) {
                    transparency += (throughput.x + throughput.y + throughput.z) * (1.0f / 3.0f);
                } else if (world_visible) {
                    radiance = radiance + c;
                    if (ev) add3(ev->emission, c);
                }
                if (ev) ev->terminated = 1u;
                alive = false;
            } else {
                Hit h;
                h.t = h4.x;
                h.u = h4.y;
                h.v = h4.z;
                h.instance = __float_as_uint(h4.w);
                h.prim = prim;
                h.object = h.instance;
                h.cycles_prim = s.meshes[s.instances[h.instance].mesh].prim_offset + prim;
                if (ev) {
                    ev->hit_object = h.object;
                    ev->hit_primitive = h.cycles_prim;
                }
                const SurfacePoint sp = surface_point(s, h, ray.d);
                const MaterialGpu mat = s.materials[sp.material];
                SurfaceClosures<kGlossy> closures;
                const ClosurePoint cpt{sp.n, sp.ng, -ray.d, safe_normalize(-ray.d, sp.n), mat.bump_correction != 0u,
                                       sp.back_facing};
                collect_surface<kGlossy>(s, mat, cpt, closures);
                // SurfaceShadingStageImpl::emit (src/luisa/path_kernel_surface_shading.cpp:117-250)
                float emission_weight = 1.0f;
                if (p.nee && s.triangle_emitters > 0u && mat.emission_sampling != 0u && mat.has_emission) {
                    const bool competing = depth > 0u && !previous_delta;
                    float selection_pdf =
                        0.5f * length(cross(sp.wp1 - sp.wp0, sp.wp2 - sp.wp0)) * s.triangle_area_pdf;
                    if (p.use_light_tree) {
                        // light_tree.forward_pdf (src/luisa/path_tracer_light_tree.cpp:799-838)
                        const float4 mn = b.mis_n[i];
                        selection_pdf = lt_pdf(s, lt_triangle_emitter(s, sp.object, sp.cycles_prim), ray.o,
                                               mk3(mn.x, mn.y, mn.z), (ps.flag & kFlagMisHadTransmission) != 0u);
                    }
                    const float light_pdf = emissive_forward_pdf(selection_pdf, mat.emission_sampling, ray.o,
                                                                 sp.position, sp.wp0, sp.wp1, sp.wp2,
                                                                 // the geometric normal before the back-face
                                                                 // flip (path_kernel_surface_shading.cpp:130-134)
                                                                 sp.back_facing ? -sp.ng : sp.ng);
                    const bool available = light_pdf > 0.0f;
                    emission_weight = forward_light_weight(p.direct_mode, previous_bsdf_pdf, light_pdf, competing, available);
                }
                const f3 ec = clamp_contribution(throughput * closures.emission * emission_weight, depth, p);
                radiance = radiance + ec;
                if (ev) add3(ev->emission, ec);
                if (terminate_on_next_surface) {
                    alive = false;
                    if (ev) ev->terminated = 1u;
                }
                if (alive) {
                    // continuation_probability (cycles_path_state.h:413-447)
                    const bool tr_state = (ps.flag & kFlagTransparent) != 0u;
                    const bool before_min = tr_state ? ps.transparent_bounce <= p.transparent_min : ps.bounce <= p.minimum;
                    const float cp = before_min ? 1.0f : minf_(sqrtf(max_abs_component(throughput)), 1.0f);
                    if (ev) ev->continuation_probability = cp;
                    if (cp <= 0.0f) {
                        alive = false;
                    } else if (cp != 1.0f) {
                        if (terminate_sample >= cp) alive = false;
                        else throughput = throughput / cp;
                    }
                    if (!alive && ev) ev->terminated = 1u;
                }
                if (alive) {
                    if (depth == 0u) {
                        f3 aov_albedo, aov_normal, aov_transparency;
                        surface_aov<kGlossy>(closures, cpt, aov_albedo, aov_normal, aov_transparency);
                        const float4 a4 = b.aov_a[i];
                        const f3 acc = mk3(a4.x, a4.y, a4.z) + throughput * aov_albedo;
                        b.aov_a[i] = make_float4(acc.x, acc.y, acc.z, 0.0f);
                        const f3 alpha = clamp3(mk3(1.0f) - aov_transparency, 0.0f, 1.0f);
                        const float average_alpha = (alpha.x + alpha.y + alpha.z) * (1.0f / 3.0f);
                        const bool writes_normal = !primary_recorded && (p.pass_alpha_threshold == 0.0f ||
                                                                         average_alpha >= p.pass_alpha_threshold);
                        if (writes_normal) {
                            b.aov_n[i] = make_float4(aov_normal.x, aov_normal.y, aov_normal.z, 0.0f);
                            primary_recorded = true;
                            ps.flag |= kFlagSinglePassDone;
                        }
                    }
                    const uint32_t runtime = runtime_flags(closures, sp.back_facing);
                    if (p.use_light_tree) {
                        // light-tree pick after shading (src/luisa/path_kernel_pipeline.cpp:150-159)
                        selected = lt_sample(s, light_sample.z, sp.position, sp.n,
                                             (runtime & kRuntimeBsdfHasTransmission) != 0u);
                        if (ev) {
                            ev->light_kind = selected.kind;
                            ev->light_index = selected.index;
                        }
                    }
                    const uint32_t lobe_mask = terminate_after_transparent ? kEventTransparent : 0xffffffffu;
                    const InstanceGpu &inst = s.instances[sp.instance];
                    // Direct lighting (src/luisa/path_kernel_pipeline.cpp:160-172)
                    if (p.nee && (runtime & kRuntimeBsdfHasEval) != 0u) {
                        f3 lp = mk3(0.0f), ldir = mk3(0.0f);
                        float ldist = 0.0f;
                        bool distant = false;
                        f3 surviving = mk3(0.0f);
                        uint32_t light_obj = kInvalid, light_prim = kInvalid;
                        bool emit = false;
                        // The light sample of either kind, then one BSDF
                        // evaluation, MIS weight and light roulette shared by
                        // both (a warp's lanes that picked triangles and lamps
                        // evaluate together).
                        bool sampled = false, weigh_mis = true;
                        f3 light_radiance = mk3(0.0f);
                        float light_pdf = 0.0f, pdf_divisor = 1.0f;
                        if (selected.kind == 0u) {
                            // EmissiveMeshLightingComponent (src/luisa/path_kernel_nee_emissive_mesh.cpp:32-296)
                            const EmitterGpu &em = s.emitters[selected.index];
                            const TriSample ls = sample_triangle(sp.position, ld3(em.p0), ld3(em.p1), ld3(em.p2),
                                                                 mk2(light_sample.x, light_sample.y));
                            const bool side = sampled_side(em.emission_sampling, ld3(em.ng), ls.direction);
                            const float pdf = ls.pdf * selected.selection_pdf;
                            if (ls.valid && side && em.area > 0.0f && pdf > 0.0f) {
                                const bool is_transmission = dot(ls.direction, sp.n) < 0.0f;
                                const bool same_primitive = em.cycles_prim == sp.cycles_prim && em.object == sp.object;
                                const f3 oriented = is_transmission ? -sp.ng : sp.ng;
                                const bool reject_self = same_primitive && dot(ls.direction, oriented) > 0.0f;
                                if (!reject_self) {
                                    sampled = true;
                                    light_radiance = material_emission(s, s.materials[em.material]);
                                    light_pdf = pdf;
                                    pdf_divisor = pdf;
                                    lp = ls.position;
                                    light_obj = em.object;
                                    light_prim = em.cycles_prim;
                                    ldir = ls.direction;
                                }
                            }
                        } else if (selected.kind == 1u) {
                            // AnalyticLightingComponent (src/luisa/path_kernel_nee_analytic.cpp:98-428)
                            const psy_light_desc &l = s.lights[selected.index];
                            if (!(depth > l.max_bounces)) {
                                const AnalyticSample a =
                                    sample_analytic(l, s.lamp_consts[selected.index], sp.position, sp.n,
                                                    (runtime & kRuntimeBsdfHasTransmission) != 0u,
                                                    mk2(light_sample.x, light_sample.y));
                                const float pdf = a.pdf * selected.selection_pdf;
                                if (a.valid && pdf > 0.0f) {
                                    sampled = true;
                                    light_radiance = ld3(l.color) * (l.power * a.eval_factor);
                                    light_pdf = pdf;
                                    pdf_divisor = maxf_(pdf, 1.0e-20f);
                                    // MIS only for lamps a BSDF ray can also hit
                                    // (path_kernel_nee_analytic.cpp:286-292)
                                    weigh_mis = (l.flags & kLightFlagForward) != 0u;
                                    lp = a.position;
                                    ldir = a.direction;
                                    distant = l.type == PSY_LIGHT_DISTANT;
                                }
                            }
                        }
                        if (sampled) {
                            const Evaluation e = evaluate_mixture<kGlossy>(closures, cpt, ldir, lobe_mask, -1);
                            const float mis = weigh_mis ? nee_light_weight(p.direct_mode, light_pdf, e.pdf) : 1.0f;
                            const f3 weighted = e.f * light_radiance * (mis / pdf_divisor);
                            if (any_nonzero(weighted)) {
                                const f3 unshadowed = weighted * mk3(1.0f);
                                surviving =
                                    unshadowed * light_roulette_weight(unshadowed, light_terminate, p.inv_rr_threshold);
                                emit = any_nonzero(surviving);
                            }
                        }
                        if (emit) {
                            // make_shadow_origin (src/luisa/path_kernel_surface_geometry.cpp:168-185)
                            const Xform w2o = xform12(inst.w2o);
                            const f3 so = origin_with_self_exclusion(sp, xform_point(w2o, sp.position),
                                                                     xform_direction(w2o, ldir));
                            const f3 off = lp - so;
                            const float fd = sqrtf(maxf_(dot(off, off), 1.0e-20f));
                            const f3 sdir = distant ? ldir : off / fd;
                            ldist = distant ? 1.0e30f : fd;
                            const f3 c = throughput * surviving;
                            sh_o = make_float4(so.x, so.y, so.z, ldist);
                            sh_d = make_float4(sdir.x, sdir.y, sdir.z, __uint_as_float(ps.transparent_bounce));
                            sh_c = make_float4(c.x, c.y, c.z, __uint_as_float(depth));
                            sh_ids = make_uint4(sp.object, sp.cycles_prim, light_obj, light_prim);
                            shadow = true;
                        }
                    }
                    // SurfaceScatterStageImpl::emit (src/luisa/path_kernel_surface_scatter.cpp:136-291)
                    const SurfaceSample ss = sample_surface<kGlossy>(closures, cpt, bs4.z, mk2(bs4.x, bs4.y), lobe_mask);
                    if (ev) {
                        ev->closure_index = ss.closure_index;
                        ev->bsdf_pdf = ss.eval.pdf;
                        set3(ev->wi, ss.wi);
                    }
                    if (!ss.valid || ss.eval.pdf <= 0.0f) {
                        alive = false;
                    } else {
                        const bool transparent = (ss.eval.events & kEventTransparent) != 0u;
                        const bool singular = (ss.eval.events & kEventSingular) != 0u;
                        const uint32_t label = label_from_events(ss.eval.events);
                        throughput = throughput * (ss.eval.f / ss.eval.pdf);
                        if (ev) {
                            ev->label = label;
                            set3(ev->throughput, throughput);
                        }
                        if (any_nan(throughput) || throughput.x < 0.0f || throughput.y < 0.0f || throughput.z < 0.0f) {
                            alive = false;
                        } else {
                            ps = next_surface(ps, label, runtime, p);
                            if (!transparent) {
                                previous_bsdf_pdf = ss.eval.pdf;
                                previous_delta = singular;
                                b.mis_n[i] = make_float4(sp.n.x, sp.n.y, sp.n.z, 0.0f);
                            }
                            if (ev) {
                                ev->bounce = ps.bounce;
                                ev->transparent_bounce = ps.transparent_bounce;
                                ev->flag = ps.flag;
                                ev->visibility = ps.visibility;
                            }
                            if (transparent) {
                                ray.tmin = next_float_up(h.t);
                            } else {
                                const f3 wi = normalize(ss.wi);
                                const Xform w2o = xform12(inst.w2o);
                                ray.o = origin_with_self_exclusion(sp, sp.object_position, xform_direction(w2o, wi));
                                ray.d = wi;
                                ray.tmin = 0.0f;
                                ray.tmax = 1.0e30f;
                            }
                            keep = true;
                            st2.y = sp.object;
                            st2.z = sp.cycles_prim;
                        }
                    }
                    if (!keep && ev) ev->terminated = 1u;
                }
            }
            const float4 rad_out = make_float4(radiance.x, radiance.y, radiance.z, transparency);
            // an ended path's radiance goes to the film's array; a path still
            // alive after the last step (none, by the step bound) is written
            // there as well
            final = !keep || step + 1u >= p.steps;
            if (final) b.rad_final[i] = rad_out;
            if (keep) {
                store_pair(b.ray_o, i, make_float4(ray.o.x, ray.o.y, ray.o.z, ray.tmin),
                           make_float4(ray.d.x, ray.d.y, ray.d.z, ray.tmax));
                store_pair(b.tp, i, make_float4(throughput.x, throughput.y, throughput.z, previous_bsdf_pdf), rad_out);
                const uint4 st_out = make_uint4(ps.flag, ps.visibility, ps.rng_offset,
                                                ps.bounce | (ps.diffuse_bounce << 8) | (ps.glossy_bounce << 16) |
                                                    (ps.transmission_bounce << 24));
                uint32_t bits = ps.transparent_bounce & 0xffu;
                if (previous_delta) bits |= kSt2Delta;
                if (primary_recorded) bits |= kSt2Primary;
                if ((ps.flag & kFlagTerminateOnNextSurface) != 0u) bits |= kSt2TermNext;
                if ((ps.flag & kFlagTerminateAfterTransparent) != 0u) bits |= kSt2TermAfter;
                st2.x = bits;
                store_pair(b.st, i, st_out, st2);
            }
        }
        const uint32_t slot = warp_push(&b.counters[1], active && keep);
        if (active && keep) b.queue_out[slot] = i;
        const uint32_t sslot = warp_push(&b.counters[2], active && shadow);
        if (active && shadow) {
            b.sh_o[sslot] = sh_o;
            b.sh_d[sslot] = sh_d;
            b.sh_c[sslot] = sh_c;
            b.sh_ids[sslot] = sh_ids;
            b.sh_path[sslot] = i | (final ? kShadowFinal : 0u);
        }
    }
}

// ------------------------------------------------------------------ shadow
// make_trace_shadow_callable (src/luisa/path_tracer_geometry.cpp:75-174)
// iterates closest hits: a transparent surface multiplies its extinction
// and advances tmin past its distance, an opaque one or the
// transparent_max_bounces budget blocks the ray.  The transmittance that
// loop produces depends only on the set of surfaces in [0, tmax]: zero if
// any is opaque or if more than (max - depth) surfaces lie on it, else the
// product in distance order (coincident distances count once, the greatest
// identity standing for them).  The kernel computes it with one any-hit
// traversal: it stops at the first opaque surface, collects transparent
// ones, and multiplies them sorted by distance.  A ray whose surface count
// outgrows the collector falls back to the iterated closest hit.

constexpr int kShadowList = 8;

__device__ __forceinline__ uint32_t surface_material(const SceneView &s, uint32_t instance, uint32_t local) {
    const InstanceGpu &inst = s.instances[instance];
    const MeshGpu mesh = s.meshes[inst.mesh];
    return mesh.material_offset == kInvalid ? inst.material : s.tri_materials[mesh.material_offset + local];
}

__device__ __noinline__ f3 shadow_iterated(const SceneView &s, const RenderParams &p, Ray ray, uint4 ids, uint32_t depth) {
    f3 transmittance = mk3(1.0f);
    for (uint32_t guard = 0; guard < 4096u; ++guard) {
        Hit h;
        if (!trace_closest(s, ray, PSY_VISIBILITY_SHADOW, ids.x, ids.y, ids.z, ids.w, h)) return transmittance;
        if (depth >= p.transparent_max) return mk3(0.0f);
        const f3 t = clamp3(transparent_extinction(s, s.materials[surface_material(s, h.instance, h.prim)]), 0.0f, 1.0f);
        if (!(max_component(t) > 0.0f)) return mk3(0.0f);
        transmittance = transmittance * t;
        depth += 1u;
        ray.tmin = h.t == 0.0f ? 1.17549435e-38f : __uint_as_float(__float_as_uint(h.t) + 1u);
    }
    return mk3(0.0f);
}

__device__ __forceinline__ f3 shadow_transmittance(const SceneView &s, const RenderParams &p, const Ray &ray,
                                                   uint4 ids, uint32_t depth) {
    float tmax = ray.tmax;
    if (!s.any_transparent) {
        bool blocked = false;
        traverse_scene(s, ray, PSY_VISIBILITY_SHADOW, ids.x, ids.y, ids.z, ids.w, tmax,
                       [&](uint32_t, uint32_t, uint32_t, float, float, float) {
                           blocked = true;
                           return true;
                       });
        return blocked ? mk3(0.0f) : mk3(1.0f);
    }
    float lt[kShadowList];
    uint32_t lo[kShadowList], lp[kShadowList], lm[kShadowList];
    int n = 0;
    bool blocked = false, overflow = false;
    traverse_scene(s, ray, PSY_VISIBILITY_SHADOW, ids.x, ids.y, ids.z, ids.w, tmax,
                   [&](uint32_t ii, uint32_t local, uint32_t cp, float t, float, float) {
                       const uint32_t mi = surface_material(s, ii, local);
                       const MaterialGpu m = s.materials[mi];
                       if (!m.has_transparent) {
                           blocked = true;
                           return true;
                       }
                       for (int k = 0; k < n; ++k) {
                           if (lt[k] == t) {  // coincident: keep the greatest identity
                               if (ii > lo[k] || (ii == lo[k] && cp > lp[k])) {
                                   lo[k] = ii;
                                   lp[k] = cp;
                                   lm[k] = mi;
                               }
                               return false;
                           }
                       }
                       if (n == kShadowList) {
                           overflow = true;
                           return true;
                       }
                       lt[n] = t;
                       lo[n] = ii;
                       lp[n] = cp;
                       lm[n] = mi;
                       ++n;
                       return false;
                   });
    if (blocked) return mk3(0.0f);
    const uint32_t budget = depth >= p.transparent_max ? 0u : p.transparent_max - depth;
    if (overflow) {
        if (uint32_t(kShadowList) > budget) return mk3(0.0f);
        return shadow_iterated(s, p, ray, ids, depth);
    }
    if (uint32_t(n) > budget) return mk3(0.0f);
    // insertion sort by distance, then multiply in that order
    for (int i = 1; i < n; ++i) {
        const float kt = lt[i];
        const uint32_t km = lm[i];
        int j = i - 1;
        while (j >= 0 && lt[j] > kt) {
            lt[j + 1] = lt[j];
            lm[j + 1] = lm[j];
            --j;
        }
        lt[j + 1] = kt;
        lm[j + 1] = km;
    }
    f3 transmittance = mk3(1.0f);
    for (int i = 0; i < n; ++i) {
        const f3 t = clamp3(transparent_extinction(s, s.materials[lm[i]]), 0.0f, 1.0f);
        if (!(max_component(t) > 0.0f)) return mk3(0.0f);
        transmittance = transmittance * t;
    }
    return transmittance;
}

// Persistent any-hit shadow kernel (same refill scheme as k_intersect).
// Opaque-only scenes stop at the first accepted candidate; otherwise
// transparent hits are collected per lane and resolved as in
// shadow_transmittance once the traversal ends.
// kMulti: shadow rays of a batched wavefront, each in its path's job.
template <bool kMulti>
__global__ void __launch_bounds__(128, PSY_SHADOW_MIN_BLOCKS)
    k_shadow(const __grid_constant__ SceneView s_arg, const __grid_constant__ RenderParams p_arg,
             const __grid_constant__ PathBuffers b, uint32_t step, uint32_t trace_path, psy_path_trace *trace,
             const JobGpu *jobs, uint32_t sort_threshold) {
    const uint32_t count = b.counters[2];
    const bool sorted = sort_threshold != 0u && count >= sort_threshold;
    TraversalState t;
    bool active = false, exhausted = false, blocked = false, overflow = false;
    uint32_t q_cur = 0u, job = 0u;
    float lt[kShadowList];
    uint32_t lo[kShadowList], lp[kShadowList], lm[kShadowList];
    int n = 0;
    for (;;) {
        uint32_t q = warp_fetch(&b.counters[4], count, !active, exhausted);
        if (sorted && q != kInvalid) q = b.queue_sorted[q];
        if (kMulti && q != kInvalid) job = b.job[b.sh_path[q] & ~kShadowFinal];
        const SceneView &s = kMulti ? jobs[job].s : s_arg;
        const RenderParams &p = kMulti ? jobs[job].p : p_arg;
        if (q != kInvalid) {
            q_cur = q;
            const float4 o = b.sh_o[q], d = b.sh_d[q];
            const uint4 ids = b.sh_ids[q];
            const Ray ray{mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), 0.0f, o.w};
            traversal_begin(t, s, ray, PSY_VISIBILITY_SHADOW, ids.x, ids.y, ids.z, ids.w);
            blocked = overflow = false;
            n = 0;
            active = true;
        }
        if (!__any_sync(kFullMask, active)) break;
        if (!active) continue;
        bool done;
        if (!s.any_transparent) {
            done = traversal_steps<false>(t, s, kTraversalBudget, [&](uint32_t, uint32_t, uint32_t, float, float, float) {
                blocked = true;
                return true;
            });
        } else {
            done = traversal_steps<false>(t, s, kTraversalBudget,
                                          [&](uint32_t ii, uint32_t local, uint32_t cp, float th, float, float) {
                const uint32_t mi = surface_material(s, ii, local);
                if (!s.materials[mi].has_transparent) {
                    blocked = true;
                    return true;
                }
                for (int k = 0; k < n; ++k) {
                    if (lt[k] == th) {
                        if (ii > lo[k] || (ii == lo[k] && cp > lp[k])) {
                            lo[k] = ii;
                            lp[k] = cp;
                            lm[k] = mi;
                        }
                        return false;
                    }
                }
                if (n == kShadowList) {
                    overflow = true;
                    return true;
                }
                lt[n] = th;
                lo[n] = ii;
                lp[n] = cp;
                lm[n] = mi;
                ++n;
                return false;
            });
        }
        if (!done) continue;
        active = false;
        const float4 d = b.sh_d[q_cur], c = b.sh_c[q_cur];
        const uint32_t depth = __float_as_uint(c.w);
        const uint32_t tdepth = __float_as_uint(d.w);
        f3 transmittance = mk3(0.0f);
        if (!blocked) {
            const uint32_t budget = tdepth >= p.transparent_max ? 0u : p.transparent_max - tdepth;
            if (overflow) {
                if (uint32_t(kShadowList) <= budget)
                    transmittance = shadow_iterated(s, p, t.ray, b.sh_ids[q_cur], tdepth);
            } else if (uint32_t(n) <= budget) {
                for (int i = 1; i < n; ++i) {
                    const float kt = lt[i];
                    const uint32_t km = lm[i];
                    int j = i - 1;
                    while (j >= 0 && lt[j] > kt) {
                        lt[j + 1] = lt[j];
                        lm[j + 1] = lm[j];
                        --j;
                    }
                    lt[j + 1] = kt;
                    lm[j + 1] = km;
                }
                transmittance = mk3(1.0f);
                for (int i = 0; i < n; ++i) {
                    const f3 e = clamp3(transparent_extinction(s, s.materials[lm[i]]), 0.0f, 1.0f);
                    if (!(max_component(e) > 0.0f)) {
                        transmittance = mk3(0.0f);
                        break;
                    }
                    transmittance = transmittance * e;
                }
            }
        }
        const uint32_t owner = b.sh_path[q_cur];
        const uint32_t path = owner & ~kShadowFinal;
        f3 contribution = mk3(0.0f);
        if (transmittance.x > 0.0f || transmittance.y > 0.0f || transmittance.z > 0.0f) {
            contribution = clamp_contribution(mk3(c.x, c.y, c.z) * transmittance, depth, p);
            float4 &dst = (owner & kShadowFinal) != 0u ? b.rad_final[path] : b.rad[path];
            float4 r = dst;
            r.x += contribution.x;
            r.y += contribution.y;
            r.z += contribution.z;
            dst = r;
        }
        if (trace && path == trace_path && step < PSY_TRACE_MAX_EVENTS) set3(trace->events[step].nee, contribution);
    }
}

// -------------------------------------------------------------------- film
// accumulate_path_sample + write_film (src/luisa/path_kernel_setup.cpp:903-1062):
// samples are added in sample order.
// One window pixel: its samples of the batch added to the film in sample
// order, one at a time, so the film does not depend on how the samples were
// grouped into batches.
__device__ __forceinline__ void film_pixel(const PathBuffers &b, uint32_t px, uint32_t pixels, uint32_t samples,
                                           uint32_t path_begin, float4 *combined, float4 *normal, float4 *albedo,
                                           uint32_t *sample_count, uint32_t trace_path, psy_path_trace *trace) {
    float4 c = combined[px], n = normal[px], a = albedo[px];
    auto add = [&](uint32_t i, const float4 &r, const float4 &nn, const float4 &aa) {
        f3 rad = mk3(r.x, r.y, r.z);
        if (any_nan(rad)) rad = mk3(0.0f);
        c.x += rad.x;
        c.y += rad.y;
        c.z += rad.z;
        c.w += r.w;
        n.x += nn.x;
        n.y += nn.y;
        n.z += nn.z;
        n.w += 1.0f;
        a.x += aa.x;
        a.y += aa.y;
        a.z += aa.z;
        a.w += 1.0f;
        if (trace && i == trace_path) set3(trace->radiance, rad);
    };
    // Four samples' loads are issued before any of them is added (the
    // trace store could alias them, so the compiler would not hoist a later
    // sample's loads above it); the sums still run in sample order.
    constexpr uint32_t kGroup = 4u;
    uint32_t k = 0;
    for (; k + kGroup <= samples; k += kGroup) {
        float4 r[kGroup], nn[kGroup], aa[kGroup];
#pragma unroll
        for (uint32_t u = 0; u < kGroup; ++u) {
            const uint32_t i = path_begin + (k + u) * pixels + px;
            r[u] = b.rad_final[i];
            nn[u] = b.aov_n[i];
            aa[u] = b.aov_a[i];
        }
#pragma unroll
        for (uint32_t u = 0; u < kGroup; ++u) add(path_begin + (k + u) * pixels + px, r[u], nn[u], aa[u]);
    }
    for (; k < samples; ++k) {
        const uint32_t i = path_begin + k * pixels + px;
        add(i, b.rad_final[i], b.aov_n[i], b.aov_a[i]);
    }
    combined[px] = c;
    normal[px] = n;
    albedo[px] = a;
    sample_count[px] += samples;
}

__global__ void k_film(PathBuffers b, uint32_t pixels, uint32_t samples, float4 *combined, float4 *normal,
                       float4 *albedo, uint32_t *sample_count, uint32_t trace_path, psy_path_trace *trace) {
    for (uint32_t px = blockIdx.x * blockDim.x + threadIdx.x; px < pixels; px += gridDim.x * blockDim.x)
        film_pixel(b, px, pixels, samples, 0u, combined, normal, albedo, sample_count, trace_path, trace);
}

// Film of every item of a batched wavefront (a job appears in at most one
// item per wavefront, so its pixels have one writer).
__global__ void k_film_batch(const JobGpu *jobs, const BatchItem *items, const uint32_t *round, PathBuffers b) {
    const uint32_t film_pixels = round[1], item_count = round[2];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < film_pixels; g += gridDim.x * blockDim.x) {
        const BatchItem it = items[find_item(items, item_count, g, [](const BatchItem &t) { return t.film_begin; })];
        const JobGpu &j = jobs[it.job];
        film_pixel(b, g - it.film_begin, it.pixels, it.samples, it.path_begin, j.combined, j.normal, j.albedo,
                   j.sample_count, kInvalid, nullptr);
    }
}

// Start of a batched wavefront: the wavefront `*cursor` of a planned call
// becomes current (its header and items copied to the fixed buffers every
// later kernel reads), the queue counters are set, and the cursor advances.
// One block.
__global__ void k_begin_round(uint32_t *counters, uint32_t *round, BatchItem *items, const uint32_t *plan_rounds,
                              const BatchItem *plan_items, uint32_t *cursor, uint32_t max_items) {
    const uint32_t w = *cursor;
    const uint32_t n = plan_rounds[4u * w + 2u];
    for (uint32_t k = threadIdx.x; k < n && k < max_items; k += blockDim.x)
        items[k] = plan_items[size_t(w) * max_items + k];
    __syncthreads();
    if (threadIdx.x == 0) {
        round[0] = plan_rounds[4u * w];
        round[1] = plan_rounds[4u * w + 1u];
        round[2] = n;
        counters[kCounterWaveGlossy] = plan_rounds[4u * w + 3u];
        counters[0] = round[0];
        counters[1] = counters[2] = counters[3] = counters[4] = 0u;
        *cursor = w + 1u;
    }
}

__global__ void k_swap_counters(uint32_t *counters) {
    counters[0] = counters[1];
    counters[1] = 0u;
    counters[2] = 0u;
    counters[3] = 0u;
    counters[4] = 0u;
}

__global__ void k_set_counters(uint32_t *counters, uint32_t n) {
    counters[0] = n;
    counters[1] = 0u;
    counters[2] = 0u;
    counters[3] = 0u;
    counters[4] = 0u;
}

// Accumulates the number of rays traced by the queues of one step.
__global__ void k_count_rays(const uint32_t *counters, unsigned long long *stats) {
    stats[0] += counters[0];
    stats[1] += counters[2];
}

__global__ void k_check_counts(const uint32_t *counts, uint32_t n, uint32_t expected, uint32_t *mismatch) {
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        bad = bad || counts[i] != expected;
    if (__any_sync(kFullMask, bad) && (threadIdx.x & 31u) == 0u) atomicOr(mismatch, 1u);
}

// write_passes (src/luisa/path_tracer_session.cpp:71-270): Combined = sum x
// exposure / samples with alpha 1 - transparency / samples clamped to [0, 1];
// Normal and Albedo = sum / samples; Sample Count as a float.
__global__ void k_resolve_pass(const float4 *film, const uint32_t *counts, uint32_t n, uint32_t kind, float exposure,
                               float *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = counts[i];
        if (kind == 2u) {
            out[i] = float(c);
            continue;
        }
        const float den = float(c > 1u ? c : 1u);
        float4 v = film[i];
        if (kind == 0u) {
            const float k = exposure / den;
            v.x *= k;
            v.y *= k;
            v.z *= k;
            const float a = 1.0f - v.w / den;
            v.w = a < 0.0f ? 0.0f : (1.0f < a ? 1.0f : a);
        } else {
            v.x /= den;
            v.y /= den;
            v.z /= den;
            v.w /= den;
        }
        reinterpret_cast<float4 *>(out)[i] = v;
    }
}

__global__ void k_debug_sobol(const float4 *table, uint32_t size, const uint32_t *queries, uint32_t count, float4 *out,
                              uint32_t *out_index) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t *q = queries + 5u * i;
    const uint32_t h = pixel_hash(q[0], q[1], q[2]);
    const uint32_t idx = shuffled_sample_index(q[3], q[4], h, size);
    out[i] = table[idx];
    out_index[i] = idx;
}

__global__ void k_debug_light_distribution(const __grid_constant__ SceneView s, const float *u, uint32_t count,
                                           uint32_t *out_kind, uint32_t *out_index, float *out_pdf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const DistEntryGpu e = distribution_sample(s, u[i]);
    out_kind[i] = e.kind;
    out_index[i] = e.index;
    out_pdf[i] = e.selection_pdf;
}

__global__ void k_debug_light_tree(const __grid_constant__ SceneView s, const float4 *queries, const uint32_t *pdf_emitters, uint32_t count,
                                   uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 a = queries[2u * i], b = queries[2u * i + 1u];
    const f3 point = mk3(a.x, a.y, a.z), n = mk3(b.x, b.y, b.z);
    const bool tr = b.w != 0.0f;
    const DistEntryGpu e = lt_sample(s, a.w, point, n, tr);
    const bool valid = e.kind == 0u || e.kind == 1u;
    out_emitters[i] = valid ? (e.kind == 0u ? e.index : s.triangle_emitters + e.index) : kInvalid;
    out_sample_pdf[i] = valid ? e.selection_pdf : 0.0f;
    out_reverse_pdf[i] = lt_pdf(s, pdf_emitters[i], point, n, tr);
}

// ----------------------------------------------------------------- launches

int launch_grid(uint32_t work, int block, const LaunchConfig &lc) {
    const uint32_t blocks = (work + uint32_t(block) - 1u) / uint32_t(block);
    const uint32_t cap = uint32_t(lc.sms) * lc.stream_blocks_per_sm;
    return int(blocks < 1u ? 1u : (blocks > cap ? cap : blocks));
}

void launch_raygen(cudaStream_t st, const LaunchConfig &lc, const RenderParams &p, const PathBuffers &b, uint32_t pixels,
                   uint32_t paths, uint32_t sample_base, uint32_t trace_path, psy_path_trace *trace) {
    k_raygen<<<launch_grid(paths, int(lc.stream_block), lc), lc.stream_block, 0, st>>>(p, b, pixels, paths, sample_base,
                                                                                    trace_path, trace);
}
void launch_set_counters(cudaStream_t st, uint32_t *counters, uint32_t n) { k_set_counters<<<1, 1, 0, st>>>(counters, n); }
// Persistent kernels: enough resident warps to fill every SM (bounded by the
// work so small queues launch few blocks).
int shade_grid(uint32_t work, const LaunchConfig &lc) {
    const uint32_t blocks = (work + 127u) / 128u;
    const uint32_t cap = uint32_t(lc.sms) * lc.shade_blocks_per_sm;
    return int(blocks < 1u ? 1u : (blocks > cap ? cap : blocks));
}
template <bool kMulti>
void launch_sort(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                 const JobGpu *jobs, uint32_t max_work) {
    k_sort_count<kMulti><<<launch_grid(max_work, 256, lc), 256, 0, st>>>(s, p, b, jobs, lc.sort_threshold);
    k_sort_scan<<<1, 1024, 0, st>>>(b, lc.sort_threshold, 0u);
    // ranks are packed in 21 bits: keep every block's chunk below 2^20 paths
    const int scatter_blocks = std::max(launch_grid(max_work, 256, lc), int((max_work >> 20) + 1u));
    k_sort_scatter<<<scatter_blocks, 256, 0, st>>>(b, lc.sort_threshold, 0u);
}
void launch_shadow_sort(cudaStream_t st, const LaunchConfig &lc, const PathBuffers &b, uint32_t max_work) {
    const uint32_t thr = lc.shadow_sort_threshold;
    k_sort_count_shadow<<<launch_grid(max_work, 256, lc), 256, 0, st>>>(b, thr);
    k_sort_scan<<<1, 1024, 0, st>>>(b, thr, 2u);
    const int scatter_blocks = std::max(launch_grid(max_work, 256, lc), int((max_work >> 20) + 1u));
    k_sort_scatter<<<scatter_blocks, 256, 0, st>>>(b, thr, 2u);
}
int persistent_grid(uint32_t work, const LaunchConfig &lc) {
    const uint32_t blocks = (work + 127u) / 128u;
    const uint32_t cap = uint32_t(lc.sms) * lc.traversal_blocks_per_sm;
    return int(blocks < 1u ? 1u : (blocks > cap ? cap : blocks));
}

template <bool kMulti>
void launch_ray_sort(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const PathBuffers &b, const JobGpu *jobs,
                     uint32_t max_work) {
    const uint32_t thr = lc.ray_sort_threshold;
    k_sort_count_rays<kMulti><<<launch_grid(max_work, 256, lc), 256, 0, st>>>(s, b, jobs, thr);
    k_sort_scan<<<1, 1024, 0, st>>>(b, thr, 0u);
    const int scatter_blocks = std::max(launch_grid(max_work, 256, lc), int((max_work >> 20) + 1u));
    k_sort_scatter<<<scatter_blocks, 256, 0, st>>>(b, thr, 0u);
}
void launch_intersect(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const PathBuffers &b, uint32_t max_work) {
    if (lc.ray_sort_threshold) launch_ray_sort<false>(st, lc, s, b, nullptr, max_work);
    k_intersect<false><<<persistent_grid(max_work, lc), 128, 0, st>>>(s, b, nullptr, lc.ray_sort_threshold);
}
void launch_shade(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                  uint32_t max_work, uint32_t step, uint32_t trace_path, psy_path_trace *trace) {
    if (lc.sort_threshold) launch_sort<false>(st, lc, s, p, b, nullptr, max_work);
    const int grid = shade_grid(max_work, lc);
    if (trace && s.has_glossy)
        k_shade<true, false, true><<<grid, 128, 0, st>>>(s, p, b, step, trace_path, trace, nullptr, lc.sort_threshold);
    else if (trace)
        k_shade<true, false, false><<<grid, 128, 0, st>>>(s, p, b, step, trace_path, trace, nullptr, lc.sort_threshold);
    else if (s.has_glossy)
        k_shade<false, false, true><<<grid, 128, 0, st>>>(s, p, b, step, trace_path, trace, nullptr, lc.sort_threshold);
    else
        k_shade<false, false, false><<<grid, 128, 0, st>>>(s, p, b, step, trace_path, trace, nullptr, lc.sort_threshold);
}
void launch_shadow(cudaStream_t st, const LaunchConfig &lc, const SceneView &s, const RenderParams &p, const PathBuffers &b,
                   uint32_t max_work, uint32_t step, uint32_t trace_path, psy_path_trace *trace) {
    if (lc.shadow_sort_threshold) launch_shadow_sort(st, lc, b, max_work);
    k_shadow<false><<<persistent_grid(max_work, lc), 128, 0, st>>>(s, p, b, step, trace_path, trace, nullptr,
                                                                   lc.shadow_sort_threshold);
}
void launch_begin_round(cudaStream_t st, uint32_t *counters, uint32_t *round, BatchItem *items,
                        const uint32_t *plan_rounds, const BatchItem *plan_items, uint32_t *cursor, uint32_t max_items) {
    k_begin_round<<<1, 256, 0, st>>>(counters, round, items, plan_rounds, plan_items, cursor, max_items);
}
void launch_swap(cudaStream_t st, uint32_t *counters) { k_swap_counters<<<1, 1, 0, st>>>(counters); }
void launch_count_rays(cudaStream_t st, const uint32_t *counters, unsigned long long *stats) {
    k_count_rays<<<1, 1, 0, st>>>(counters, stats);
}
void launch_check_counts(cudaStream_t st, const uint32_t *counts, uint32_t n, uint32_t expected, uint32_t *mismatch) {
    cudaMemsetAsync(mismatch, 0, sizeof(uint32_t), st);
    const uint32_t blocks = n == 0u ? 1u : (n + 255u) / 256u;
    k_check_counts<<<blocks < 1184u ? blocks : 1184u, 256, 0, st>>>(counts, n, expected, mismatch);
}
void launch_resolve_pass(cudaStream_t st, const float4 *film, const uint32_t *counts, uint32_t n, uint32_t kind,
                         float exposure, float *out) {
    const uint32_t blocks = n == 0u ? 1u : (n + 255u) / 256u;
    k_resolve_pass<<<blocks < 2368u ? blocks : 2368u, 256, 0, st>>>(film, counts, n, kind, exposure, out);
}
void launch_film(cudaStream_t st, const LaunchConfig &lc, const PathBuffers &b, uint32_t pixels, uint32_t samples, float4 *combined,
                 float4 *normal, float4 *albedo, uint32_t *sample_count, uint32_t trace_path, psy_path_trace *trace) {
    k_film<<<launch_grid(pixels, int(lc.stream_block), lc), lc.stream_block, 0, st>>>(b, pixels, samples, combined, normal,
                                                                                      albedo, sample_count, trace_path,
                                                                                      trace);
}
// Batched wavefront: every kernel reads each path's job record.
void launch_raygen_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const BatchItem *items, const uint32_t *round,
                         const PathBuffers &b, uint32_t max_paths) {
    k_raygen_batch<<<launch_grid(max_paths, int(lc.stream_block), lc), lc.stream_block, 0, st>>>(jobs, items, round, b);
}
void launch_intersect_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work) {
    if (lc.ray_sort_threshold) launch_ray_sort<true>(st, lc, SceneView{}, b, jobs, max_work);
    k_intersect<true><<<persistent_grid(max_work, lc), 128, 0, st>>>(SceneView{}, b, jobs, lc.ray_sort_threshold);
}
void launch_shade_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work,
                        uint32_t step) {
    if (lc.sort_threshold) launch_sort<true>(st, lc, SceneView{}, RenderParams{}, b, jobs, max_work);
    const int grid = shade_grid(max_work, lc);
    k_shade<false, true, false><<<grid, 128, 0, st>>>(SceneView{}, RenderParams{}, b, step, kInvalid, nullptr, jobs,
                                                      lc.sort_threshold);
    k_shade<false, true, true><<<grid, 128, 0, st>>>(SceneView{}, RenderParams{}, b, step, kInvalid, nullptr, jobs,
                                                     lc.sort_threshold);
}
void launch_shadow_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const PathBuffers &b, uint32_t max_work,
                         uint32_t step) {
    if (lc.shadow_sort_threshold) launch_shadow_sort(st, lc, b, max_work);
    k_shadow<true><<<persistent_grid(max_work, lc), 128, 0, st>>>(SceneView{}, RenderParams{}, b, step, kInvalid,
                                                                  nullptr, jobs, lc.shadow_sort_threshold);
}
void launch_film_batch(cudaStream_t st, const LaunchConfig &lc, const JobGpu *jobs, const BatchItem *items, const uint32_t *round,
                       const PathBuffers &b, uint32_t max_pixels) {
    k_film_batch<<<launch_grid(max_pixels, int(lc.stream_block), lc), lc.stream_block, 0, st>>>(jobs, items, round, b);
}

void launch_debug_light_tree(cudaStream_t st, const SceneView &s, const float4 *queries, const uint32_t *pdf_emitters,
                             uint32_t count, uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf) {
    k_debug_light_tree<<<(count + 127u) / 128u, 128, 0, st>>>(s, queries, pdf_emitters, count, out_emitters,
                                                               out_sample_pdf, out_reverse_pdf);
}
void launch_debug_light_distribution(cudaStream_t st, const SceneView &s, const float *u, uint32_t count,
                                     uint32_t *out_kind, uint32_t *out_index, float *out_pdf) {
    k_debug_light_distribution<<<(count + 127u) / 128u, 128, 0, st>>>(s, u, count, out_kind, out_index, out_pdf);
}
void launch_debug_sobol(cudaStream_t st, const float4 *table, uint32_t size, const uint32_t *queries, uint32_t count,
                        float4 *out, uint32_t *out_index) {
    k_debug_sobol<<<(count + 127u) / 128u, 128, 0, st>>>(table, size, queries, count, out, out_index);
}

cudaError_t take_stack_overflows(cudaStream_t st, uint32_t *count) {
    unsigned int v = 0u;
    cudaError_t e = cudaMemcpyFromSymbolAsync(&v, g_stack_overflows, sizeof(v), 0, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && v != 0u) {
        const unsigned int zero = 0u;
        e = cudaMemcpyToSymbolAsync(g_stack_overflows, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    *count = v;
    return e;
}

}  // namespace psy
