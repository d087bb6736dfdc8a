// Device-resident scene and render parameters of the B200 path tracer.
//
// HBM layout (one allocation per array, all 16-byte aligned):
//   tlas / blas   4-wide BVH nodes, 128 B each (two 64-byte lines): six
//                 float4 hold the four children's x/y/z slabs lane by
//                 lane, two int4 the child links and leaf counts
//   tris          leaf-ordered triangles of all meshes, 3 float4 per
//                 triangle (48 B): object-space vertices, v0.w = local
//                 primitive index bits
//   positions / normals / indices  the meshes' shading data
//   instances     InstanceGpu (object<->world transforms, mesh, material)
//   materials / code / scalars / vectors  closure programs and their
//                 parameter blocks (rebinding rewrites scalars/vectors)
//   emitters / distribution  emissive triangles and the flat light CDF
//   lights        analytic lights (psy_light_desc)
#pragma once

#include <cstdint>

#include "../../include/psycles_cuda.h"
#include "psy_light_tree.h"

namespace psy {

constexpr uint32_t kInvalidId = 0xffffffffu;

// Light flags the host derives at compile (src/luisa/path_tracer_scene.cpp:1787-1830):
// the effective use_mis (MIS only for lamps with a finite extent) and
// whether BSDF / camera rays can hit the lamp.
constexpr uint32_t kLightFlagUseMis = 1u << 30;
constexpr uint32_t kLightFlagForward = 1u << 31;

struct alignas(16) BvhNodeGpu {
    float4 x;    // left.lo.x, left.hi.x, right.lo.x, right.hi.x
    float4 y;    // left.lo.y, left.hi.y, right.lo.y, right.hi.y
    float4 z;    // left.lo.z, left.hi.z, right.lo.z, right.hi.z
    int4 child;  // x/y: >= 0 inner node, < 0 leaf ~first; z/w: leaf counts
};
static_assert(sizeof(BvhNodeGpu) == 64, "BVH node is one 64-byte line");

// 4-wide node, collapsed from the binary build: child k's slabs in lane k.
// link >= 0: inner node (relative to the BVH's first node); link < 0 with
// count > 0: a leaf (~first triangle, or ~instance in the TLAS); count 0
// with link < 0: an empty slot.
// Traversal stack entries carry a 2-bit tag: a TLAS node, a BLAS node
// (global index), an instance to enter, or the marker that returns to the
// world ray.
constexpr uint32_t kTagTlas = 0u, kTagBlas = 1u << 30, kTagInstance = 2u << 30, kTagLeave = 3u << 30;
constexpr uint32_t kTagMask = 3u << 30;
// Entries of the per-ray traversal stack.  Scene compile proves, from the
// built trees, that no ray can push more (see blas_stack_need /
// tlas_instance_depths in psy_host.cpp), rebuilding a mesh with median
// splits or rejecting the scene where needed; a debug build
// (-DPSY_STACK_CHECK=1) also counts pushes that would not fit on the device.
constexpr uint32_t kTraversalStackSize = 48u;
constexpr uint32_t kGgxETableSize = 32u * 32u, kGgxEavgTableSize = 32u;
// Entries (node groups) of the 8-wide traversal's stack.
constexpr uint32_t kTraversalStackSize8 = 32u;

// Four children of a wide BVH node: boxes as six planes of four lanes, and
// per child either a ready stack entry (count 0: a tagged global node index
// or, in the TLAS, a tagged instance) or the first of `count` triangles in
// the global triangle array.  Empty slots have +inf planes and count 0.
struct alignas(16) WideNodeGpu {
    float4 lox, hix, loy, hiy, loz, hiz;
    int4 link;
    int4 count;
};
static_assert(sizeof(WideNodeGpu) == 128, "wide BVH node is two 64-byte lines");

// Compressed 8-wide BVH node (80 B, after Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017):
// the eight children's boxes as bytes on a per-node grid -- origin p and a
// power-of-two cell 2^(e - 127) per axis -- rounded outward (plus a margin
// that covers the float rounding of the slab test), so every dequantised
// box contains the child's padded box.  Inner children are stored
// contiguously from child_base in slot order, leaves (one triangle record,
// or in the TLAS one instance id) contiguously from leaf_base in slot order.
// Slots are assigned by octant: slot s holds the child nearest to a ray of
// direction octant s (bit a set where component a is negative).
struct alignas(16) CwNodeGpu {
    float px, py, pz;
    uint32_t exps_imask;  // ex | ey << 8 | ez << 16 | imask << 24 (imask bit k: slot k is an inner child)
    uint32_t child_base;  // global index of the first inner child
    uint32_t leaf_base;   // global index of the first leaf entry
    uint32_t leafmask;    // bit k: slot k is a leaf
    uint32_t pad;
    uint32_t q[12];       // lo x, lo y, lo z, hi x, hi y, hi z: two words of eight bytes each, slot k in byte k
};
static_assert(sizeof(CwNodeGpu) == 80, "compressed 8-wide node is five 16-byte words");

struct alignas(16) InstanceGpu {
    float o2w[12];  // column-major c0, c1, c2, c3 (xyz each)
    float w2o[12];
    float nrm[12];  // normal-to-world columns (c3 unused)
    uint32_t mesh, material, visibility, pad;
};

struct alignas(16) MeshGpu {
    uint32_t node_offset;    // root of the mesh BLAS in `blas`
    uint32_t tri_offset;     // first leaf triangle in `tris`
    uint32_t triangle_count;
    uint32_t prim_offset;    // Cycles primitive id of local primitive 0
    uint32_t vertex_offset;  // into positions / normals (vertices)
    uint32_t index_offset;   // into indices (uint32 elements)
    uint32_t material_offset;  // into tri_materials, kInvalid = instance material
    uint32_t smooth;
};

struct alignas(16) MaterialGpu {
    uint32_t code_offset, code_count, root, scalar_offset;
    uint32_t vector_offset, emission_sampling, has_emission, has_transparent;
    uint32_t value_offset, value_count;
    uint32_t bump_correction;  // contract::Material::use_bump_map_correction
    uint32_t pad0;
};

// Value instructions a material's program may hold (its stream is
// evaluated into a per-thread array of this many entries).
constexpr uint32_t kMaxValues = 64u;

struct alignas(16) EmitterGpu {
    float p0[3], p1[3], p2[3], ng[3];
    float area;
    uint32_t material, object, cycles_prim;
    uint32_t emission_sampling, pad0, pad1, pad2;
};

struct alignas(16) DistEntryGpu {
    float cumulative, selection_pdf;
    uint32_t kind, index;
};

// Per-lamp constants of analytic_light_sampling.h that depend on the lamp
// alone, computed once on the host with the kernels' float expressions
// (transcendentals in double, rounded once): the inverse of the spot axes
// (spot_light_to_local, :309-329) with cos(spot_angle / 2) and the smooth
// blend (:331-345), the spot spread cap (:355-376), point_eval_factor
// (:880-896), and the distant lamp's cone and eval factor (:84-108).
struct alignas(16) LampConstGpu {
    float4 spot_rx;  // xyz: first row of the inverse spot axes; w: cos(spot_angle / 2)
    float4 spot_ry;  // w: (1 - cos(spot_angle / 2)) * spot_smooth
    float4 spot_rz;  // w: one minus cosine of the spot's spread cone
    float4 factors;  // x: point eval factor, y: distant cone one minus cosine, z: distant eval factor
};

// Width of the BVH the kernels traverse: 4 (WideNodeGpu) or 8 (CwNodeGpu).
#ifndef PSY_BVH_WIDTH
#define PSY_BVH_WIDTH 4
#endif

struct SceneView {
    const WideNodeGpu *tlas;  // 4-wide trees
    const WideNodeGpu *blas;
    const CwNodeGpu *tlas8;   // compressed 8-wide trees
    const CwNodeGpu *blas8;
    const uint32_t *tlas_ids;  // instance id of each TLAS leaf entry (8-wide)
    const float4 *tris;
    const InstanceGpu *instances;
    const MeshGpu *meshes;
    const float *positions;
    const float *normals;
    const uint32_t *indices;
    const uint32_t *tri_materials;
    const MaterialGpu *materials;
    const psy_closure_instruction *code;
    const psy_value_instruction *values;
    const float *scalars;
    const float *vectors;
    const EmitterGpu *emitters;
    const DistEntryGpu *distribution;
    // Cycles' GGX albedo tables (null unless a material has a MULTI_GGX glossy
    // closure): E, 32 rows of incoming cosine x 32 columns of roughness, and
    // its average over the cosine, 32 values of roughness
    const float *ggx_e;
    const float *ggx_eavg;
    const psy_light_desc *lights;
    uint32_t instance_count;
    uint32_t emitter_count;   // distribution entries - 1 (triangles + lights)
    uint32_t triangle_emitters;
    uint32_t light_count;
    // lamps a ray can hit (area lamps, finite point / spot disks) in light
    // order: bounding sphere (centre, radius^2) and light index
    const float4 *lamp_bounds;
    const LampConstGpu *lamp_consts;  // one per light
    float4 world_lo, world_hi;        // bounds of the instances (xyz)
    const uint32_t *lamp_ids;
    uint32_t lamp_count;
    float triangle_area_pdf;
    float light_selection_pdf;
    float background[3];
    uint32_t world_visibility;
    uint32_t any_transparent;
    uint32_t has_glossy;  // a material holds a glossy, glass or refraction closure (selects the shading variant)
    // many-light tree (empty when the scene has no emitter with energy)
    const LtNodeGpu *lt_nodes;
    const LtEmitterGpu *lt_emitters;
    const uint2 *lt_mapping;  // emitter id -> (tree emitter, leaf node)
    const uint4 *lt_lookup;   // sorted (object, primitive, emitter id)
    uint32_t lt_node_count, lt_emitter_count, lt_lookup_count, lt_root;
};

struct RenderParams {
    uint32_t full_w, full_h, win_x, win_y, win_w, win_h;
    uint32_t seed, transparent_background;
    float pass_alpha_threshold;
    uint32_t maximum, minimum, max_diffuse, max_glossy, max_transmission;
    uint32_t transparent_min, transparent_max, steps;
    float clamp_direct, clamp_indirect, inv_rr_threshold;
    uint32_t direct_mode, nee, use_light_tree;
    float cam[12];  // camera_to_world columns c0..c3
    float htan, vtan, shift_x, shift_y, near_clip, far_clip;
    uint32_t projection, aperture_blades, depth_of_field, pad_camera;  // PSY_CAMERA_*; DOF on / off
    float ortho_span, aperture_radius, focal_distance, aperture_ratio, aperture_rotation;
    const float4 *sobol;
    uint32_t sobol_size;
    const float *filter;  // 1024 entries
};

// Wavefront path state, structure of arrays over `capacity` paths.
// The per-path fields every bounce reads and writes share one 128-byte
// record per path, in four 32-byte sectors: ray origin and direction; the
// two state words; throughput and radiance; the hit and its primitive
// (whose sector's other 12 bytes are written as zeros, so the closest-hit
// kernel writes whole sectors).  The shading kernel takes its paths in
// material order, and one cache line per path then replaces a sector in
// each of eight arrays.
constexpr size_t kPathRecordBytes = 128u;
template <class T>
struct PathField {
    unsigned char *base;  // the field in path 0's record
    __host__ __device__ __forceinline__ T &operator[](size_t i) const {
        return *reinterpret_cast<T *>(base + i * kPathRecordBytes);
    }
};
constexpr size_t kRecRayO = 0u, kRecRayD = 16u, kRecSt = 32u, kRecSt2 = 48u, kRecTp = 64u, kRecRad = 80u,
                 kRecHit = 96u, kRecHitPrim = 112u;

struct PathBuffers {
    PathField<float4> ray_o;    // origin, tmin
    PathField<float4> ray_d;    // direction, tmax
    PathField<float4> tp;       // throughput, previous bsdf pdf
    PathField<float4> rad;      // radiance, transparency
    PathField<uint4> st;        // flag, cycles visibility, rng_offset, packed counters
    PathField<uint4> st2;       // transparent bounce | bits, source object, source prim, pixel
    uint32_t *sample;           // absolute sample index
    float4 *aov_n;              // first-surface normal
    float4 *aov_a;              // albedo
    float4 *mis_n;              // shading normal of the last non-transparent scatter (light-tree MIS)
    PathField<float4> hit;      // t, u, v, instance bits
    PathField<uint4> hit_prim;  // x: primitive (kInvalid on a miss); y, z, w: 0
    float4 *rad_final;          // radiance and transparency of an ended path (the film reads these
                                // coalesced instead of a 16-byte field of each 128-byte record)
    float4 *sh_o;     // shadow origin, tmax
    float4 *sh_d;     // shadow direction, transparent depth bits
    float4 *sh_c;     // unshadowed contribution
    uint4 *sh_ids;    // source object, source prim, light object, light prim
    uint32_t *sh_path;
    uint32_t *queue_in;
    uint32_t *queue_out;
    uint32_t *shadow_queue;
    uint32_t *counters;  // [0] in count, [1] out count, [2] shadow count, [3..4] fetch cursors,
                         // [kCounterWaveGlossy] a batched wavefront's glossy flag
    uint32_t *job;       // batched wavefronts: the job of each path
    // shading-queue sort by material: per-queue-entry bucket, the sorted
    // queue, and kSortBuckets-word histogram / offset arrays
    uint32_t *sort_keys, *queue_sorted, *sort_hist, *sort_offsets;
};

constexpr uint32_t kSortBuckets = 2048u;
constexpr uint32_t kCounterWaveGlossy = 8u;
// sh_path top bit: the shadow ray's path has ended, its contribution goes to rad_final
constexpr uint32_t kShadowFinal = 0x80000000u;

// One job of a batched wavefront: a session's render parameters, its scene
// and its film.  Paths of many jobs share the path state; each path reads
// its job's record.
struct alignas(16) JobGpu {
    RenderParams p;
    SceneView s;
    float4 *combined, *normal, *albedo;
    uint32_t *sample_count;
};

// A block of paths of one job in a batched wavefront: samples
// [sample_base, sample_base + samples) over the job's `pixels` window
// pixels, laid out sample-major from path_begin.  film_begin is the item's
// first pixel in the batch-wide pixel numbering the film kernel walks.
struct BatchItem {
    uint32_t job, path_begin, pixels, samples, sample_base, film_begin, pad0, pad1;
};

// Packed counters of st.w: bounce | diffuse << 8 | glossy << 16 | transmission << 24.
// st2.x: transparent bounce (bits 0-7), previous_delta (8), primary_recorded
// (9), terminate_on_next_surface (10), terminate_after_transparent (11).
constexpr uint32_t kSt2Delta = 1u << 8, kSt2Primary = 1u << 9, kSt2TermNext = 1u << 10, kSt2TermAfter = 1u << 11;

}  // namespace psy
