/*
 * psycles_cuda.h -- C ABI of the B200 path-trace integrator.
 *
 * This is the drop-in boundary for Psycles' render contract.  Each entry
 * point replaces one call of the reference interface; the mapping is given
 * beside every declaration (paths are relative to the Psycles source tree):
 *
 *   contract::RendererBackend::compile_scene   include/psycles/contract/render.h:176
 *   contract::RendererBackend::create_session  include/psycles/contract/render.h:179
 *   contract::RenderSession::reset             include/psycles/contract/render.h:167
 *   contract::RenderSession::render_samples    include/psycles/contract/render.h:168
 *   contract::RenderSession::cancel            include/psycles/contract/render.h:169
 *   contract::OutputSink::write (pass data)    include/psycles/contract/render.h:141
 *   contract::CompiledScene::source_revision   include/psycles/contract/render.h:153
 *
 * Conventions: plain pointers and sizes, no exceptions, every call returns a
 * psy_status; psy_last_error() returns a thread-local message for the last
 * failing call.  Matrices are column-major 4x4 (elements 0..3 are column 0,
 * the translation is elements 12..14), the layout of psycles::Mat4f
 * (include/psycles/core/math.h:31).
 */
#ifndef PSYCLES_CUDA_H
#define PSYCLES_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSY_ABI_VERSION 2u

typedef enum psy_status {
    PSY_OK = 0,
    PSY_ERROR_INVALID_ARGUMENT = 1,
    PSY_ERROR_OUT_OF_MEMORY = 2,
    PSY_ERROR_CUDA = 3,
    PSY_ERROR_CANCELLED = 4,
    PSY_ERROR_RANGE = 5,
    PSY_ERROR_UNSUPPORTED = 6,
    PSY_ERROR_STATE = 7,
    PSY_ERROR_TIMEOUT = 8
} psy_status;

typedef struct psy_context psy_context;
typedef struct psy_scene psy_scene;
typedef struct psy_session psy_session;
typedef struct psy_batch psy_batch;
typedef struct psy_server psy_server;

/* ---------------------------------------------------------------- scene -- */

/* Triangle mesh.  Mirrors contract::MeshDesc positions/normals/indices
 * (include/psycles/contract/scene.h).  `materials` optionally assigns a
 * material per triangle (Cycles' per-face shader); NULL uses the instance
 * material. */
typedef struct psy_mesh_desc {
    const float *positions;      /* vertex_count * 3 */
    const float *normals;        /* vertex_count * 3; may be NULL if !smooth */
    const uint32_t *indices;     /* triangle_count * 3 */
    const uint32_t *materials;   /* triangle_count, or NULL */
    uint32_t vertex_count;
    uint32_t triangle_count;
    uint32_t smooth;             /* 1: interpolate vertex normals */
    uint32_t reserved;
} psy_mesh_desc;

/* Contract RayVisibility bits (include/psycles/contract/scene.h:282). */
#define PSY_VISIBILITY_CAMERA 1u
#define PSY_VISIBILITY_DIFFUSE 2u
#define PSY_VISIBILITY_GLOSSY 4u
#define PSY_VISIBILITY_TRANSMISSION 8u
#define PSY_VISIBILITY_SHADOW 16u
#define PSY_VISIBILITY_VOLUME_SCATTER 32u
#define PSY_VISIBILITY_ALL 63u

/* Mirrors contract::InstanceDesc (include/psycles/contract/scene.h:304). */
typedef struct psy_instance_desc {
    float object_to_world[16];   /* column-major */
    uint32_t mesh;
    uint32_t material;
    uint32_t visibility;         /* PSY_VISIBILITY_* */
    uint32_t reserved;
} psy_instance_desc;

/* Closure operations of the in-scope SurfaceProgram subset
 * (compiler::ClosureOperation, include/psycles/compiler/surface_program.h:415). */
typedef enum psy_closure_op {
    PSY_CLOSURE_NULL = 0,
    PSY_CLOSURE_DIFFUSE = 1,
    PSY_CLOSURE_EMISSION = 2,
    PSY_CLOSURE_TRANSPARENT = 3,
    PSY_CLOSURE_ADD = 4,
    PSY_CLOSURE_MIX = 5,
    PSY_CLOSURE_GLOSSY = 6,
    PSY_CLOSURE_GLASS = 7,
    PSY_CLOSURE_REFRACTION = 8
} psy_closure_op;

/* Microfacet distribution of a glossy, glass or refraction closure (`a` of
 * its instruction): the node's Distribution property (GGX, the default, or
 * BECKMANN; MULTI_GGX's tabulated energy preservation is not in the subset
 * and a scene that uses it is rejected).  A glass closure must be the only
 * BSDF closure of its material: its selection weight among other closures
 * comes from Cycles' tabulated Fresnel albedo, which is not in the subset. */
#define PSY_GLOSSY_GGX 0u
#define PSY_GLOSSY_BECKMANN 1u
/* glossy only: GGX with Cycles' multiple-scattering energy preservation
 * (MULTI_GGX); the scene must carry the GGX albedo tables (ggx_e, ggx_eavg) */
#define PSY_GLOSSY_MULTI_GGX 2u

/* Closure inputs.  A closure input (colour, strength / factor, roughness)
 * is either a slot of the material's parameter block that belongs to the
 * closure node itself -- an unlinked socket, the literal
 * estimate_surface_emission reads (src/compiler/surface_program.cpp:180-186)
 * -- or, with PSY_INPUT_VALUE set, the index of an instruction of the
 * material's value stream (a ValueExpressionId: a linked socket).
 * PSY_INPUT_NONE marks an absent optional input (roughness 0). */
#define PSY_INPUT_VALUE 0x80000000u
#define PSY_INPUT_NONE 0xffffffffu

/* One closure instruction (compiler::ClosureInstruction,
 * include/psycles/compiler/surface_program.h:415-470, in-scope fields):
 * `color` (vector input: diffuse / glossy / transparent / emission
 * colour, glass tint, refraction colour), `scalar` (emission strength, mix
 * factor, glass / refraction IOR), `roughness` (diffuse roughness: Lambert
 * below 1e-5, else Oren-Nayar; glossy, glass and refraction roughness, whose
 * square is the microfacet alpha), `a`/`b` child instruction indices of add
 * and mix, and for glossy, glass and refraction `a` = PSY_GLOSSY_*.  Every
 * closure's Normal input is the shading normal (the socket unlinked). */
typedef struct psy_closure_instruction {
    uint32_t op;
    uint32_t a;
    uint32_t b;
    uint32_t color;
    uint32_t scalar;
    uint32_t roughness;
} psy_closure_instruction;

/* Value operations of the in-scope subset, numbered as
 * compiler::ValueOperation (include/psycles/compiler/surface_program.h:51);
 * semantics of src/luisa/graph_surface_value_math.cpp,
 * graph_surface_value_context.cpp and graph_surface_value_procedural.cpp. */
#define PSY_VALUE_PARAMETER 0u          /* the block's `parameter` slot (scalar or vector block by type) */
#define PSY_VALUE_PASSTHROUGH 1u        /* a */
#define PSY_VALUE_SCALAR_TO_COLOR 2u    /* (a, a, a) */
#define PSY_VALUE_SCALAR_TO_BOOLEAN 3u  /* int(a) != 0 */
#define PSY_VALUE_COLOR_TO_SCALAR 4u    /* dot(a, Film::rgb_to_y) */
#define PSY_VALUE_VECTOR_TO_SCALAR 5u   /* (a.x + a.y + a.z) / 3 */
#define PSY_VALUE_ADD 6u
#define PSY_VALUE_SUBTRACT 7u
#define PSY_VALUE_MULTIPLY 8u
#define PSY_VALUE_DIVIDE 9u             /* 0 where |b| <= 1e-20 */
#define PSY_VALUE_MINIMUM 10u
#define PSY_VALUE_MAXIMUM 11u
#define PSY_VALUE_POWER 12u             /* pow(max(a, 0), b) */
#define PSY_VALUE_ABSOLUTE 14u
#define PSY_VALUE_CLAMP01 15u
#define PSY_VALUE_CLAMP_RANGE 16u       /* clamp(a, b, c); static_u0 1: swap reversed bounds */
#define PSY_VALUE_MIX_FLOAT 21u         /* lerp(a, b, c); static_u0: clamp c */
#define PSY_VALUE_MIX_VECTOR 22u        /* lerp(a, b, t); static_u0: vector t, static_u1: clamp t */
#define PSY_VALUE_MIX 23u               /* colour blend static_u0 (PSY_BLEND_*), static_u1 bit 0: clamp c */
#define PSY_VALUE_MULTIPLY_COLOR 24u    /* lerp(a, a * b, clamp(c, 0, 1)) */
#define PSY_VALUE_INVERT 26u            /* lerp(a, 1 - a, b) */
#define PSY_VALUE_SEPARATE_R 100u       /* static_u0 0 (RGB) only */
#define PSY_VALUE_SEPARATE_G 101u
#define PSY_VALUE_SEPARATE_B 102u
#define PSY_VALUE_COMBINE_COLOR 103u    /* (a, b, c); static_u0 0 (RGB) only */

/* compiler::BlendOperation (surface_program.h:239) of PSY_VALUE_MIX. */
#define PSY_BLEND_MIX 0u
#define PSY_BLEND_DARKEN 1u
#define PSY_BLEND_MULTIPLY 2u
#define PSY_BLEND_LIGHTEN 4u
#define PSY_BLEND_SCREEN 5u
#define PSY_BLEND_ADD 7u
#define PSY_BLEND_DIFFERENCE 11u
#define PSY_BLEND_SUBTRACT 13u

#define PSY_VALUE_TYPE_SCALAR 0u
#define PSY_VALUE_TYPE_VECTOR 1u

/* One value instruction (compiler::ValueInstruction, surface_program.h:359):
 * operands a, b, c name earlier instructions of the same stream, which is
 * topologically ordered. */
typedef struct psy_value_instruction {
    uint32_t op;                 /* PSY_VALUE_* */
    uint32_t type;               /* PSY_VALUE_TYPE_* of the result */
    uint32_t parameter;          /* PSY_VALUE_PARAMETER: block slot */
    uint32_t a;
    uint32_t b;
    uint32_t c;
    uint32_t static_u0;
    uint32_t static_u1;
} psy_value_instruction;

/* contract::EmissionSampling (include/psycles/contract/scene.h:69). */
#define PSY_EMISSION_SAMPLING_NONE 0u
#define PSY_EMISSION_SAMPLING_AUTOMATIC 1u
#define PSY_EMISSION_SAMPLING_FRONT 2u
#define PSY_EMISSION_SAMPLING_BACK 3u
#define PSY_EMISSION_SAMPLING_FRONT_BACK 4u

/* A compiled SurfaceProgram (value stream + closure tree) with its
 * SurfaceParameterBlock (compiler::SurfaceProgram surface_program.h:512,
 * SurfaceParameterBlock surface_program.h:570).  The block is split into
 * scalar and vector slots; a program compiled by the reference gives each
 * ParameterDesc the same index in both. */
typedef struct psy_material_desc {
    const psy_closure_instruction *closures;
    uint32_t closure_count;
    uint32_t root;
    const float *scalars;        /* scalar_count floats */
    uint32_t scalar_count;
    uint32_t vector_count;
    const float *vectors;        /* vector_count * 3 floats */
    uint32_t emission_sampling;  /* PSY_EMISSION_SAMPLING_* */
    uint32_t value_count;        /* at most 64 */
    const psy_value_instruction *values;
    uint32_t flags;              /* PSY_MATERIAL_* */
    uint32_t reserved;
} psy_material_desc;

/* contract::Material::use_bump_map_correction (include/psycles/contract/
 * scene.h:111-114) is on by default: glossy closures then correct their
 * normal so the specular reflection of the viewing direction stays above
 * the geometric surface.  This flag turns it off. */
#define PSY_MATERIAL_NO_BUMP_MAP_CORRECTION 1u

/* contract::LightType order (include/psycles/contract/scene.h:369). */
typedef enum psy_light_type {
    PSY_LIGHT_POINT = 0,
    PSY_LIGHT_SPOT = 1,
    PSY_LIGHT_AREA = 2,
    PSY_LIGHT_DISTANT = 3
} psy_light_type;

#define PSY_LIGHT_FLAG_SPHERE 1u      /* point/spot radius is a sphere */
#define PSY_LIGHT_FLAG_NORMALIZE 2u   /* divide power by emitter area */
#define PSY_LIGHT_FLAG_ELLIPSE 4u     /* area light: ellipse, else rectangle */
#define PSY_LIGHT_FLAG_USE_MIS 8u     /* LightDesc::use_mis (contract default on) */

/* Analytic light (LightGpu, src/luisa/path_tracer_types.h:142). */
typedef struct psy_light_desc {
    uint32_t type;
    uint32_t flags;              /* PSY_LIGHT_FLAG_*; bits 16-31 reserved (0) */
    uint32_t max_bounces;
    uint32_t visibility;         /* LightDesc::visibility_mask, PSY_VISIBILITY_* */
    float position[3];
    float axis_x[3];
    float axis_y[3];
    float axis_z[3];             /* spot/area: emission axis; sun: D at centre */
    float axis_scale[3];
    float color[3];
    float power;
    float radius;
    float size_u;
    float size_v;
    float spot_angle;
    float spot_smooth;
    float angle;                 /* sun angular diameter */
    float spread;                /* area light spread; pi = full */
} psy_light_desc;

/* contract::CameraProjection (include/psycles/contract/scene.h:335). */
#define PSY_CAMERA_PERSPECTIVE 0u
#define PSY_CAMERA_ORTHOGRAPHIC 1u
#define PSY_CAMERA_PANORAMA 2u   /* equirectangular: 360 x 180 degrees */

/* contract::CameraDesc (include/psycles/contract/scene.h:347).  Depth of
 * field applies to perspective cameras with aperture_radius > 0 and
 * focal_distance > 0 (src/luisa/path_tracer_kernel.cpp:275-278); a zero
 * aperture_ratio is taken as 1e-5, as the reference clamps it. */
typedef struct psy_camera_desc {
    float camera_to_world[16];   /* column-major */
    float field_of_view;         /* vertical angle, radians */
    float horizontal_field_of_view;
    uint32_t sensor_fit;         /* 0 automatic, 1 horizontal, 2 vertical */
    float lens_shift_x;
    float lens_shift_y;
    float near_clip;
    float far_clip;
    uint32_t projection;         /* PSY_CAMERA_* */
    float orthographic_scale;    /* along the fitted sensor dimension */
    float aperture_radius;
    float focal_distance;
    uint32_t aperture_blades;    /* 0: round aperture, else a regular polygon */
    float aperture_rotation;
    float aperture_ratio;        /* anamorphic ratio, 1 = round */
    uint32_t reserved;
} psy_camera_desc;

/* A flattened SceneSnapshot (include/psycles/contract/scene.h:458). */
typedef struct psy_scene_desc {
    const psy_mesh_desc *meshes;
    const psy_instance_desc *instances;
    const psy_material_desc *materials;
    const psy_light_desc *lights;
    uint32_t mesh_count;
    uint32_t instance_count;
    uint32_t material_count;
    uint32_t light_count;
    psy_camera_desc camera;
    float background[3];         /* constant world colour */
    uint32_t world_visibility;   /* PSY_VISIBILITY_* */
    uint64_t revision;           /* SceneSnapshot revision */
    /* Cycles' GGX directional albedo E (32 rows of incoming cosine x 32
     * columns of roughness, both over [0, 1]) and its average over the
     * cosine (32 values of roughness): the tables table_ggx_E and
     * table_ggx_Eavg that MULTI_GGX glossy closures read
     * (src/luisa/graph_surface_scattering.cpp:170-198).  The caller passes
     * the reference's own tables; null when no material asks for them. */
    const float *ggx_e;
    const float *ggx_eavg;
} psy_scene_desc;

/* ------------------------------------------------------------- settings -- */

/* contract::PassKind values used by psy_session_read_pass
 * (include/psycles/contract/render.h:14). */
#define PSY_PASS_COMBINED 0u
#define PSY_PASS_NORMAL 2u
#define PSY_PASS_ALBEDO 4u
#define PSY_PASS_DENOISING_NORMAL 18u
#define PSY_PASS_DENOISING_ALBEDO 19u
#define PSY_PASS_SAMPLE_COUNT 20u

/* contract::PixelFilter (render.h:69). */
#define PSY_FILTER_BOX 0u
#define PSY_FILTER_GAUSSIAN 1u
#define PSY_FILTER_BLACKMAN_HARRIS 2u

/* contract::DirectLightSampling (render.h:75). */
#define PSY_DIRECT_LIGHT_MIS 0u
#define PSY_DIRECT_LIGHT_FORWARD 1u
#define PSY_DIRECT_LIGHT_NEE 2u

/* contract::RenderSettings + PathIntegratorSettings (render.h:81-115) and
 * the next_event_estimation option of the Luisa backend
 * (include/psycles/luisa/path_tracer.h:46). */
typedef struct psy_render_settings {
    uint32_t full_width;
    uint32_t full_height;
    uint32_t window_x;
    uint32_t window_y;
    uint32_t window_width;       /* 0 -> full extent */
    uint32_t window_height;
    uint32_t seed;
    uint32_t transparent_background;
    uint32_t pixel_filter;
    float filter_width;
    float pass_alpha_threshold;
    uint32_t max_bounces;
    uint32_t min_bounces;
    uint32_t diffuse_bounces;
    uint32_t glossy_bounces;
    uint32_t transmission_bounces;
    uint32_t transparent_min_bounces;
    uint32_t transparent_max_bounces;
    float sample_clamp_direct;
    float sample_clamp_indirect;
    float film_exposure;
    float light_sampling_threshold;
    uint32_t use_light_tree;
    uint32_t direct_light_sampling;
    uint32_t next_event_estimation;
    uint32_t reserved;
} psy_render_settings;

/* Fills the defaults of contract::RenderSettings / PathIntegratorSettings. */
void psy_render_settings_default(psy_render_settings *settings);

/* --------------------------------------------------------- entry points -- */

const char *psy_last_error(void);
uint32_t psy_abi_version(void);

/* One context per CUDA device; owns the stream all sessions launch on.
 * Destroy every server, batch, session and scene of a context before the
 * context: their device memory is freed in the order of its stream. */
psy_status psy_context_create(int device, psy_context **out);
void psy_context_destroy(psy_context *context);

/* RendererBackend::compile_scene (render.h:176, implemented by
 * LuisaPathTracerBackend at src/luisa/path_tracer_scene.cpp:50): uploads
 * geometry, builds the two-level BVH, parameter blocks, emitter tables and
 * the flat light distribution.  The descriptor is copied; the caller may
 * free it on return. */
psy_status psy_scene_compile(psy_context *context, const psy_scene_desc *desc,
                             psy_scene **out);
void psy_scene_destroy(psy_scene *scene);
/* CompiledScene::source_revision (render.h:153). */
uint64_t psy_scene_source_revision(const psy_scene *scene);

/* Wall-clock phases of psy_scene_compile, the BVH build and upload times
 * the reference reports apart from render time (VALIDATION.md:751-755).
 * The light tree is built the first time a session of the scene asks for
 * it (use_light_tree), and again after a parameter edit of an emissive
 * material once built; light_tree_ms is its latest build. */
typedef struct psy_scene_build_stats {
    double total_ms;        /* psy_scene_compile, validation to upload */
    double validate_ms;
    double blas_ms;         /* per-mesh BVH builds, parallel over meshes */
    double tlas_ms;
    double emitters_ms;     /* materials, emissive triangles, flat distribution */
    double upload_ms;
    double light_tree_ms;
    uint32_t build_threads; /* host threads of the BLAS builds */
    uint32_t light_tree_builds;
    /* Traversal stack: the largest stack any ray can build in this scene's
     * trees (TLAS entries + the return to the world ray + BLAS entries),
     * proved at compile time to fit the device stack of stack_capacity
     * entries; a mesh whose SAH tree would not fit is rebuilt with median
     * splits (counted in median_rebuilds), and a scene that still would
     * not fit fails to compile with PSY_ERROR_UNSUPPORTED. */
    uint32_t stack_need;
    uint32_t stack_capacity;
    uint32_t median_rebuilds;
    uint32_t reserved;
    uint64_t upload_bytes;  /* host -> device bytes of the compile */
} psy_scene_build_stats;
psy_status psy_scene_get_build_stats(const psy_scene *scene, psy_scene_build_stats *out);

/* Parameter-only material edit: the MaterialLibrary `parameters_rebound`
 * outcome (src/compiler/material_library.cpp:51-97) applied on the device.
 * Rewrites the material's parameter block in place; no BVH or program
 * rebuild.  Counts must equal the compiled block's counts. */
psy_status psy_scene_rebind_parameters(psy_scene *scene, uint32_t material,
                                       const float *scalars,
                                       uint32_t scalar_count,
                                       const float *vectors,
                                       uint32_t vector_count);

/* RendererBackend::create_session (render.h:179,
 * src/luisa/path_tracer.cpp:23).  Returns PSY_ERROR_INVALID_ARGUMENT where
 * the reference returns nullptr. */
psy_status psy_session_create(psy_scene *scene,
                              const psy_render_settings *settings,
                              psy_session **out);
void psy_session_destroy(psy_session *session);
/* Renders the session's scene through `camera` (NULL: the scene's own
 * camera) and clears the film.  No counterpart in the reference, where a
 * camera move is a new SceneSnapshot revision recompiled by compile_scene;
 * here a viewport moves without touching the resident scene. */
psy_status psy_session_set_camera(psy_session *session, const psy_camera_desc *camera);
/* RenderSession::reset (render.h:167): clears the film. */
psy_status psy_session_reset(psy_session *session,
                             const psy_render_settings *settings);

/* RenderSession::render_samples (render.h:168,
 * src/luisa/path_tracer_session.cpp:272).  Renders AA samples
 * [first + offset, first + offset + count) of a render whose total sample
 * count is `total` (SampleRange, render.h:119).  Blocks until the film is
 * updated.  Fails with PSY_ERROR_RANGE for count == 0 or a range beyond
 * total, PSY_ERROR_STATE if total changed within the session, and
 * PSY_ERROR_CANCELLED after cancel(). */
psy_status psy_session_render_samples(psy_session *session, uint32_t first,
                                      uint32_t count, uint32_t offset,
                                      uint32_t total);

/* Allocation-free render_samples, for callers that cannot allocate device
 * memory at render time (a plugin held to its host application's fixed
 * device-memory budget, or a real-time viewport thread that must not stall
 * on an allocation's implicit synchronisation).  No counterpart in the
 * reference.  Renders the same samples with the same kernels, in the same
 * order, as psy_session_render_samples, so the film is bit-identical; the
 * path state lives in static device arrays (about 17 MiB that every GPU
 * loading the library holds until exit) and the session's Sobol table is not
 * used: at most 65536 window pixels and renders of at most 256 total samples
 * (PSY_ERROR_RANGE beyond).  It calls no cudaMalloc, cudaFree or other
 * allocating routine.  Like psy_session_render_samples it issues its work on
 * the context's stream and blocks until the film is updated.  The first call
 * on a device takes the arrays' device addresses and fills the static Sobol
 * table; make that first call before any stream capture.  Calls on one
 * context are serialised; calls on different contexts of one device share
 * the arrays and race when they overlap on the GPU. */
psy_status psy_session_render_samples_static(psy_session *session,
                                             uint32_t first, uint32_t count,
                                             uint32_t offset, uint32_t total);

/* RenderSession::cancel (render.h:169); callable from any thread. */
void psy_session_cancel(psy_session *session);

/* Pass readback, the data write_passes() hands to OutputSink::write
 * (src/luisa/path_tracer_session.cpp:71-270): the window's pixels,
 * row-major, `channels` floats each (4, or 1 for sample count), already
 * divided by the per-pixel sample count.  `capacity` counts floats. */
psy_status psy_session_read_pass(psy_session *session, uint32_t pass_kind,
                                 float *out, uint64_t capacity,
                                 uint32_t *channels);

/* Rendered samples per pixel so far. */
uint32_t psy_session_rendered_samples(const psy_session *session);

/* Per-path trace of one (full-film pixel, absolute sample) for the next
 * render_samples call (LuisaPathTraceRequest,
 * include/psycles/luisa/path_tracer.h:34).  x counts from the left and y
 * from the top of the output image. */
#define PSY_TRACE_MAX_EVENTS 16u
typedef struct psy_path_event {
    uint32_t rng_offset;
    uint32_t bounce;
    uint32_t transparent_bounce;
    uint32_t flag;               /* path flags after the transition */
    uint32_t visibility;         /* Cycles path visibility after it */
    uint32_t hit_object;         /* 0xffffffff on a miss */
    uint32_t hit_primitive;
    uint32_t closure_index;      /* selected closure, 0xffffffff if none */
    uint32_t label;              /* Cycles ClosureLabel of the sample */
    uint32_t light_kind;         /* LightDistributionEmitterKind */
    uint32_t light_index;
    uint32_t terminated;         /* 1 when the path ended at this event */
    float hit_t;
    float hit_u;
    float hit_v;
    float random_terminate;
    float random_light[3];
    float random_light_terminate;
    float random_bsdf[3];
    float continuation_probability;
    float bsdf_pdf;
    float wi[3];
    float throughput[3];         /* after the scatter */
    float emission[3];           /* contribution added at this event */
    float nee[3];                /* NEE contribution (after the shadow ray) */
} psy_path_event;

typedef struct psy_path_trace {
    uint32_t pixel_x;
    uint32_t pixel_y;
    uint32_t sample;
    uint32_t rng_hash;
    uint32_t event_count;
    uint32_t valid;
    float filter[2];
    float ray_origin[3];
    float ray_direction[3];
    float radiance[3];
    psy_path_event events[PSY_TRACE_MAX_EVENTS];
} psy_path_trace;

psy_status psy_session_request_trace(psy_session *session, uint32_t x,
                                     uint32_t y, uint32_t sample);
psy_status psy_session_read_trace(psy_session *session, psy_path_trace *out);

/* Counters of the last render_samples call: traced rays and device time
 * per kernel class, measured with CUDA events on the session stream. */
typedef struct psy_render_stats {
    uint64_t camera_rays;
    uint64_t closest_rays;       /* camera + continuation rays traced */
    uint64_t shadow_rays;
    uint64_t path_segments;
    float ms_total;
    float ms_intersect;
    float ms_shade;
    float ms_shadow;
    float ms_film;
    uint32_t kernel_launches;
    uint32_t batches;
} psy_render_stats;

psy_status psy_session_stats(const psy_session *session,
                             psy_render_stats *out);

/* Per-kernel-class device time of the last render_samples call in profiling
 * mode (CUDA events around every launch; one host synchronisation per path
 * step) and the algorithmic HBM bytes each class moved: the path-state,
 * ray, hit, queue, shadow and film records it must read and write, counted
 * from the live queue sizes.  No reference counterpart: measurement
 * support for the roofline report. */
typedef struct psy_kernel_profile {
    uint32_t raygen_launches;
    uint32_t intersect_launches;
    uint32_t shade_launches;
    uint32_t shadow_launches;
    uint32_t film_launches;
    uint32_t reserved;
    float raygen_ms;
    float intersect_ms;
    float shade_ms;
    float shadow_ms;
    float film_ms;
    float reserved_ms;
    double raygen_bytes;
    double intersect_bytes;
    double shade_bytes;
    double shadow_bytes;
    double film_bytes;
    double reserved_bytes;
} psy_kernel_profile;

psy_status psy_session_set_profiling(psy_session *session, uint32_t enabled);
psy_status psy_session_profile(const psy_session *session,
                               psy_kernel_profile *out);

/* ------------------------------------------- host precompute (no GPU) -- */

/* tabulated_sobol::sequence_size_for_samples
 * (src/sampling/tabulated_sobol.cpp:156). */
uint32_t psy_sobol_sequence_size_for_samples(uint32_t samples);
/* tabulated_sobol::generate_table (src/sampling/tabulated_sobol.cpp:175):
 * writes 256 * sequence_size float4 rows (4 floats each) to `out`. */
psy_status psy_sobol_generate_table(uint32_t sequence_size, float *out);
/* sampling::make_pixel_filter_table (src/sampling/pixel_filter.cpp:30):
 * writes 1024 floats. */
psy_status psy_pixel_filter_table(uint32_t filter, float width, float *out);

/* Launch and capacity tuning of a context (what psycles_b200.autotune
 * searches).  No counterpart in the reference, whose dispatch size is
 * max_samples_per_dispatch.  Zero fields take the defaults. */
typedef struct psy_tuning {
    uint32_t path_capacity;            /* paths per session wavefront; 0 = 16 Mi */
    uint32_t stream_blocks_per_sm;     /* grid cap of grid-stride kernels; 0 = 16 */
    uint32_t traversal_blocks_per_sm;  /* persistent closest-hit / shadow grid; 0 = 12 */
    uint32_t shade_blocks_per_sm;      /* shading grid cap; 0 = 32 */
    uint32_t sort_threshold;           /* sort shading queues of at least this many paths by material;
                                          0 = never, 0xffffffff = the default 65536 */
    uint32_t shadow_sort_threshold;    /* sort shadow queues of at least this many rays by direction;
                                          0 = never (the default), 0xffffffff = the default */
    uint32_t ray_sort_threshold;       /* sort closest-hit queues of at least this many rays by origin
                                          cell and octant; 0 = never (the default), 0xffffffff = the default */
    uint32_t stream_block_size;        /* threads per block of the camera-ray and film kernels: 128, 256 or
                                          512; 0 = 256.  The persistent traversal and shading kernels keep
                                          128-thread blocks (their register budgets are compiled in; their
                                          occupancy is tuned by blocks per SM) */
} psy_tuning;

psy_status psy_context_set_tuning(psy_context *context, const psy_tuning *tuning);
psy_status psy_context_get_tuning(const psy_context *context, psy_tuning *tuning);

/* ------------------------------------------------- batched wavefronts -- */
/* A batch renders sample ranges of many sessions in shared wavefronts:
 * camera paths of every session fill one path state of `path_capacity`
 * paths, and each kernel reads the scene and parameters of its path's
 * session.  No counterpart in the reference, whose sessions dispatch
 * separately (LuisaRenderSession::render_samples,
 * src/luisa/path_tracer_session.cpp:272-397); each session's result is the
 * one render_samples gives, bit for bit, because every pixel adds its
 * samples to the film one at a time in sample order. */
typedef struct psy_batch_config {
    uint32_t path_capacity;      /* paths per wavefront; 0 = the context's (16 Mi); grown to the largest window */
    uint32_t max_jobs;           /* sessions per psy_batch_render call; 0 = 256 */
    uint32_t use_graph;          /* 1: each wavefront replays one captured CUDA graph */
    uint32_t check_interval;     /* without graphs: host check of live paths every N steps (0 = 4) */
} psy_batch_config;

typedef struct psy_batch_stats {
    uint64_t samples;            /* pixel samples rendered by the last call */
    uint64_t closest_rays;
    uint64_t shadow_rays;
    float ms_total;              /* device time of the last call */
    uint32_t wavefronts;
    uint32_t jobs;
    uint32_t graph_launches;
    uint32_t kernel_launches;    /* launched directly or as graph nodes */
} psy_batch_stats;

psy_status psy_batch_create(psy_context *context, const psy_batch_config *config, psy_batch **out);
void psy_batch_destroy(psy_batch *batch);
/* Renders, for each i < n, sessions[i]'s sample range (first[i], count[i],
 * offset[i], total[i]) with the validation and film result of
 * psy_session_render_samples.  Sessions must belong to the batch's context;
 * a session listed twice is rejected.  Per-path traces are not recorded.  A
 * session cancelled during the call stops at the next wavefront and the
 * call returns PSY_ERROR_CANCELLED after finishing the others. */
psy_status psy_batch_render(psy_batch *batch, psy_session *const *sessions, const uint32_t *first,
                            const uint32_t *count, const uint32_t *offset, const uint32_t *total, uint32_t n);
psy_status psy_batch_get_stats(const psy_batch *batch, psy_batch_stats *out);
/* The wavefront plan of a batch, without a GPU: for n jobs of pixels[i]
 * window pixels and samples[i] samples, the items of each wavefront of at
 * most `capacity` paths.  Writes up to max_items records of 6 words (job,
 * wavefront, path_begin, first sample offset, samples, film_begin) and the
 * item count; PSY_ERROR_RANGE when max_items is too small. */
psy_status psy_batch_plan(const uint32_t *pixels, const uint32_t *samples, uint32_t n, uint32_t capacity,
                          uint32_t *out_items, uint32_t max_items, uint32_t *out_count);

/* ----------------------------------------------------------- serving -- */
/* A render server: a request loop thread over resident scenes that admits
 * jobs against an HBM budget and renders all running jobs in shared
 * wavefronts (continuous batching: a job submitted while others run joins
 * the next wavefront).  No counterpart in the reference.  A job's passes
 * equal those of a session rendering the same settings and samples alone.
 * Scenes stay owned by the caller and must outlive their jobs; they must
 * belong to the server's context, and the caller issues no other work on
 * that context while the server runs except psy_scene_compile. */
typedef struct psy_server_config {
    uint64_t hbm_budget_bytes;   /* scenes + job films/tables + path state; 0 = 120 GiB */
    uint32_t path_capacity;      /* paths per wavefront; 0 = the context's (16 Mi) */
    uint32_t max_running;        /* jobs sharing the wavefronts; 0 = 256 */
    uint32_t use_graph;          /* 1: wavefronts replay a captured CUDA graph */
    uint32_t reserved;
} psy_server_config;

#define PSY_JOB_QUEUED 0u
#define PSY_JOB_RUNNING 1u
#define PSY_JOB_DONE 2u
#define PSY_JOB_FAILED 3u
#define PSY_JOB_CANCELLED 4u

typedef struct psy_job_info {
    uint32_t state;              /* PSY_JOB_* */
    int32_t status;              /* psy_status of a failed job */
    uint32_t samples_done;
    uint32_t samples_total;
    double submit_ms;            /* since the server started */
    double admit_ms;
    double done_ms;
} psy_job_info;

typedef struct psy_server_stats {
    uint64_t jobs_submitted;
    uint64_t jobs_done;
    uint64_t jobs_failed;
    uint64_t samples;            /* pixel samples issued */
    uint64_t wavefronts;
    uint64_t bytes_in_use;       /* admitted against the budget */
    uint64_t bytes_peak;
    double busy_ms;              /* wall time with work on the GPU */
    double latency_p50_ms;       /* submit -> done over finished jobs */
    double latency_p99_ms;
    uint32_t latency_jobs;
    uint32_t reserved;
    double device_ms;            /* sum of the wavefronts' event-timed device spans */
} psy_server_stats;

psy_status psy_server_create(psy_context *context, const psy_server_config *config, psy_server **out);
/* Stops the loop after the wavefronts in flight; queued jobs are dropped. */
void psy_server_destroy(psy_server *server);
/* Queues a job rendering `samples` samples of `scene` with `settings`
 * (window and all) through `camera` (NULL: the scene's camera).  A job whose
 * bytes cannot fit the budget even alone fails with PSY_ERROR_OUT_OF_MEMORY. */
psy_status psy_server_submit(psy_server *server, psy_scene *scene, const psy_render_settings *settings,
                             const psy_camera_desc *camera, uint32_t samples, uint64_t *job);
/* A parameter-only material edit (psy_scene_rebind_parameters) ordered
 * with the jobs: applied once no running job uses the scene, before any job
 * submitted after it is admitted. */
psy_status psy_server_rebind_parameters(psy_server *server, psy_scene *scene, uint32_t material,
                                        const float *scalars, uint32_t scalar_count,
                                        const float *vectors, uint32_t vector_count);
psy_status psy_server_poll(psy_server *server, uint64_t job, psy_job_info *out);
/* Waits for a job to end (bounded); PSY_ERROR_TIMEOUT if it has not. */
psy_status psy_server_wait(psy_server *server, uint64_t job, uint32_t timeout_ms);
/* A finished job's pass, as psy_session_read_pass. */
psy_status psy_server_read_pass(psy_server *server, uint64_t job, uint32_t pass_kind, float *out,
                                uint64_t capacity, uint32_t *channels);
/* Frees a finished job's film and returns its bytes to the budget. */
psy_status psy_server_release(psy_server *server, uint64_t job);
psy_status psy_server_cancel(psy_server *server, uint64_t job);
psy_status psy_server_get_stats(psy_server *server, psy_server_stats *out);
/* Device bytes of a compiled scene (what a server counts against its budget). */
uint64_t psy_scene_device_bytes(const psy_scene *scene);

/* ------------------------------------------------ device probes (GPU) -- */

/* Evaluates cycles_sampler::sample_4d (include/psycles/luisa/cycles_sampler.h:260)
 * on the device for `count` queries of (x, y_cycles, seed, sample, dimension)
 * against the table of `sequence_size`, writing 4 floats per query and the
 * shuffled table index per query. */
psy_status psy_debug_sobol_samples(psy_context *context,
                                   uint32_t sequence_size,
                                   const uint32_t *queries, uint32_t count,
                                   float *out_samples, uint32_t *out_indices);

/* Evaluates the compiled scene's many-light tree on the device for `count`
 * shading points: light_tree.surface_sample and light_tree.surface_pdf
 * (src/luisa/path_tracer_light_tree.cpp:547-760).  `queries` holds 8 floats
 * per point: position xyz, random u, shading normal xyz, has-transmission
 * (0 or 1).  Writes the selected emitter identity (emissive triangles first,
 * then analytic lights; 0xffffffff for none) with its selection pdf, and the
 * reverse pdf of emitter `pdf_emitters[i]` from the same point.  Fails with
 * PSY_ERROR_UNSUPPORTED when the scene has no usable tree. */
psy_status psy_debug_light_tree(psy_scene *scene,
                                const float *queries, const uint32_t *pdf_emitters, uint32_t count,
                                uint32_t *out_emitters, float *out_sample_pdf, float *out_reverse_pdf);

/* Evaluates the compiled scene's flat light distribution pick
 * (src/luisa/path_tracer_light_distribution.cpp:12-55) on the device for
 * `count` random numbers: the selected entry's kind (0 emissive triangle,
 * 1 analytic light, 3 none), index and selection pdf. */
psy_status psy_debug_light_distribution(psy_scene *scene, const float *u, uint32_t count, uint32_t *out_kind,
                                        uint32_t *out_index, float *out_pdf);

#ifdef __cplusplus
}
#endif

#endif /* PSYCLES_CUDA_H */
