// TEST INFRASTRUCTURE -- drives the CUDA backend adapter
// (psycles_b200/adapter/cuda_path_tracer.cpp) from a real Psycles
// SceneSnapshot, built with the reference's own contract API (SceneDelta
// committed through SceneDatabase::apply) and compiled by the reference's own
// MaterialLibrary.  Built by `make -C oracle adapter` into
// oracle/_ref/libpsycles_adapter_probe.so together with the reference's
// libpsycles_core sources; tests/test_adapter*.py call it through ctypes.
//
// The scene is the Cornell-style room of the reference's Luisa demo
// (examples/render_luisa_demo.cpp:203-305): a floor and three walls with
// per-triangle material slots, a scaled block, a ceiling area light, a
// background light and rough diffuse materials.  The "graph" variant feeds
// the block's colour and roughness through value nodes (an RGB node through
// a colour mix, a Value node through float math) so that the reference's
// compiler emits a non-trivial value stream.  The "glossy" variant makes the
// block a GGX Glossy BSDF and the plaster a mix of rough diffuse and
// Beckmann glossy; the "multiscatter" variant asks for the MULTI_GGX
// distribution, which the adapter must refuse; the "glass" variant makes the
// (open-bottomed) block a rough GGX Glass BSDF and the plaster a mix of rough
// diffuse and Beckmann Refraction.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <psycles/adapter/blender_scene.h>
#include <psycles/compiler/core_nodes.h>
#include <psycles/compiler/material_library.h>
#include <psycles/contract/scene.h>
#include <psycles/io/image.h>

#include "../../psycles_b200/adapter/cuda_path_tracer.h"

using namespace psycles;
using namespace psycles::contract;

namespace {

Vec3f v3(float x, float y, float z) { return {x, y, z}; }

// Column-major affine transform from three axes and an origin.
Mat4f columns(Vec3f x, Vec3f y, Vec3f z, Vec3f t) {
    Mat4f m;
    m.elements = {x.x, x.y, x.z, 0.0f, y.x, y.y, y.z, 0.0f, z.x, z.y, z.z, 0.0f, t.x, t.y, t.z, 1.0f};
    return m;
}

Vec3f unit(Vec3f v) {
    const float s = 1.0f / std::sqrt(std::max(v.x * v.x + v.y * v.y + v.z * v.z, 1.0e-20f));
    return {v.x * s, v.y * s, v.z * s};
}

Vec3f cross3(Vec3f a, Vec3f b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// Camera at `eye` looking at `target` (+y up), camera space -z forward.
Mat4f view(Vec3f eye, Vec3f target) {
    const Vec3f forward = unit({target.x - eye.x, target.y - eye.y, target.z - eye.z});
    const Vec3f right = unit(cross3(forward, v3(0.0f, 1.0f, 0.0f)));
    const Vec3f back = {-forward.x, -forward.y, -forward.z};
    const Vec3f up = unit(cross3(back, right));
    return columns(right, up, back, eye);
}

ShaderGraph rough_diffuse(Vec3f color, float roughness) {
    ShaderGraph g;
    const NodeId d = g.add_node(compiler::node_type::diffuse_bsdf, "Diffuse");
    (void)g.set_input(d, "Color", SocketValue::color(color));
    (void)g.set_input(d, "Roughness", SocketValue::floating(roughness));
    g.set_root(ShaderDomain::surface, OutputRef{d, "Closure"});
    return g;
}

// The block's material through value nodes: Color = mix(rgb_a, rgb_b, 0.3),
// Roughness = clamp(value * 0.5).
ShaderGraph graph_diffuse() {
    ShaderGraph g;
    const NodeId a = g.add_node(compiler::node_type::constant_color, "A");
    (void)g.set_input(a, "Color", SocketValue::color(v3(0.035f, 0.18f, 0.85f)));
    const NodeId b = g.add_node(compiler::node_type::constant_color, "B");
    (void)g.set_input(b, "Color", SocketValue::color(v3(0.9f, 0.5f, 0.1f)));
    const NodeId mix = g.add_node(compiler::node_type::mix_color, "Mix");
    (void)g.set_input(mix, "Factor", SocketValue::floating(0.3f));
    (void)g.connect(OutputRef{a, "Color"}, mix, "A");
    (void)g.connect(OutputRef{b, "Color"}, mix, "B");
    const NodeId value = g.add_node(compiler::node_type::constant_float, "Value");
    (void)g.set_input(value, "Value", SocketValue::floating(0.6f));
    const NodeId mul = g.add_node(compiler::node_type::multiply_float, "Multiply");
    (void)g.connect(OutputRef{value, "Value"}, mul, "A");
    (void)g.set_input(mul, "B", SocketValue::floating(0.5f));
    const NodeId clamp = g.add_node(compiler::node_type::clamp_float, "Clamp");
    (void)g.connect(OutputRef{mul, "Value"}, clamp, "Value");
    const NodeId d = g.add_node(compiler::node_type::diffuse_bsdf, "Diffuse");
    (void)g.connect(OutputRef{mix, "Color"}, d, "Color");
    (void)g.connect(OutputRef{clamp, "Value"}, d, "Roughness");
    g.set_root(ShaderDomain::surface, OutputRef{d, "Closure"});
    return g;
}

ShaderGraph glossy(Vec3f color, float roughness, const char *distribution) {
    ShaderGraph g;
    const NodeId n = g.add_node(compiler::node_type::glossy_bsdf, "Glossy");
    (void)g.set_input(n, "Color", SocketValue::color(color));
    (void)g.set_input(n, "Roughness", SocketValue::floating(roughness));
    (void)g.set_property(n, "Distribution", SocketValue::string(distribution));
    g.set_root(ShaderDomain::surface, OutputRef{n, "Closure"});
    return g;
}

// Plaster as Mix(0.25, rough diffuse, Beckmann glossy).
ShaderGraph glossy_plaster() {
    ShaderGraph g;
    const NodeId d = g.add_node(compiler::node_type::diffuse_bsdf, "Diffuse");
    (void)g.set_input(d, "Color", SocketValue::color(v3(0.72f, 0.72f, 0.72f)));
    (void)g.set_input(d, "Roughness", SocketValue::floating(0.35f));
    const NodeId s = g.add_node(compiler::node_type::glossy_bsdf, "Glossy");
    (void)g.set_input(s, "Color", SocketValue::color(v3(0.9f, 0.9f, 0.85f)));
    (void)g.set_input(s, "Roughness", SocketValue::floating(0.2f));
    (void)g.set_property(s, "Distribution", SocketValue::string("BECKMANN"));
    const NodeId m = g.add_node(compiler::node_type::mix_closure, "Mix");
    (void)g.set_input(m, "Factor", SocketValue::floating(0.25f));
    (void)g.connect(OutputRef{d, "Closure"}, m, "A");
    (void)g.connect(OutputRef{s, "Closure"}, m, "B");
    g.set_root(ShaderDomain::surface, OutputRef{m, "Closure"});
    return g;
}

ShaderGraph dielectric(const char *type, Vec3f color, float roughness, float ior, const char *distribution) {
    ShaderGraph g;
    const NodeId n = g.add_node(type, "Dielectric");
    (void)g.set_input(n, "Color", SocketValue::color(color));
    (void)g.set_input(n, "Roughness", SocketValue::floating(roughness));
    (void)g.set_input(n, "IOR", SocketValue::floating(ior));
    (void)g.set_property(n, "Distribution", SocketValue::string(distribution));
    g.set_root(ShaderDomain::surface, OutputRef{n, "Closure"});
    return g;
}

// Plaster as Mix(0.3, rough diffuse, Beckmann refraction).
ShaderGraph refractive_plaster() {
    ShaderGraph g;
    const NodeId d = g.add_node(compiler::node_type::diffuse_bsdf, "Diffuse");
    (void)g.set_input(d, "Color", SocketValue::color(v3(0.72f, 0.72f, 0.72f)));
    (void)g.set_input(d, "Roughness", SocketValue::floating(0.35f));
    const NodeId r = g.add_node(compiler::node_type::refraction_bsdf, "Refraction");
    (void)g.set_input(r, "Color", SocketValue::color(v3(0.9f, 0.9f, 0.85f)));
    (void)g.set_input(r, "Roughness", SocketValue::floating(0.2f));
    (void)g.set_input(r, "IOR", SocketValue::floating(1.3f));
    (void)g.set_property(r, "Distribution", SocketValue::string("BECKMANN"));
    const NodeId m = g.add_node(compiler::node_type::mix_closure, "Mix");
    (void)g.set_input(m, "Factor", SocketValue::floating(0.3f));
    (void)g.connect(OutputRef{d, "Closure"}, m, "A");
    (void)g.connect(OutputRef{r, "Closure"}, m, "B");
    g.set_root(ShaderDomain::surface, OutputRef{m, "Closure"});
    return g;
}

void quad(TriangleMeshDesc &m, Vec3f a, Vec3f b, Vec3f c, Vec3f d, Vec3f n, std::uint32_t slot) {
    const auto base = static_cast<std::uint32_t>(m.positions.size());
    for (const Vec3f &p : {a, b, c, d}) {
        m.positions.push_back(p);
        m.normals.values.push_back(n);
    }
    m.triangles.push_back({base, base + 1u, base + 2u});
    m.triangles.push_back({base, base + 2u, base + 3u});
    m.triangle_material_slots.push_back(slot);
    m.triangle_material_slots.push_back(slot);
}

// variant: 0 plain, 1 value-graph block, 2 glossy block and plaster,
// 3 a MULTI_GGX block, 4 glass block and refractive plaster
SceneSnapshot demo_snapshot(int variant) {
    const MaterialId plaster{1u}, red{2u}, green{3u}, block{4u};
    const bool graph_material = variant == 1;
    SceneDelta delta;
    delta.base_revision = 0u;
    delta.emplace<UpsertMaterial>(
        plaster, MaterialDesc{.name = "Plaster",
                              .shader = variant == 2   ? glossy_plaster()
                                        : variant == 4 ? refractive_plaster()
                                                       : rough_diffuse(v3(0.72f, 0.72f, 0.72f), 0.35f)});
    delta.emplace<UpsertMaterial>(red, MaterialDesc{.name = "Red wall", .shader = rough_diffuse(v3(0.72f, 0.06f, 0.035f), 0.45f)});
    delta.emplace<UpsertMaterial>(green, MaterialDesc{.name = "Green wall", .shader = rough_diffuse(v3(0.04f, 0.54f, 0.12f), 0.45f)});
    ShaderGraph block_shader = graph_material ? graph_diffuse() : rough_diffuse(v3(0.035f, 0.18f, 0.85f), 0.16f);
    if (variant == 2) block_shader = glossy(v3(0.035f, 0.18f, 0.85f), 0.3f, "GGX");
    if (variant == 3) block_shader = glossy(v3(0.035f, 0.18f, 0.85f), 0.3f, "MULTI_GGX");
    if (variant == 4)
        block_shader = dielectric(compiler::node_type::glass_bsdf, v3(0.9f, 0.95f, 1.0f), 0.15f, 1.45f, "GGX");
    delta.emplace<UpsertMaterial>(block, MaterialDesc{.name = "Blue block", .shader = std::move(block_shader)});
    TriangleMeshDesc room;
    room.name = "Room";
    room.material_slots = {plaster, red, green};
    quad(room, v3(-3, 0, 2.5f), v3(3, 0, 2.5f), v3(3, 0, -3), v3(-3, 0, -3), v3(0, 1, 0), 0u);
    quad(room, v3(-3, 0, -3), v3(3, 0, -3), v3(3, 4.5f, -3), v3(-3, 4.5f, -3), v3(0, 0, 1), 0u);
    quad(room, v3(-3, 0, 2.5f), v3(-3, 0, -3), v3(-3, 4.5f, -3), v3(-3, 4.5f, 2.5f), v3(1, 0, 0), 1u);
    quad(room, v3(3, 0, -3), v3(3, 0, 2.5f), v3(3, 4.5f, 2.5f), v3(3, 4.5f, -3), v3(-1, 0, 0), 2u);
    TriangleMeshDesc cube;
    cube.name = "Cube";
    cube.material_slots = {block};
    quad(cube, v3(-1, -1, 1), v3(1, -1, 1), v3(1, 1, 1), v3(-1, 1, 1), v3(0, 0, 1), 0u);
    quad(cube, v3(1, -1, -1), v3(-1, -1, -1), v3(-1, 1, -1), v3(1, 1, -1), v3(0, 0, -1), 0u);
    quad(cube, v3(-1, -1, -1), v3(-1, -1, 1), v3(-1, 1, 1), v3(-1, 1, -1), v3(-1, 0, 0), 0u);
    quad(cube, v3(1, -1, 1), v3(1, -1, -1), v3(1, 1, -1), v3(1, 1, 1), v3(1, 0, 0), 0u);
    quad(cube, v3(-1, 1, 1), v3(1, 1, 1), v3(1, 1, -1), v3(-1, 1, -1), v3(0, 1, 0), 0u);
    delta.emplace<UpsertGeometry>(GeometryId{10u}, std::move(room));
    delta.emplace<UpsertGeometry>(GeometryId{11u}, std::move(cube));
    delta.emplace<UpsertInstance>(InstanceId{30u}, InstanceDesc{.name = "Room", .geometry = GeometryId{10u},
                                                                .visibility_mask = ~std::uint32_t{0u}});
    delta.emplace<UpsertInstance>(
        InstanceId{31u},
        InstanceDesc{.name = "Block", .geometry = GeometryId{11u},
                     .transform = columns(v3(0.72f, 0, 0), v3(0, 1.15f, 0), v3(0, 0, 0.72f), v3(0.35f, 1.15f, -0.55f)),
                     .visibility_mask = ~std::uint32_t{0u}});
    constexpr float kPi = 3.14159265358979323846f;
    delta.emplace<UpsertCamera>(CameraId{20u},
                                CameraDesc{.name = "Camera",
                                           .projection = CameraProjection::perspective,
                                           .transform = view(v3(0.0f, 2.05f, 7.0f), v3(0.0f, 1.5f, -0.8f)),
                                           .field_of_view = 47.0f * kPi / 180.0f,
                                           .horizontal_field_of_view = 47.0f * kPi / 180.0f,
                                           .sensor_fit = CameraSensorFit::vertical,
                                           .orthographic_scale = 1.0f,
                                           .near_clip = 1.0e-3f,
                                           .far_clip = 100.0f});
    delta.emplace<SetActiveCamera>(CameraId{20u});
    delta.emplace<UpsertLight>(LightId{40u},
                               LightDesc{.name = "Softbox",
                                         .type = LightType::area,
                                         .transform = columns(v3(1, 0, 0), v3(0, 0, 1), v3(0, 1, 0), v3(-0.4f, 4.25f, -0.6f)),
                                         .color = v3(1.0f, 0.82f, 0.62f),
                                         .power = 18.0f,
                                         .size = 1.8f,
                                         .spread = kPi});
    delta.emplace<UpsertLight>(LightId{41u}, LightDesc{.name = "World",
                                                       .type = LightType::background,
                                                       .color = v3(0.008f, 0.012f, 0.025f),
                                                       .power = 1.0f});
    SceneDatabase db;
    const SceneApplyResult applied = db.apply(delta);
    if (!applied.committed) return {};
    return db.snapshot();
}

void set_error(char *error, std::size_t capacity, const std::string &message) {
    if (error && capacity) {
        std::strncpy(error, message.c_str(), capacity - 1u);
        error[capacity - 1u] = '\0';
    }
}

struct Flattened {
    cuda_backend::FlatScene flat;
};

}  // namespace

extern "C" {

// The demo snapshot compiled by the reference's MaterialLibrary and
// flattened by the adapter; null with a message on failure.
void *probe_demo_flatten(int variant, char *error, std::size_t capacity) {
    const SceneSnapshot snapshot = demo_snapshot(variant);
    if (snapshot.revision == 0u) {
        set_error(error, capacity, "SceneDatabase::apply rejected the demo delta");
        return nullptr;
    }
    compiler::ShaderCompiler shader_compiler{compiler::make_core_node_registry()};
    compiler::MaterialLibrary library;
    const compiler::MaterialLibraryUpdate update = library.update(snapshot, shader_compiler);
    if (!update.committed) {
        set_error(error, capacity, update.diagnostics.empty() ? "material update failed" : update.diagnostics[0].message);
        return nullptr;
    }
    auto result = std::make_unique<Flattened>();
    std::vector<RenderDiagnostic> diagnostics;
    if (!cuda_backend::flatten(snapshot, library, result->flat, diagnostics)) {
        set_error(error, capacity, diagnostics.empty() ? "flatten failed" : diagnostics[0].message);
        return nullptr;
    }
    return result.release();
}

// The reference's io::write_pfm of a pass image (row-major, top row first).
int probe_write_pfm(std::uint32_t width, std::uint32_t height, std::uint32_t channels, const float *pixels,
                    const char *path) {
    io::PassImage image;
    image.pass = PassRequest{PassKind::combined, "Combined", "", channels};
    image.extent = {width, height};
    image.channels = channels;
    image.pixels.assign(pixels, pixels + std::size_t(width) * height * channels);
    return io::write_pfm(image, path) ? 0 : 1;
}

const psy_scene_desc *probe_flat_desc(const void *flattened) {
    return &static_cast<const Flattened *>(flattened)->flat.desc();
}

void probe_flat_destroy(void *flattened) { delete static_cast<Flattened *>(flattened); }

// Renders the demo snapshot through CudaPathTracerBackend: compile_scene,
// create_session and render_samples(SampleRange, OutputSink&) into the
// reference's io::MemoryOutputSink, in `chunks` equal sample ranges.  Copies
// the Combined, Normal, Albedo (4 channels) and Sample Count (1 channel)
// passes out, and writes the Combined pass with the reference's write_pfm to
// `pfm_path` when it is not null.  Returns 0, or 1 with a message.
int probe_demo_render(int device, int variant, std::uint32_t width, std::uint32_t height, std::uint32_t spp,
                      std::uint32_t chunks, float *combined, float *normal, float *albedo, float *sample_count,
                      const char *pfm_path, char *error, std::size_t capacity) {
    const SceneSnapshot snapshot = demo_snapshot(variant);
    cuda_backend::CudaPathTracerBackend backend{{.device = device, .next_event_estimation = true}};
    if (!backend.valid()) {
        set_error(error, capacity, backend.context_error());
        return 1;
    }
    SceneCompilation compiled = backend.compile_scene(snapshot);
    if (!compiled.ok()) {
        set_error(error, capacity, compiled.diagnostics.empty() ? "compile failed" : compiled.diagnostics[0].message);
        return 1;
    }
    if (compiled.scene->source_revision() != snapshot.revision) {
        set_error(error, capacity, "source revision differs");
        return 1;
    }
    RenderSettings settings;
    settings.full_extent = {width, height};
    settings.integrator.max_bounces = 4u;
    settings.passes = {PassRequest{PassKind::combined, "Combined", "", 4u}, PassRequest{PassKind::normal, "Normal", "", 4u},
                       PassRequest{PassKind::albedo, "Albedo", "", 4u},
                       PassRequest{PassKind::sample_count, "Sample Count", "", 1u}};
    std::unique_ptr<RenderSession> session = backend.create_session(*compiled.scene, settings);
    if (!session) {
        set_error(error, capacity, "create_session returned nullptr");
        return 1;
    }
    io::MemoryOutputSink sink;
    const std::uint32_t step = std::max(1u, spp / std::max(chunks, 1u));
    for (std::uint32_t first = 0; first < spp; first += step) {
        const SampleRange range{first, std::min(step, spp - first), 0u, spp};
        if (!session->render_samples(range, sink)) {
            set_error(error, capacity, std::string("render_samples failed: ") + psy_last_error());
            return 1;
        }
    }
    float *outs[4] = {combined, normal, albedo, sample_count};
    const PassKind kinds[4] = {PassKind::combined, PassKind::normal, PassKind::albedo, PassKind::sample_count};
    for (int k = 0; k < 4; ++k) {
        const io::PassImage *image = sink.find(kinds[k]);
        if (!image) {
            set_error(error, capacity, "a pass is missing from the sink");
            return 1;
        }
        std::memcpy(outs[k], image->pixels.data(), image->pixels.size() * sizeof(float));
    }
    if (pfm_path && !io::write_pfm(*sink.find(PassKind::combined), pfm_path)) {
        set_error(error, capacity, "write_pfm failed");
        return 1;
    }
    // the reference's rejections reach the caller as nullptr
    RenderSettings bad = settings;
    bad.passes.push_back(PassRequest{PassKind::emission, "Emission", "", 4u});
    if (backend.create_session(*compiled.scene, bad)) {
        set_error(error, capacity, "an unsupported pass was accepted");
        return 1;
    }
    return 0;
}

}  // extern "C"

// ---- Blender scene bundles -------------------------------------------------
// The reference's importer (load_blender_scene_bundle) feeding the CUDA
// backend, as examples/render_blender_scene.cpp:232-420 feeds the Luisa one.

namespace {

// The render settings a bundle asks for (render_blender_scene.cpp:400-417),
// with the passes the CUDA path produces.
RenderSettings bundle_settings(const adapter::BlenderSceneImport &imported) {
    RenderSettings settings;
    settings.full_extent = {imported.width, imported.height};
    settings.seed = imported.seed;
    settings.transparent_background = imported.transparent_background;
    settings.pixel_filter = imported.pixel_filter;
    settings.filter_width = imported.filter_width;
    settings.pass_alpha_threshold = imported.pass_alpha_threshold;
    settings.integrator = imported.integrator;
    settings.passes = {PassRequest{PassKind::combined, "Combined", "", 4u}, PassRequest{PassKind::normal, "Normal", "", 4u},
                       PassRequest{PassKind::albedo, "Albedo", "", 4u},
                       PassRequest{PassKind::sample_count, "Sample Count", "", 1u}};
    return settings;
}

std::string import_error(const adapter::BlenderSceneImport &imported) {
    for (const auto &d : imported.diagnostics)
        if (d.severity == adapter::BlenderSceneDiagnosticSeverity::error) return d.message;
    return "the bundle holds no scene";
}

}  // namespace

extern "C" {

// A bundle imported by load_blender_scene_bundle, compiled by the
// reference's MaterialLibrary and flattened by the adapter; `settings`
// receives the psy_render_settings the adapter makes of the bundle's render
// settings and `samples` the bundle's sample count.  Null with a message on
// failure (the importer's first error diagnostic, or the adapter's).
void *probe_bundle_flatten(const char *directory, psy_render_settings *settings, std::uint32_t *samples, char *error,
                           std::size_t capacity) {
    const adapter::BlenderSceneImport imported = adapter::load_blender_scene_bundle(directory);
    if (!imported.ok()) {
        set_error(error, capacity, import_error(imported));
        return nullptr;
    }
    compiler::ShaderCompiler shader_compiler{compiler::make_core_node_registry()};
    compiler::MaterialLibrary library;
    const compiler::MaterialLibraryUpdate update = library.update(*imported.scene, shader_compiler);
    if (!update.committed) {
        set_error(error, capacity, update.diagnostics.empty() ? "material update failed" : update.diagnostics[0].message);
        return nullptr;
    }
    auto result = std::make_unique<Flattened>();
    std::vector<RenderDiagnostic> diagnostics;
    if (!cuda_backend::flatten(*imported.scene, library, result->flat, diagnostics)) {
        set_error(error, capacity, diagnostics.empty() ? "flatten failed" : diagnostics[0].message);
        return nullptr;
    }
    if (settings) *settings = cuda_backend::to_psy_settings(bundle_settings(imported), true);
    if (samples) *samples = imported.samples;
    return result.release();
}

// Renders a bundle through CudaPathTracerBackend with the bundle's own
// render settings: compile_scene(*imported.scene), create_session,
// render_samples(SampleRange, OutputSink&) into io::MemoryOutputSink in
// `chunks` sample ranges of a `spp`-sample render; copies out Combined,
// Normal, Albedo (4 channels) and Sample Count (1 channel).  Returns 0, or
// 1 with a message.
int probe_bundle_render(int device, const char *directory, std::uint32_t spp, std::uint32_t chunks, float *combined,
                        float *normal, float *albedo, float *sample_count, char *error, std::size_t capacity) {
    const adapter::BlenderSceneImport imported = adapter::load_blender_scene_bundle(directory);
    if (!imported.ok()) {
        set_error(error, capacity, import_error(imported));
        return 1;
    }
    cuda_backend::CudaPathTracerBackend backend{{.device = device, .next_event_estimation = true}};
    if (!backend.valid()) {
        set_error(error, capacity, backend.context_error());
        return 1;
    }
    SceneCompilation compiled = backend.compile_scene(*imported.scene);
    if (!compiled.ok()) {
        set_error(error, capacity, compiled.diagnostics.empty() ? "compile failed" : compiled.diagnostics[0].message);
        return 1;
    }
    const RenderSettings settings = bundle_settings(imported);
    std::unique_ptr<RenderSession> session = backend.create_session(*compiled.scene, settings);
    if (!session) {
        set_error(error, capacity, "create_session returned nullptr");
        return 1;
    }
    io::MemoryOutputSink sink;
    const std::uint32_t step = std::max(1u, spp / std::max(chunks, 1u));
    for (std::uint32_t first = 0; first < spp; first += step) {
        const SampleRange range{first, std::min(step, spp - first), 0u, spp};
        if (!session->render_samples(range, sink)) {
            set_error(error, capacity, std::string("render_samples failed: ") + psy_last_error());
            return 1;
        }
    }
    float *outs[4] = {combined, normal, albedo, sample_count};
    const PassKind kinds[4] = {PassKind::combined, PassKind::normal, PassKind::albedo, PassKind::sample_count};
    for (int k = 0; k < 4; ++k) {
        const io::PassImage *image = sink.find(kinds[k]);
        if (!image) {
            set_error(error, capacity, "a pass is missing from the sink");
            return 1;
        }
        std::memcpy(outs[k], image->pixels.data(), image->pixels.size() * sizeof(float));
    }
    return 0;
}

}  // extern "C"
