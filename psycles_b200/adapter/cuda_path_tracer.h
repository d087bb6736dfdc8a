// CudaPathTracerBackend: Psycles' renderer contract over the CUDA path tracer.
//
// A drop-in for LuisaPathTracerBackend (include/psycles/luisa/path_tracer.h:
// 61-79) behind contract::RendererBackend / RenderSession / OutputSink
// (include/psycles/contract/render.h:136-183).  It is compiled against the
// Psycles headers and libpsycles_core (contract, compiler) and calls the C ABI
// of libpsycles_cuda.so (include/psycles_cuda.h):
//
//   compile_scene(snapshot)  MaterialLibrary::update (the reference's own
//                            SurfaceProgram compiler) -> flatten() ->
//                            psy_scene_compile
//   create_session           settings -> psy_render_settings -> psy_session_create
//   render_samples           psy_session_render_samples, then every requested
//                            pass through psy_session_read_pass to the sink, as
//                            LuisaRenderSession::write_passes hands them
//                            (src/luisa/path_tracer_session.cpp:71-255)
//   cancel                   psy_session_cancel
//
// Errors follow the reference: diagnostics (and no scene) from
// compile_scene, nullptr from create_session, false from render_samples;
// no exception crosses the C ABI.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <psycles/compiler/material_library.h>
#include <psycles/contract/render.h>

#include "../../include/psycles_cuda.h"

namespace psycles::cuda_backend {

// A SceneSnapshot flattened into the C ABI's psy_scene_desc, with the arrays
// the descriptor points into.  Movable, not copyable (the descriptor points
// into its own vectors).
class FlatScene {
public:
    FlatScene() = default;
    FlatScene(const FlatScene &) = delete;
    FlatScene &operator=(const FlatScene &) = delete;
    FlatScene(FlatScene &&) = default;
    FlatScene &operator=(FlatScene &&) = default;

    [[nodiscard]] const psy_scene_desc &desc() const noexcept { return _desc; }
    // snapshot MaterialId of each flattened material index
    [[nodiscard]] const std::vector<contract::MaterialId> &material_ids() const noexcept { return _material_ids; }

private:
    friend struct Flattener;
    struct Mesh {
        std::vector<float> positions, normals;
        std::vector<std::uint32_t> indices, materials;
        bool smooth = false;
        bool per_triangle = false;
    };
    struct Material {
        std::vector<psy_closure_instruction> closures;
        std::vector<psy_value_instruction> values;
        std::vector<float> scalars, vectors;
        std::uint32_t root = 0;
        std::uint32_t emission_sampling = PSY_EMISSION_SAMPLING_AUTOMATIC;
        std::uint32_t flags = 0u;  // PSY_MATERIAL_*
    };
    std::vector<Mesh> _meshes;
    std::vector<Material> _materials;
    std::vector<psy_mesh_desc> _mesh_descs;
    std::vector<psy_material_desc> _material_descs;
    std::vector<psy_instance_desc> _instances;
    std::vector<psy_light_desc> _lights;
    std::vector<contract::MaterialId> _material_ids;
    psy_scene_desc _desc{};
};

// Flattens a snapshot whose materials `library` has compiled (the library's
// source revision must be the snapshot's).  Returns false with diagnostics
// for what the CUDA path does not support: closures other than diffuse /
// emission / transparent / add / mix, value operations outside
// psy_value_instruction's set, normal inputs other than the shading normal,
// curves, motion, environments and world shaders, shadow catchers, lights
// with shaders or without shadows, meshes that mix flat and smooth triangles.
bool flatten(const contract::SceneSnapshot &snapshot, const compiler::MaterialLibrary &library, FlatScene &out,
             std::vector<contract::RenderDiagnostic> &diagnostics);

// contract::RenderSettings as the C ABI's settings.
psy_render_settings to_psy_settings(const contract::RenderSettings &settings, bool next_event_estimation);

struct CudaPathTracerOptions {
    int device = 0;
    // LuisaPathTracerOptions::next_event_estimation (path_tracer.h:46)
    bool next_event_estimation = true;
};

class CudaPathTracerBackend final : public contract::RendererBackend {
public:
    explicit CudaPathTracerBackend(CudaPathTracerOptions options = {});
    ~CudaPathTracerBackend() noexcept override;
    CudaPathTracerBackend(const CudaPathTracerBackend &) = delete;
    CudaPathTracerBackend &operator=(const CudaPathTracerBackend &) = delete;

    [[nodiscard]] contract::SceneCompilation compile_scene(const contract::SceneSnapshot &snapshot) override;
    [[nodiscard]] std::unique_ptr<contract::RenderSession> create_session(
        const contract::CompiledScene &scene, const contract::RenderSettings &settings) override;

    // false when no CUDA context could be created (the reason in
    // context_error())
    [[nodiscard]] bool valid() const noexcept { return _context != nullptr; }
    [[nodiscard]] const std::string &context_error() const noexcept { return _context_error; }

private:
    CudaPathTracerOptions _options;
    psy_context *_context = nullptr;
    std::string _context_error;
};

}  // namespace psycles::cuda_backend
