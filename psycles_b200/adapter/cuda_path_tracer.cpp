// CudaPathTracerBackend: contract::RendererBackend over libpsycles_cuda.so.
// See cuda_path_tracer.h for the mapping onto the reference interface.
#include "cuda_path_tracer.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <optional>
#include <set>
#include <utility>

#include <psycles/compiler/core_nodes.h>
#include <psycles/compiler/shader_program.h>
#include <psycles/compiler/surface_program.h>

namespace psycles::cuda_backend {

namespace {

using compiler::ClosureOperation;
using compiler::ValueOperation;
using contract::SocketType;

bool scalar_type(SocketType t) {
    return t == SocketType::boolean || t == SocketType::integer || t == SocketType::unsigned_integer ||
           t == SocketType::floating;
}

bool vector_type(SocketType t) {
    return t == SocketType::float2 || t == SocketType::float3 || t == SocketType::color ||
           t == SocketType::spectrum || t == SocketType::point || t == SocketType::vector || t == SocketType::normal;
}

// A parameter literal as the kernels read it (scalar_parameter_value /
// vector_parameter_value of src/luisa/path_tracer_common.cpp:457-496).
std::optional<float> scalar_literal(const contract::SocketValue &v) {
    switch (v.type) {
    case SocketType::boolean: return std::get<bool>(v.value) ? 1.0f : 0.0f;
    case SocketType::integer: return static_cast<float>(std::get<std::int64_t>(v.value));
    case SocketType::unsigned_integer: return static_cast<float>(std::get<std::uint64_t>(v.value));
    case SocketType::floating: return std::get<float>(v.value);
    default: return std::nullopt;
    }
}

std::optional<Vec3f> vector_literal(const contract::SocketValue &v) {
    if (v.type == SocketType::float2) {
        const auto u = std::get<Vec2f>(v.value);
        return Vec3f{u.x, u.y, 0.0f};
    }
    if (vector_type(v.type)) return std::get<Vec3f>(v.value);
    return std::nullopt;
}

// The value operations psy_value_instruction carries (identical numbering).
bool supported_value_operation(ValueOperation op) {
    switch (op) {
    case ValueOperation::parameter:
    case ValueOperation::passthrough:
    case ValueOperation::scalar_to_color:
    case ValueOperation::scalar_to_boolean:
    case ValueOperation::color_to_scalar:
    case ValueOperation::vector_to_scalar:
    case ValueOperation::add:
    case ValueOperation::subtract:
    case ValueOperation::multiply:
    case ValueOperation::divide:
    case ValueOperation::minimum:
    case ValueOperation::maximum:
    case ValueOperation::power:
    case ValueOperation::absolute:
    case ValueOperation::clamp01:
    case ValueOperation::clamp_range:
    case ValueOperation::mix_float:
    case ValueOperation::mix_vector:
    case ValueOperation::mix:
    case ValueOperation::multiply_color:
    case ValueOperation::invert:
    case ValueOperation::separate_r:
    case ValueOperation::separate_g:
    case ValueOperation::separate_b:
    case ValueOperation::combine_color:
        return true;
    default:
        return false;
    }
}

std::uint32_t closure_op(ClosureOperation op) {
    switch (op) {
    case ClosureOperation::null_closure: return PSY_CLOSURE_NULL;
    case ClosureOperation::diffuse: return PSY_CLOSURE_DIFFUSE;
    case ClosureOperation::emission: return PSY_CLOSURE_EMISSION;
    case ClosureOperation::transparent: return PSY_CLOSURE_TRANSPARENT;
    case ClosureOperation::add: return PSY_CLOSURE_ADD;
    case ClosureOperation::mix: return PSY_CLOSURE_MIX;
    case ClosureOperation::glossy: return PSY_CLOSURE_GLOSSY;
    case ClosureOperation::glass: return PSY_CLOSURE_GLASS;
    case ClosureOperation::refraction: return PSY_CLOSURE_REFRACTION;
    default: return 0xffffffffu;
    }
}

void copy3(float out[3], Vec3f v) {
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

}  // namespace

// The flattening pass; a friend of FlatScene.
struct Flattener {
    const contract::SceneSnapshot &snapshot;
    const compiler::MaterialLibrary &library;
    FlatScene &out;
    std::vector<contract::RenderDiagnostic> &diagnostics;
    std::map<contract::MaterialId, std::uint32_t> material_index;

    bool error(std::string message) {
        diagnostics.push_back({std::move(message)});
        return false;
    }

    // SurfaceProgram + SurfaceParameterBlock -> psy material
    bool material(const compiler::CompiledMaterial &m, const contract::MaterialDesc &desc) {
        const compiler::SurfaceProgram &program = *m.surface_program();
        const std::string who = "Material '" + m.name() + "': ";
        if (!program.root().valid()) return error(who + "has no surface closure");
        if (program.volume_root().valid() || program.surface_normal_root().valid() ||
            program.displacement_root().valid())
            return error(who + "volumes, automatic bump and displacement are not available in the CUDA path");
        FlatScene::Material f;
        // the block: one scalar and one vector slot per ParameterDesc, at its id
        const auto &parameters = program.parameters();
        f.scalars.assign(parameters.size(), 0.0f);
        f.vectors.assign(3u * parameters.size(), 0.0f);
        for (const auto &p : parameters) {
            if (p.id.value >= parameters.size()) return error(who + "parameter id out of range");
            const contract::SocketValue *value = m.parameters().find(p.id);
            if (value == nullptr) continue;
            if (scalar_type(p.type)) {
                if (auto s = scalar_literal(*value)) f.scalars[p.id.value] = *s;
            } else if (vector_type(p.type)) {
                if (auto v = vector_literal(*value)) copy3(&f.vectors[3u * p.id.value], *v);
            } else {
                return error(who + "parameter of a type the CUDA path cannot hold");
            }
        }
        const auto &values = program.value_instructions();
        if (values.size() > 64u) return error(who + "value stream longer than 64 instructions");
        for (const auto &v : values) {
            if (!supported_value_operation(v.operation))
                return error(who + "value operation " + std::to_string(static_cast<unsigned>(v.operation)) +
                             " is not available in the CUDA path");
            if (v.d.valid() || v.e.valid() || v.f.valid() || v.g.valid() || v.h.valid() || v.i.valid() ||
                v.j.valid() || v.static_u0 > 0xffffffffull || v.static_u1 > 0xffffffffull)
                return error(who + "value instruction with operands beyond a, b, c");
            psy_value_instruction w{};
            w.op = static_cast<std::uint32_t>(v.operation);
            if (scalar_type(v.result_type)) w.type = PSY_VALUE_TYPE_SCALAR;
            else if (vector_type(v.result_type)) w.type = PSY_VALUE_TYPE_VECTOR;
            else return error(who + "value of a type the CUDA path cannot hold");
            w.parameter = v.parameter.valid() ? v.parameter.value : 0u;
            w.a = v.a.valid() ? v.a.value : 0u;
            w.b = v.b.valid() ? v.b.value : 0u;
            w.c = v.c.valid() ? v.c.value : 0u;
            w.static_u0 = static_cast<std::uint32_t>(v.static_u0);
            w.static_u1 = static_cast<std::uint32_t>(v.static_u1);
            f.values.push_back(w);
        }
        // a closure input: the closure node's own parameter (an unlinked
        // socket) as its slot, anything else as a value id
        bool ok = true;
        auto input = [&](compiler::ValueExpressionId id, const compiler::ClosureInstruction &c, bool optional) {
            if (!id.valid()) {
                if (!optional) ok = error(who + "closure without a required input");
                return PSY_INPUT_NONE;
            }
            if (id.value >= values.size()) {
                ok = error(who + "closure input out of range");
                return PSY_INPUT_NONE;
            }
            const auto &v = values[id.value];
            if (v.operation == ValueOperation::parameter && v.parameter.valid() && v.source_node == c.source_node)
                return v.parameter.value;
            return PSY_INPUT_VALUE | id.value;
        };
        // the closure normal must be the shading normal: an unlinked Normal
        // socket holding the zero vector, which safe_normalize replaces by
        // the shading normal
        auto shading_normal = [&](const compiler::ClosureInstruction &c) {
            if (c.normal_uses_bump || !c.normal.valid() || c.normal.value >= values.size()) return false;
            const auto &n = values[c.normal.value];
            if (n.operation != ValueOperation::parameter || !n.parameter.valid() ||
                n.parameter.value >= parameters.size())
                return false;
            const float *v = &f.vectors[3u * n.parameter.value];
            return v[0] == 0.0f && v[1] == 0.0f && v[2] == 0.0f;
        };
        for (const auto &c : program.closure_instructions()) {
            const std::uint32_t op = closure_op(c.operation);
            if (op == 0xffffffffu)
                return error(who + "closure operation " + std::to_string(static_cast<unsigned>(c.operation)) +
                             " is not available in the CUDA path");
            psy_closure_instruction k{op, 0u, 0u, PSY_INPUT_NONE, PSY_INPUT_NONE, PSY_INPUT_NONE};
            switch (c.operation) {
            case ClosureOperation::diffuse:
                k.color = input(c.color, c, false);
                k.roughness = input(c.roughness, c, true);
                if (!shading_normal(c))
                    return error(who + "closure normals other than the shading normal are not available in the CUDA path");
                break;
            case ClosureOperation::glossy:
                // Distribution GGX (default) or BECKMANN; MULTI_GGX's
                // tabulated energy preservation is not in the CUDA path
                if (c.preserve_ggx_energy)
                    return error(who + "the Multiscatter GGX distribution is not available in the CUDA path");
                k.a = c.beckmann ? PSY_GLOSSY_BECKMANN : PSY_GLOSSY_GGX;
                k.color = input(c.color, c, false);
                k.roughness = input(c.roughness, c, false);
                if (!shading_normal(c))
                    return error(who + "closure normals other than the shading normal are not available in the CUDA path");
                break;
            case ClosureOperation::glass:
            case ClosureOperation::refraction:
                if (c.preserve_ggx_energy)
                    return error(who + "the Multiscatter GGX distribution is not available in the CUDA path");
                k.a = c.beckmann ? PSY_GLOSSY_BECKMANN : PSY_GLOSSY_GGX;
                k.color = input(c.color, c, false);
                k.roughness = input(c.roughness, c, false);
                k.scalar = input(c.ior, c, false);
                if (!shading_normal(c))
                    return error(who + "closure normals other than the shading normal are not available in the CUDA path");
                break;
            case ClosureOperation::emission:
                k.color = input(c.color, c, false);
                k.scalar = input(c.strength, c, false);
                break;
            case ClosureOperation::transparent:
                k.color = input(c.color, c, false);
                break;
            case ClosureOperation::add:
                k.a = c.a.valid() ? c.a.value : 0xffffffffu;
                k.b = c.b.valid() ? c.b.value : 0xffffffffu;
                break;
            case ClosureOperation::mix:
                k.a = c.a.valid() ? c.a.value : 0xffffffffu;
                k.b = c.b.valid() ? c.b.value : 0xffffffffu;
                k.scalar = input(c.factor, c, false);
                break;
            default:
                break;
            }
            if (!ok) return false;
            f.closures.push_back(k);
        }
        f.root = program.root().value;
        f.emission_sampling = static_cast<std::uint32_t>(desc.emission_sampling);
        f.flags = desc.use_bump_map_correction ? 0u : PSY_MATERIAL_NO_BUMP_MAP_CORRECTION;
        out._materials.push_back(std::move(f));
        return true;
    }

    // A triangle's material (triangle_material,
    // src/luisa/path_tracer_light_sampling_scene.cpp:23-40).
    std::optional<contract::MaterialId> triangle_material(const contract::TriangleMeshDesc &g,
                                                          const contract::InstanceDesc &inst, std::size_t k) {
        const std::uint32_t slot = k < g.triangle_material_slots.size() ? g.triangle_material_slots[k] : 0u;
        if (slot < inst.material_overrides.size()) return inst.material_overrides[slot];
        if (g.material_slots.empty()) return std::nullopt;
        return g.material_slots[std::min<std::size_t>(slot, g.material_slots.size() - 1u)];
    }

    // A geometry as a psy mesh (positions, flat or smooth normals).
    bool mesh(const contract::TriangleMeshDesc &g, FlatScene::Mesh &m) {
        const std::string who = "Geometry '" + g.name + "': ";
        std::size_t smooth = 0u;
        for (std::size_t k = 0; k < g.triangles.size(); ++k)
            if (k < g.triangle_smooth.size() && g.triangle_smooth[k] != 0u) ++smooth;
        if (smooth != 0u && smooth != g.triangles.size())
            return error(who + "meshes that mix flat and smooth triangles are not available in the CUDA path");
        m.smooth = smooth != 0u;
        const bool corner = !g.normals.values.empty() && g.normals.domain == contract::MeshAttributeDomain::corner;
        if (!g.normals.values.empty() && g.normals.domain == contract::MeshAttributeDomain::face)
            return error(who + "face-domain normals are not a Cycles triangle attribute");
        for (const auto &t : g.triangles)
            for (std::uint32_t c = 0; c < 3; ++c)
                if (t[c] >= g.positions.size()) return error(who + "contains an out-of-range index");
        if (corner) {
            // one vertex per corner, so the corner normals become point normals
            if (g.normals.values.size() != 3u * g.triangles.size()) return error(who + "corner normal count");
            for (std::size_t k = 0; k < g.triangles.size(); ++k)
                for (std::uint32_t c = 0; c < 3; ++c) {
                    const Vec3f p = g.positions[g.triangles[k][c]];
                    const Vec3f n = g.normals.values[3u * k + c];
                    m.positions.insert(m.positions.end(), {p.x, p.y, p.z});
                    m.normals.insert(m.normals.end(), {n.x, n.y, n.z});
                    m.indices.push_back(std::uint32_t(3u * k + c));
                }
        } else {
            if (!g.normals.values.empty() && g.normals.values.size() != g.positions.size())
                return error(who + "point normal count differs from the vertex count");
            for (const Vec3f &p : g.positions) m.positions.insert(m.positions.end(), {p.x, p.y, p.z});
            for (std::size_t v = 0; v < g.positions.size(); ++v) {
                const Vec3f n = g.normals.values.empty() ? Vec3f{} : g.normals.values[v];
                m.normals.insert(m.normals.end(), {n.x, n.y, n.z});
            }
            for (const auto &t : g.triangles) m.indices.insert(m.indices.end(), {t[0], t[1], t[2]});
        }
        return true;
    }

    // The world shader's emission where it is constant: the closure tree
    // walked as GraphSurfaceImplementation::constant_emission does
    // (src/luisa/graph_surface_emission.cpp:33-96) -- emission colour x
    // strength x weight, both children of an add, a mix split by its
    // clamped factor, nothing from any other closure.  A world whose
    // emission varies with direction (EmissionEvaluationMode::deferred) is
    // refused: the CUDA path's world is one constant colour.
    bool world_emission(contract::MaterialId id, Vec3f &world) {
        const compiler::CompiledMaterial *m = library.find(id);
        if (m == nullptr) return error("the world shader was not compiled");
        const compiler::SurfaceProgram &program = *m->surface_program();
        if (program.volume_root().valid()) return error("world volumes are not available in the CUDA path");
        if (program.emission_evaluation() == compiler::EmissionEvaluationMode::none) return true;
        if (program.emission_evaluation() != compiler::EmissionEvaluationMode::constant || !program.root().valid())
            return error("world shaders whose emission varies with direction are not available in the CUDA path");
        const auto &values = program.value_instructions();
        auto slot = [&](compiler::ValueExpressionId e) -> const contract::SocketValue * {
            if (!e.valid() || e.value >= values.size() || !values[e.value].parameter.valid()) return nullptr;
            return m->parameters().find(values[e.value].parameter);
        };
        auto scalar = [&](compiler::ValueExpressionId e) {
            const contract::SocketValue *v = slot(e);
            return v == nullptr ? 0.0f : scalar_literal(*v).value_or(0.0f);
        };
        auto vector = [&](compiler::ValueExpressionId e) {
            const contract::SocketValue *v = slot(e);
            return v == nullptr ? Vec3f{} : vector_literal(*v).value_or(Vec3f{});
        };
        const auto &closures = program.closure_instructions();
        auto visit = [&](auto &&self, compiler::ClosureExpressionId c, float weight, int depth) -> void {
            if (!c.valid() || c.value >= closures.size() || depth > 64) return;
            const auto &k = closures[c.value];
            switch (k.operation) {
            case ClosureOperation::emission: {
                const Vec3f color = vector(k.color);
                const float strength = scalar(k.strength);
                world.x += color.x * strength * weight;
                world.y += color.y * strength * weight;
                world.z += color.z * strength * weight;
                return;
            }
            case ClosureOperation::add:
                self(self, k.a, weight, depth + 1);
                self(self, k.b, weight, depth + 1);
                return;
            case ClosureOperation::mix: {
                const float mix = std::clamp(scalar(k.factor), 0.0f, 1.0f);
                self(self, k.a, weight * (1.0f - mix), depth + 1);
                self(self, k.b, weight * mix, depth + 1);
                return;
            }
            default: return;
            }
        };
        visit(visit, program.root(), 1.0f, 0);
        return true;
    }

    bool run() {
        const std::string stale = "the material library was not updated from this snapshot";
        if (library.source_revision() != snapshot.revision) return error(stale);
        if (!snapshot.curve_geometries.empty()) return error("curves are not available in the CUDA path");
        if (snapshot.environment) return error("environments are not available in the CUDA path");
        Vec3f world{};
        if (snapshot.world_shader && !world_emission(*snapshot.world_shader, world)) return false;
        // materials some instance's triangle uses, in MaterialId order; the
        // others (an importer's default surface, the world and light
        // shaders) never reach the device, so what they hold is not refused
        std::set<contract::MaterialId> used;
        for (const auto &[iid, inst] : snapshot.instances) {
            const auto git = snapshot.geometries.find(inst.geometry);
            if (git == snapshot.geometries.end()) continue;
            for (std::size_t k = 0; k < git->second.triangles.size(); ++k)
                if (const auto mid = triangle_material(git->second, inst, k)) used.insert(*mid);
        }
        for (const auto &[id, desc] : snapshot.materials) {
            if (!used.count(id)) continue;
            const compiler::CompiledMaterial *m = library.find(id);
            if (m == nullptr) return error("Material " + std::to_string(id.value) + " was not compiled");
            material_index[id] = static_cast<std::uint32_t>(out._materials.size());
            out._material_ids.push_back(id);
            if (!material(*m, desc)) return false;
        }
        // instances, in InstanceId order; one psy mesh per geometry for the
        // instances whose triangles share one material, and one per distinct
        // per-triangle material list otherwise
        std::map<contract::GeometryId, std::uint32_t> uniform_mesh;
        std::map<std::pair<contract::GeometryId, std::vector<std::uint32_t>>, std::uint32_t> per_triangle_mesh;
        for (const auto &[iid, inst] : snapshot.instances) {
            const std::string who = "Instance '" + inst.name + "': ";
            const auto git = snapshot.geometries.find(inst.geometry);
            if (git == snapshot.geometries.end()) return error(who + "references a missing geometry");
            const contract::TriangleMeshDesc &g = git->second;
            if (!inst.motion.empty()) return error(who + "motion blur is not available in the CUDA path");
            if (inst.is_shadow_catcher) return error(who + "shadow catchers are not available in the CUDA path");
            if (inst.shadow_terminator_geometry_offset > 0.0f)
                return error(who + "a shadow-terminator offset is not available in the CUDA path");
            if (g.triangles.empty()) continue;
            std::vector<std::uint32_t> mats(g.triangles.size());
            for (std::size_t k = 0; k < g.triangles.size(); ++k) {
                const auto mid = triangle_material(g, inst, k);
                if (!mid) return error(who + "a triangle without a material");
                const auto mi = material_index.find(*mid);
                if (mi == material_index.end()) return error(who + "references a missing material");
                mats[k] = mi->second;
            }
            const bool uniform = std::all_of(mats.begin(), mats.end(), [&](std::uint32_t v) { return v == mats[0]; });
            std::uint32_t mesh_index;
            if (uniform) {
                auto [it, fresh] = uniform_mesh.try_emplace(inst.geometry, std::uint32_t(out._meshes.size()));
                if (fresh) {
                    out._meshes.emplace_back();
                    if (!mesh(g, out._meshes.back())) return false;
                }
                mesh_index = it->second;
            } else {
                auto [it, fresh] =
                    per_triangle_mesh.try_emplace({inst.geometry, mats}, std::uint32_t(out._meshes.size()));
                if (fresh) {
                    out._meshes.emplace_back();
                    FlatScene::Mesh &m = out._meshes.back();
                    if (!mesh(g, m)) return false;
                    m.materials = mats;
                    m.per_triangle = true;
                }
                mesh_index = it->second;
            }
            psy_instance_desc d{};
            std::memcpy(d.object_to_world, inst.transform.elements.data(), sizeof(d.object_to_world));
            d.mesh = mesh_index;
            d.material = mats[0];
            // a mask of all ones means every ray (path_tracer_scene.cpp:1492-1496)
            d.visibility = inst.visibility_mask == ~std::uint32_t{0u} ? PSY_VISIBILITY_ALL
                                                                      : (inst.visibility_mask & PSY_VISIBILITY_ALL);
            out._instances.push_back(d);
        }
        // lights: position and axes from the transform, a background light
        // adds to the constant world colour (path_tracer_scene.cpp:1723-1877)
        Vec3f background{};
        for (const auto &[lid, light] : snapshot.lights) {
            const std::string who = "Light '" + light.name + "': ";
            if (light.type == contract::LightType::background) {
                background.x += light.color.x * light.power;
                background.y += light.color.y * light.power;
                background.z += light.color.z * light.power;
                continue;
            }
            if (light.shader) return error(who + "light shaders are not available in the CUDA path");
            if (!light.cast_shadow) return error(who + "lights without shadows are not available in the CUDA path");
            if (light.is_shadow_catcher) return error(who + "shadow catchers are not available in the CUDA path");
            auto axis = [&](std::size_t column, float &length) {
                const float *e = light.transform.elements.data() + 4u * column;
                length = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
                if (length <= 1.0e-20f) {
                    length = 0.0f;
                    return Vec3f{};
                }
                return Vec3f{e[0] / length, e[1] / length, e[2] / length};
            };
            float lx = 0.0f, ly = 0.0f, lz = 0.0f;
            const Vec3f ax = axis(0u, lx), ay = axis(1u, ly);
            Vec3f az = axis(2u, lz);
            if (az == Vec3f{}) az = {0.0f, 0.0f, 1.0f};
            psy_light_desc d{};
            switch (light.type) {
            case contract::LightType::point: d.type = PSY_LIGHT_POINT; break;
            case contract::LightType::spot: d.type = PSY_LIGHT_SPOT; break;
            case contract::LightType::area: d.type = PSY_LIGHT_AREA; break;
            case contract::LightType::distant: d.type = PSY_LIGHT_DISTANT; break;
            default: return error(who + "unknown light type");
            }
            d.flags = (light.normalize ? PSY_LIGHT_FLAG_NORMALIZE : 0u) | (light.ellipse ? PSY_LIGHT_FLAG_ELLIPSE : 0u) |
                      (light.is_sphere ? PSY_LIGHT_FLAG_SPHERE : 0u) | (light.use_mis ? PSY_LIGHT_FLAG_USE_MIS : 0u);
            d.max_bounces = light.max_bounces;
            d.visibility = light.visibility_mask == ~std::uint32_t{0u} ? PSY_VISIBILITY_ALL
                                                                       : (light.visibility_mask & PSY_VISIBILITY_ALL);
            const float *t = light.transform.elements.data();
            d.position[0] = t[12];
            d.position[1] = t[13];
            d.position[2] = t[14];
            copy3(d.axis_x, ax);
            copy3(d.axis_y, ay);
            copy3(d.axis_z, az);
            d.axis_scale[0] = lx;
            d.axis_scale[1] = ly;
            d.axis_scale[2] = lz;
            copy3(d.color, light.color);
            d.power = light.power;
            d.radius = light.size;
            d.size_u = light.size * lx;
            d.size_v = (light.size_y > 0.0f ? light.size_y : light.size) * ly;
            d.spot_angle = light.spot_angle;
            d.spot_smooth = light.spot_smooth;
            d.angle = light.angle;
            d.spread = light.spread;
            out._lights.push_back(d);
        }
        // camera
        if (!snapshot.active_camera) return error("the snapshot has no active camera");
        const auto cit = snapshot.cameras.find(*snapshot.active_camera);
        if (cit == snapshot.cameras.end()) return error("the active camera is missing");
        const contract::CameraDesc &cam = cit->second;
        psy_camera_desc c{};
        std::memcpy(c.camera_to_world, cam.transform.elements.data(), sizeof(c.camera_to_world));
        c.field_of_view = cam.field_of_view;
        c.horizontal_field_of_view = cam.horizontal_field_of_view;
        c.sensor_fit = cam.sensor_fit == contract::CameraSensorFit::horizontal ? 1u
                       : cam.sensor_fit == contract::CameraSensorFit::vertical ? 2u
                                                                               : 0u;
        c.lens_shift_x = cam.lens_shift_x;
        c.lens_shift_y = cam.lens_shift_y;
        c.near_clip = cam.near_clip;
        c.far_clip = cam.far_clip;
        c.projection = cam.projection == contract::CameraProjection::orthographic ? PSY_CAMERA_ORTHOGRAPHIC
                       : cam.projection == contract::CameraProjection::panorama   ? PSY_CAMERA_PANORAMA
                                                                                  : PSY_CAMERA_PERSPECTIVE;
        c.orthographic_scale = cam.orthographic_scale;
        c.aperture_radius = cam.aperture_radius;
        c.focal_distance = cam.focal_distance;
        c.aperture_blades = cam.aperture_blades;
        c.aperture_rotation = cam.aperture_rotation;
        c.aperture_ratio = cam.aperture_ratio;
        // descriptors over the owned arrays
        for (const FlatScene::Mesh &m : out._meshes) {
            psy_mesh_desc d{};
            d.positions = m.positions.data();
            d.normals = m.smooth ? m.normals.data() : nullptr;
            d.indices = m.indices.data();
            d.materials = m.per_triangle ? m.materials.data() : nullptr;
            d.vertex_count = std::uint32_t(m.positions.size() / 3u);
            d.triangle_count = std::uint32_t(m.indices.size() / 3u);
            d.smooth = m.smooth ? 1u : 0u;
            out._mesh_descs.push_back(d);
        }
        for (const FlatScene::Material &m : out._materials) {
            psy_material_desc d{};
            d.closures = m.closures.data();
            d.closure_count = std::uint32_t(m.closures.size());
            d.root = m.root;
            d.scalars = m.scalars.data();
            d.scalar_count = std::uint32_t(m.scalars.size());
            d.vectors = m.vectors.data();
            d.vector_count = std::uint32_t(m.vectors.size() / 3u);
            d.emission_sampling = m.emission_sampling;
            d.flags = m.flags;
            d.values = m.values.data();
            d.value_count = std::uint32_t(m.values.size());
            out._material_descs.push_back(d);
        }
        psy_scene_desc &s = out._desc;
        s = psy_scene_desc{};
        s.meshes = out._mesh_descs.data();
        s.instances = out._instances.data();
        s.materials = out._material_descs.data();
        s.lights = out._lights.data();
        s.mesh_count = std::uint32_t(out._mesh_descs.size());
        s.instance_count = std::uint32_t(out._instances.size());
        s.material_count = std::uint32_t(out._material_descs.size());
        s.light_count = std::uint32_t(out._lights.size());
        s.camera = c;
        // the constant environment is the background lights plus the world
        // shader's constant emission (make_environment_callables,
        // src/luisa/path_tracer_environment.cpp:39-50)
        copy3(s.background, Vec3f{background.x + world.x, background.y + world.y, background.z + world.z});
        s.world_visibility = snapshot.world_visibility_mask == ~std::uint32_t{0u}
                                 ? PSY_VISIBILITY_ALL
                                 : (snapshot.world_visibility_mask & PSY_VISIBILITY_ALL);
        s.revision = snapshot.revision;
        return true;
    }
};

bool flatten(const contract::SceneSnapshot &snapshot, const compiler::MaterialLibrary &library, FlatScene &out,
             std::vector<contract::RenderDiagnostic> &diagnostics) {
    out = FlatScene{};
    Flattener f{snapshot, library, out, diagnostics, {}};
    return f.run();
}

psy_render_settings to_psy_settings(const contract::RenderSettings &r, bool next_event_estimation) {
    psy_render_settings s{};
    psy_render_settings_default(&s);
    s.full_width = r.full_extent.width;
    s.full_height = r.full_extent.height;
    s.window_x = r.window.x;
    s.window_y = r.window.y;
    s.window_width = r.window.width;
    s.window_height = r.window.height;
    s.seed = r.seed;
    s.transparent_background = r.transparent_background ? 1u : 0u;
    s.pixel_filter = static_cast<std::uint32_t>(r.pixel_filter);
    s.filter_width = r.filter_width;
    s.pass_alpha_threshold = r.pass_alpha_threshold;
    const contract::PathIntegratorSettings &i = r.integrator;
    s.max_bounces = i.max_bounces;
    s.min_bounces = i.min_bounces;
    s.diffuse_bounces = i.diffuse_bounces;
    s.glossy_bounces = i.glossy_bounces;
    s.transmission_bounces = i.transmission_bounces;
    s.transparent_min_bounces = i.transparent_min_bounces;
    s.transparent_max_bounces = i.transparent_max_bounces;
    s.sample_clamp_direct = i.sample_clamp_direct;
    s.sample_clamp_indirect = i.sample_clamp_indirect;
    s.film_exposure = i.film_exposure;
    s.light_sampling_threshold = i.light_sampling_threshold;
    s.use_light_tree = i.use_light_tree ? 1u : 0u;
    s.direct_light_sampling = static_cast<std::uint32_t>(i.direct_light_sampling);
    s.next_event_estimation = next_event_estimation ? 1u : 0u;
    return s;
}

namespace {

// CompiledScene over a psy_scene (the device owns the uploaded scene).
class CudaCompiledScene final : public contract::CompiledScene {
public:
    CudaCompiledScene(psy_scene *scene, std::uint32_t light_count, bool glossy)
        : scene(scene), light_count(light_count), glossy(glossy) {}
    ~CudaCompiledScene() noexcept override { psy_scene_destroy(scene); }
    [[nodiscard]] std::uint64_t source_revision() const noexcept override { return psy_scene_source_revision(scene); }
    psy_scene *scene;
    std::uint32_t light_count;
    bool glossy;  // a material holds a glossy, glass or refraction closure
};

bool supported_pass(contract::PassKind kind) {
    switch (kind) {
    case contract::PassKind::combined:
    case contract::PassKind::normal:
    case contract::PassKind::albedo:
    case contract::PassKind::denoising_normal:
    case contract::PassKind::denoising_albedo:
    case contract::PassKind::sample_count:
        return true;
    default:
        return false;
    }
}

class CudaRenderSession final : public contract::RenderSession {
public:
    CudaRenderSession(psy_session *session, contract::RenderSettings settings, bool nee)
        : _session(session), _settings(std::move(settings)), _nee(nee) {}
    ~CudaRenderSession() noexcept override { psy_session_destroy(_session); }

    void reset(const contract::RenderSettings &settings) override {
        const psy_render_settings s = to_psy_settings(settings, _nee);
        if (psy_session_reset(_session, &s) == PSY_OK) _settings = settings;
    }

    // render_samples + write_passes (src/luisa/path_tracer_session.cpp:71-397)
    bool render_samples(const contract::SampleRange &range, contract::OutputSink &output) override {
        if (psy_session_render_samples(_session, range.first, range.count, range.offset, range.total) != PSY_OK)
            return false;
        const contract::PixelWindow window = effective_window();
        const std::size_t pixels = std::size_t(window.width) * window.height;
        std::vector<float> source(4u * pixels);
        output.begin(_settings);
        for (const contract::PassRequest &pass : _settings.passes) {
            std::uint32_t channels = 0u;
            if (psy_session_read_pass(_session, static_cast<std::uint32_t>(pass.kind), source.data(), source.size(),
                                      &channels) != PSY_OK) {
                output.end(true);
                return false;
            }
            // pass_channels (src/luisa/path_tracer_common.cpp:511-514): at
            // least one channel; channel c takes component min(c, 3) of the
            // pass value, and the sample count fills every component
            const std::uint32_t out_channels = std::max(pass.channels, 1u);
            std::vector<float> tile(pixels * out_channels);
            for (std::size_t i = 0; i < pixels; ++i)
                for (std::uint32_t c = 0; c < out_channels; ++c)
                    tile[i * out_channels + c] =
                        channels == 1u ? source[i] : source[4u * i + std::min<std::uint32_t>(c, 3u)];
            output.write(contract::PassTile{pass, window, _settings.full_extent, std::span<const float>{tile}});
        }
        output.end(false);
        return true;
    }

    void cancel() noexcept override { psy_session_cancel(_session); }

private:
    contract::PixelWindow effective_window() const {
        contract::PixelWindow w = _settings.window;
        if (w.width == 0u || w.height == 0u)
            w = {0u, 0u, _settings.full_extent.width, _settings.full_extent.height};
        return w;
    }

    psy_session *_session;
    contract::RenderSettings _settings;
    bool _nee;
};

}  // namespace

CudaPathTracerBackend::CudaPathTracerBackend(CudaPathTracerOptions options) : _options(options) {
    if (psy_context_create(options.device, &_context) != PSY_OK) {
        _context = nullptr;
        _context_error = psy_last_error();
    }
}

CudaPathTracerBackend::~CudaPathTracerBackend() noexcept {
    if (_context) psy_context_destroy(_context);
}

contract::SceneCompilation CudaPathTracerBackend::compile_scene(const contract::SceneSnapshot &snapshot) {
    contract::SceneCompilation result;
    if (!_context) {
        result.diagnostics.push_back({"no CUDA context: " + _context_error});
        return result;
    }
    // the reference's own material compiler (path_tracer_scene.cpp:122-139)
    compiler::ShaderCompiler shader_compiler{compiler::make_core_node_registry()};
    compiler::MaterialLibrary library;
    const compiler::MaterialLibraryUpdate update = library.update(snapshot, shader_compiler);
    if (!update.committed) {
        for (const auto &d : update.diagnostics)
            result.diagnostics.push_back({"Material " + std::to_string(d.material.value) + ": " + d.message});
        if (result.diagnostics.empty()) result.diagnostics.push_back({"the material library rejected the snapshot"});
        return result;
    }
    FlatScene flat;
    if (!flatten(snapshot, library, flat, result.diagnostics)) return result;
    psy_scene *scene = nullptr;
    if (psy_scene_compile(_context, &flat.desc(), &scene) != PSY_OK) {
        result.diagnostics.push_back({psy_last_error()});
        return result;
    }
    bool glossy = false;
    for (std::uint32_t i = 0; i < flat.desc().material_count; ++i) {
        const psy_material_desc &m = flat.desc().materials[i];
        for (std::uint32_t k = 0; k < m.closure_count; ++k)
            glossy = glossy || m.closures[k].op == PSY_CLOSURE_GLOSSY || m.closures[k].op == PSY_CLOSURE_GLASS ||
                     m.closures[k].op == PSY_CLOSURE_REFRACTION;
    }
    result.scene = std::make_unique<CudaCompiledScene>(scene, flat.desc().light_count, glossy);
    return result;
}

std::unique_ptr<contract::RenderSession> CudaPathTracerBackend::create_session(
    const contract::CompiledScene &scene, const contract::RenderSettings &settings) {
    const auto &compiled = static_cast<const CudaCompiledScene &>(scene);
    // the reference's rejections (src/luisa/path_tracer.cpp:23-76)
    if (settings.full_extent.width == 0u || settings.full_extent.height == 0u) return nullptr;
    if (!_options.next_event_estimation &&
        settings.integrator.direct_light_sampling != contract::DirectLightSampling::forward_path_tracing)
        return nullptr;
    if (settings.integrator.direct_light_sampling == contract::DirectLightSampling::forward_path_tracing &&
        compiled.light_count > 0u)
        return nullptr;
    for (const auto &pass : settings.passes)
        if (!supported_pass(pass.kind)) return nullptr;
    // glossy, glass and refraction closures render with Filter Glossy off and
    // both caustics on (the contract's defaults): the glossy blur and the
    // caustics lobe masks are not in the CUDA path
    if (compiled.glossy && (settings.integrator.filter_glossy > 0.0f || !settings.integrator.reflective_caustics ||
                            !settings.integrator.refractive_caustics))
        return nullptr;
    const psy_render_settings s = to_psy_settings(settings, _options.next_event_estimation);
    psy_session *session = nullptr;
    if (psy_session_create(compiled.scene, &s, &session) != PSY_OK) return nullptr;
    return std::make_unique<CudaRenderSession>(session, settings, _options.next_event_estimation);
}

}  // namespace psycles::cuda_backend
