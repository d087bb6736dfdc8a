"""Writes a Blender scene bundle -- the directory that the reference's
exporter (tools/export_psycles_scene.py) emits and its importer
load_blender_scene_bundle reads (src/adapter/blender_scene.cpp:285-1622):
`scene.json` (schema "psycles.blender-scene.v1") plus `geometry.bin`
("PSYGEO1\\0" followed by the little-endian sections that each geometry's
`positions` / `normals` / `uv` / `generated` / `indices` /
`triangle_material_slots` / `triangle_random_per_island` entries point at by
byte offset; point-domain attributes in v1).

Test infrastructure: no exported bundle is in the reference checkout, so the
tests write this Cornell-style room with the node trees Blender would export
(Diffuse, Glossy, Mix Shader, Emission and RGB / Value nodes, a Background
world) and render it through the importer, the reference's material compiler
and the CUDA backend; the expectations below restate what the importer and
the adapter must make of it."""

from __future__ import annotations

import json
import math
import pathlib

import numpy as np

from psycles_b200 import _abi, scenes

WIDTH, HEIGHT = 96, 72
SEED = 7
MAX_BOUNCES = 5
WORLD_COLOR = (0.02, 0.03, 0.05)
WORLD_STRENGTH = 0.8
LAMP = dict(position=(0.45, 1.55, 0.35), color=(1.0, 0.85, 0.7), energy=6.0, size=0.08)

WHITE = (0.73, 0.73, 0.73)
RED = (0.65, 0.05, 0.05)
GREEN = (0.12, 0.45, 0.15)
GLOSSY = (0.9, 0.8, 0.6)
GLOSSY_ROUGHNESS = 0.3
MIX_FACTOR = 0.35
LIGHT_STRENGTH = 15.0


def _socket(identifier, kind, default=None, linked=False, name=None):
    s = {"identifier": identifier, "name": name or identifier, "type": kind, "linked": linked}
    if default is not None:
        s["default"] = default
    return s


def _node(name, kind, inputs=(), outputs=(), properties=None):
    return {"name": name, "label": "", "type": kind, "bl_idname": "", "inputs": list(inputs),
            "outputs": list(outputs), "properties": properties or {}, "special": {}, "image": None,
            "node_tree": None}


def _link(from_node, from_socket, to_node, to_socket):
    return {"from_node": from_node, "from_socket": from_socket, "to_node": to_node, "to_socket": to_socket}


def _rgba(c):
    return [float(c[0]), float(c[1]), float(c[2]), 1.0]


def _diffuse(name, color, linked_color=False):
    return _node(name, "BSDF_DIFFUSE",
                 [_socket("Color", "NodeSocketColor", _rgba(color), linked_color),
                  _socket("Roughness", "NodeSocketFloat", 0.0),
                  _socket("Normal", "NodeSocketVector", [0.0, 0.0, 0.0])],
                 [_socket("BSDF", "NodeSocketShader", linked=True)])


def _tree(name, root_node, root_socket, nodes, links=()):
    return {"name": name, "surface_root": {"node": root_node, "socket": root_socket}, "volume_root": None,
            "displacement_root": None, "links": list(links), "nodes": list(nodes)}


def _material(name, tree):
    return {"name": name, "use_bump_map_correction": True, "emission_sampling": "AUTO",
            "volume_sampling": "MULTIPLE_IMPORTANCE", "displacement_method": "BUMP", "node_tree": tree}


def materials_json():
    """White: Diffuse.  Red: Diffuse whose colour comes from an RGB node (a
    linked socket, so a value instruction).  Green: Mix Shader of a Diffuse
    and a GGX Glossy, its factor from a Value node.  Light: Emission."""
    white = _tree("White", "Diffuse BSDF", "BSDF", [_diffuse("Diffuse BSDF", WHITE)])
    red = _tree("Red", "Diffuse BSDF", "BSDF",
                [_node("RGB", "RGB", [], [_socket("Color", "NodeSocketColor", _rgba(RED), True)]),
                 _diffuse("Diffuse BSDF", RED, linked_color=True)],
                [_link("RGB", "Color", "Diffuse BSDF", "Color")])
    glossy = _node("Glossy BSDF", "BSDF_GLOSSY",
                   [_socket("Color", "NodeSocketColor", _rgba(GLOSSY)),
                    _socket("Roughness", "NodeSocketFloat", GLOSSY_ROUGHNESS),
                    _socket("Normal", "NodeSocketVector", [0.0, 0.0, 0.0])],
                   [_socket("BSDF", "NodeSocketShader", linked=True)], {"distribution": "GGX"})
    mix = _node("Mix Shader", "MIX_SHADER",
                [_socket("Fac", "NodeSocketFloat", 0.5, True),
                 _socket("Shader", "NodeSocketShader", linked=True),
                 _socket("Shader_001", "NodeSocketShader", linked=True, name="Shader")],
                [_socket("Shader", "NodeSocketShader", linked=True)])
    value = _node("Value", "VALUE", [], [_socket("Value", "NodeSocketFloat", MIX_FACTOR, True)])
    green = _tree("Green", "Mix Shader", "Shader", [_diffuse("Diffuse BSDF", GREEN), glossy, value, mix],
                  [_link("Value", "Value", "Mix Shader", "Fac"),
                   _link("Diffuse BSDF", "BSDF", "Mix Shader", "Shader"),
                   _link("Glossy BSDF", "BSDF", "Mix Shader", "Shader_001")])
    light = _tree("Light", "Emission", "Emission",
                  [_node("Emission", "EMISSION",
                         [_socket("Color", "NodeSocketColor", [1.0, 1.0, 1.0, 1.0]),
                          _socket("Strength", "NodeSocketFloat", LIGHT_STRENGTH)],
                         [_socket("Emission", "NodeSocketShader", linked=True)])])
    return [_material("White", white), _material("Red", red), _material("Green", green),
            _material("Light", light)]


def room_geometry():
    """The five walls in one mesh (slots White, Red, Green per triangle),
    the cube and the lamp quad, as scenes.cornell_box() lays them out."""
    box = scenes.cornell_box()
    walls = box.meshes[:5]
    positions = np.concatenate([m.positions for m in walls]).astype(np.float32)
    indices, offset = [], 0
    for m in walls:
        indices.append(m.indices + offset)
        offset += m.positions.shape[0]
    indices = np.concatenate(indices).astype(np.uint32)
    # floor, ceiling, back wall: White; left wall: Red; right wall: Green
    slots = np.array([0, 0, 0, 0, 0, 0, 1, 1, 2, 2], np.uint32)
    room = scenes.Mesh(positions, indices, None, slots)
    return [("Room", room, ["White", "Red", "Green"]), ("Cube", box.meshes[5], ["White"]),
            ("Lamp", box.meshes[6], ["Light"])]


def _column_major(m):
    return [float(v) for v in np.asarray(m, np.float64).T.reshape(-1)]


def cube_transform():
    return scenes.translate(0.3, 0.3, -0.2) @ scenes.rotate_y(math.radians(20.0))


def camera_transform():
    return scenes.look_at((0.0, 1.0, 3.9), (0.0, 1.0, 0.0))


def write_bundle(directory, *, world_tree: bool = True, schema: str = "psycles.blender-scene.v1") -> pathlib.Path:
    """Writes scene.json and geometry.bin into `directory` and returns it.
    With `world_tree` the world is a Background node tree (colour and
    strength); without, the importer builds its emission graph from the
    world's `color`."""
    directory = pathlib.Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    blob = bytearray(b"PSYGEO1\0")

    def section(array):
        offset = len(blob)
        blob.extend(np.ascontiguousarray(array).tobytes())
        return {"offset": offset}

    geometries = []
    for name, mesh, slots in room_geometry():
        v = mesh.positions.shape[0]
        t = mesh.triangle_count
        normals = np.zeros((v, 3), np.float32)
        geometries.append({
            "name": name, "triangle_count": t, "vertex_count": v,
            "positions": section(mesh.positions.astype("<f4")),
            "normals": section(normals.astype("<f4")),
            "uv": section(np.zeros((v, 2), "<f4")),
            "generated": section(mesh.positions.astype("<f4")),
            "indices": section(mesh.indices.astype("<u4")),
            "triangle_material_slots": section((mesh.materials if mesh.materials is not None
                                                else np.zeros(t, np.uint32)).astype("<u4")),
            "triangle_smooth": section(np.zeros(t, "<u4")),
            "triangle_random_per_island": section(np.zeros(t, "<f4")),
            "uv_layers": [],
            "material_slots": slots,
        })
    identity = np.eye(4)
    instances = [
        {"name": "Room", "geometry": 0, "transform": _column_major(identity), "random_id": 0},
        {"name": "Cube", "geometry": 1, "transform": _column_major(cube_transform()), "random_id": 0},
        {"name": "Lamp Quad", "geometry": 2, "transform": _column_major(identity), "random_id": 0},
    ]
    lamp_transform = scenes.translate(*LAMP["position"])
    lights = [{"name": "Point", "type": "POINT", "transform": _column_major(lamp_transform),
               "color": list(LAMP["color"]), "energy": LAMP["energy"], "size": LAMP["size"],
               "use_soft_falloff": False, "node_tree": None}]
    world = {"name": "World", "color": list(WORLD_COLOR)}
    if world_tree:
        world["node_tree"] = _tree("World", "Background", "Background", [
            _node("Background", "BACKGROUND",
                  [_socket("Color", "NodeSocketColor", _rgba(WORLD_COLOR)),
                   _socket("Strength", "NodeSocketFloat", WORLD_STRENGTH)],
                  [_socket("Background", "NodeSocketShader", linked=True)])])
    fov = math.radians(40.0)
    document = {
        "schema": schema,
        "images": [],
        "node_groups": [],
        "materials": materials_json(),
        "render": {
            "width": WIDTH, "height": HEIGHT, "percentage": 100, "filter_width": 1.5,
            "pixel_filter_type": "BLACKMAN_HARRIS", "transparent": False,
            "cycles": {"samples": 16, "seed": SEED, "max_bounces": MAX_BOUNCES, "use_light_tree": False,
                       "use_adaptive_sampling": False, "use_denoising": False},
        },
        "camera": {"name": "Camera", "type": "PERSP", "sensor_fit": "VERTICAL", "angle": fov, "angle_x": fov,
                   "angle_y": fov, "transform": _column_major(camera_transform()), "clip_start": 1.0e-4,
                   "clip_end": 1.0e5, "shift_x": 0.0, "shift_y": 0.0, "dof": {"enabled": False}},
        "geometries": geometries,
        "instances": instances,
        "lights": lights,
        "world": world,
    }
    (directory / "scene.json").write_text(json.dumps(document, indent=1))
    (directory / "geometry.bin").write_bytes(bytes(blob))
    return directory


def room_desc_arrays():
    """Positions, indices and per-triangle materials of the bundle's meshes,
    for the field-by-field comparison with the flattened snapshot."""
    return [(m.positions.astype(np.float32), m.indices.astype(np.uint32), m.materials)
            for _, m, _ in room_geometry()]


def lamp_expectation():
    """The psy_light_desc fields the adapter derives from the bundle's point
    light (LightDesc via blender_scene.cpp:1360-1490: power = energy x
    2^exposure, spot and spread defaults, use_soft_falloff false -> a sphere,
    normalize and MIS on)."""
    return dict(type=_abi.LIGHT_POINT, position=LAMP["position"], color=LAMP["color"], power=LAMP["energy"],
                radius=LAMP["size"], size_u=LAMP["size"], size_v=LAMP["size"],
                flags=_abi.LIGHT_FLAG_NORMALIZE | _abi.LIGHT_FLAG_SPHERE | _abi.LIGHT_FLAG_USE_MIS,
                spot_angle=0.78539816339, spot_smooth=0.15, spread=3.14159265, max_bounces=1024)
