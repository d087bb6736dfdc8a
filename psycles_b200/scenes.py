"""Scene snapshots and the seeded synthetic workloads.

`Scene` is the flattened SceneSnapshot the C ABI compiles
(psy_scene_desc): meshes, instances, compiled materials, analytic lights,
camera and a constant world colour.  `SceneDatabase.apply` mirrors the
reference's transactional deltas (src/contract/scene.cpp:427): a delta is
validated completely before a new revision is committed.

Workloads (all generated from seeds; no external data):
  * cornell_box()        closed box of 5 quads + a cube rotated 20 degrees
                         about Y, 0.73 / 0.65 / 0.12 albedos, one 0.5 x 0.5
                         emissive quad of strength 15, 40 degree pinhole
  * procedural_scene()   64 instances of 8 geodesic spheres (2k-40k
                         triangles, ~1M instanced), 32 random closure graphs,
                         point / spot / sun lights, constant background
  * many_light_scene()   ground + 200 boxes + emissive triangles scattered
                         in a 20^3 volume with log-uniform strengths
"""

from __future__ import annotations

import copy
import ctypes
import dataclasses
import math

import numpy as np

from . import _abi
from .materials import (CompiledMaterial, ShaderGraph, compile_surface_program, diffuse_material,
                        emission_material, glass_material, glossy_material, glossy_mixture_material,
                        random_material, value_graph_material)


@dataclasses.dataclass
class Mesh:
    positions: np.ndarray            # float32 [V, 3]
    indices: np.ndarray              # uint32 [T, 3]
    normals: np.ndarray | None = None  # float32 [V, 3]
    materials: np.ndarray | None = None  # uint32 [T]

    @property
    def triangle_count(self) -> int:
        return int(self.indices.shape[0])


@dataclasses.dataclass
class Instance:
    mesh: int
    material: int
    transform: np.ndarray = dataclasses.field(default_factory=lambda: np.eye(4, dtype=np.float32))
    visibility: int = _abi.VIS_ALL


@dataclasses.dataclass
class Light:
    type: int
    color: tuple = (1.0, 1.0, 1.0)
    power: float = 1.0
    position: tuple = (0.0, 0.0, 0.0)
    axis_x: tuple = (1.0, 0.0, 0.0)
    axis_y: tuple = (0.0, 1.0, 0.0)
    axis_z: tuple = (0.0, 0.0, 1.0)
    axis_scale: tuple = (1.0, 1.0, 1.0)
    radius: float = 0.0
    size_u: float = 1.0
    size_v: float = 1.0
    spot_angle: float = math.pi / 4
    spot_smooth: float = 0.0
    angle: float = 0.0
    spread: float = math.pi
    flags: int = _abi.LIGHT_FLAG_NORMALIZE
    max_bounces: int = 1024
    use_mis: bool = True            # LightDesc::use_mis
    visibility: int = _abi.VIS_ALL  # LightDesc::visibility_mask


@dataclasses.dataclass
class Camera:
    transform: np.ndarray  # camera-to-world 4x4 (column vectors)
    field_of_view: float = math.radians(40.0)
    horizontal_field_of_view: float = math.radians(40.0)
    sensor_fit: int = 2  # vertical
    lens_shift_x: float = 0.0
    lens_shift_y: float = 0.0
    near_clip: float = 1.0e-4
    far_clip: float = 1.0e5
    projection: int = 0  # _abi.CAMERA_*
    orthographic_scale: float = 1.0
    aperture_radius: float = 0.0
    focal_distance: float = 0.0
    aperture_blades: int = 0
    aperture_rotation: float = 0.0
    aperture_ratio: float = 1.0


@dataclasses.dataclass
class Scene:
    meshes: list[Mesh]
    instances: list[Instance]
    materials: list[CompiledMaterial]
    lights: list[Light]
    camera: Camera
    background: tuple = (0.0, 0.0, 0.0)
    world_visibility: int = _abi.VIS_ALL
    revision: int = 1
    # Cycles' GGX albedo tables (E: 1024 floats, Eavg: 32) for MULTI_GGX glossy
    # closures; the caller supplies the reference's own tables
    ggx_tables: tuple | None = None

    @property
    def instanced_triangles(self) -> int:
        return sum(self.meshes[i.mesh].triangle_count for i in self.instances)

    def to_desc(self) -> "SceneDescHandle":
        return SceneDescHandle(self)


def _column_major(m: np.ndarray) -> list[float]:
    """4x4 row-major numpy matrix (column vectors) -> Mat4f element order."""
    return [float(v) for v in np.asarray(m, dtype=np.float64).T.reshape(-1)]


def camera_desc(cam: "Camera") -> _abi.CameraDesc:
    """contract::CameraDesc of a Camera (perspective)."""
    c = _abi.CameraDesc()
    c.camera_to_world[:] = _column_major(cam.transform)
    c.field_of_view = cam.field_of_view
    c.horizontal_field_of_view = cam.horizontal_field_of_view
    c.sensor_fit = cam.sensor_fit
    c.lens_shift_x, c.lens_shift_y = cam.lens_shift_x, cam.lens_shift_y
    c.near_clip, c.far_clip = cam.near_clip, cam.far_clip
    c.projection, c.orthographic_scale = cam.projection, cam.orthographic_scale
    c.aperture_radius, c.focal_distance = cam.aperture_radius, cam.focal_distance
    c.aperture_blades, c.aperture_rotation, c.aperture_ratio = cam.aperture_blades, cam.aperture_rotation, cam.aperture_ratio
    return c


def _material_descs(mats) -> tuple:
    """psy_material_desc array of `mats`: every closure program, value
    stream, scalar block and vector block concatenated into one array each,
    and the descriptors filled as one structured numpy array (a scene may
    hold thousands of materials; per-material ctypes pointers would dominate
    its flattening)."""
    n = max(len(mats), 1)
    codes = [np.ascontiguousarray(cm.program.closures, dtype=np.uint32).reshape(-1, 6) for cm in mats]
    vals = [np.ascontiguousarray(cm.program.values, dtype=np.uint32).reshape(-1, 8) for cm in mats]
    scal = [np.ascontiguousarray(cm.parameters.scalars, dtype=np.float32).reshape(-1) for cm in mats]
    vecs = [np.ascontiguousarray(cm.parameters.vectors, dtype=np.float32).reshape(-1) for cm in mats]
    code_all = np.concatenate(codes) if codes else np.zeros((1, 6), np.uint32)
    val_all = np.concatenate(vals + [np.zeros((1, 8), np.uint32)])
    scal_all = np.concatenate(scal + [np.zeros(1, np.float32)])
    vec_all = np.concatenate(vecs + [np.zeros(3, np.float32)])
    c_counts = np.array([c.shape[0] for c in codes], np.uint64)
    w_counts = np.array([v.shape[0] for v in vals], np.uint64)
    s_counts = np.array([s.size for s in scal], np.uint64)
    v_counts = np.array([v.size for v in vecs], np.uint64)
    start = lambda counts: np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint64) if len(counts) else counts
    rec = np.zeros(n, dtype=_MATERIAL_DESC_DTYPE)
    if mats:
        rec["closures"] = np.uint64(code_all.ctypes.data) + start(c_counts) * np.uint64(24)
        rec["closure_count"] = c_counts
        rec["root"] = [cm.program.root for cm in mats]
        rec["scalars"] = np.uint64(scal_all.ctypes.data) + start(s_counts) * np.uint64(4)
        rec["scalar_count"] = s_counts
        rec["vector_count"] = v_counts // np.uint64(3)
        rec["vectors"] = np.uint64(vec_all.ctypes.data) + start(v_counts) * np.uint64(4)
        rec["emission_sampling"] = [cm.emission_sampling for cm in mats]
        rec["value_count"] = w_counts
        rec["values"] = np.uint64(val_all.ctypes.data) + start(w_counts) * np.uint64(32)
        rec["flags"] = [0 if getattr(cm, "use_bump_map_correction", True) else _abi.MATERIAL_NO_BUMP_MAP_CORRECTION
                        for cm in mats]
    descs = (_abi.MaterialDesc * n).from_buffer(rec)
    return descs, [rec, code_all, val_all, scal_all, vec_all]


# psy_material_desc of include/psycles_cuda.h on LP64 hosts (64 bytes)
_MATERIAL_DESC_DTYPE = np.dtype({
    "names": ["closures", "closure_count", "root", "scalars", "scalar_count", "vector_count", "vectors",
              "emission_sampling", "value_count", "values", "flags", "reserved"],
    "formats": [np.uint64, np.uint32, np.uint32, np.uint64, np.uint32, np.uint32, np.uint64, np.uint32, np.uint32,
                np.uint64, np.uint32, np.uint32],
    "offsets": [0, 8, 12, 16, 24, 28, 32, 40, 44, 48, 56, 60], "itemsize": 64})


class SceneDescHandle:
    """A psy_scene_desc plus the arrays it points into (kept alive here)."""

    def __init__(self, scene: Scene):
        keep = []
        meshes = (_abi.MeshDesc * max(len(scene.meshes), 1))()
        for i, m in enumerate(scene.meshes):
            p = np.ascontiguousarray(m.positions, dtype=np.float32)
            idx = np.ascontiguousarray(m.indices, dtype=np.uint32)
            n = None if m.normals is None else np.ascontiguousarray(m.normals, dtype=np.float32)
            mats = None if m.materials is None else np.ascontiguousarray(m.materials, dtype=np.uint32)
            keep += [p, idx, n, mats]
            meshes[i].positions = _abi.ptr(p)
            meshes[i].normals = _abi.ptr(n)
            meshes[i].indices = _abi.ptr(idx, ctypes.c_uint32)
            meshes[i].materials = _abi.ptr(mats, ctypes.c_uint32)
            meshes[i].vertex_count = p.shape[0]
            meshes[i].triangle_count = idx.shape[0]
            meshes[i].smooth = 1 if n is not None else 0
        instances = (_abi.InstanceDesc * max(len(scene.instances), 1))()
        for i, inst in enumerate(scene.instances):
            instances[i].object_to_world[:] = _column_major(inst.transform)
            instances[i].mesh = inst.mesh
            instances[i].material = inst.material
            instances[i].visibility = inst.visibility
        materials, material_arrays = _material_descs(scene.materials)
        keep += material_arrays
        lights = (_abi.LightDesc * max(len(scene.lights), 1))()
        for i, l in enumerate(scene.lights):
            d = lights[i]
            d.type, d.max_bounces, d.visibility = l.type, l.max_bounces, l.visibility
            d.flags = l.flags | (_abi.LIGHT_FLAG_USE_MIS if l.use_mis else 0)
            d.position[:] = l.position
            d.axis_x[:] = l.axis_x
            d.axis_y[:] = l.axis_y
            d.axis_z[:] = l.axis_z
            d.axis_scale[:] = l.axis_scale
            d.color[:] = l.color
            d.power, d.radius, d.size_u, d.size_v = l.power, l.radius, l.size_u, l.size_v
            d.spot_angle, d.spot_smooth, d.angle, d.spread = l.spot_angle, l.spot_smooth, l.angle, l.spread
        desc = _abi.SceneDesc()
        desc.meshes, desc.instances, desc.materials, desc.lights = meshes, instances, materials, lights
        desc.mesh_count = len(scene.meshes)
        desc.instance_count = len(scene.instances)
        desc.material_count = len(scene.materials)
        desc.light_count = len(scene.lights)
        cam = scene.camera
        desc.camera = camera_desc(cam)
        desc.background[:] = scene.background
        desc.world_visibility = scene.world_visibility
        desc.revision = scene.revision
        tables = ()
        if scene.ggx_tables is not None:
            tables = tuple(np.ascontiguousarray(t, dtype=np.float32) for t in scene.ggx_tables)
            desc.ggx_e = tables[0].ctypes.data_as(_abi.c_float_p)
            desc.ggx_eavg = tables[1].ctypes.data_as(_abi.c_float_p)
        self.desc = desc
        self._keep = (keep, meshes, instances, materials, lights, tables)

    @property
    def pointer(self):
        return ctypes.byref(self.desc)


# ------------------------------------------------------------ transforms

def translate(x, y, z) -> np.ndarray:
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m


def rotate_y(angle: float) -> np.ndarray:
    c, s = math.cos(angle), math.sin(angle)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
    return m


def scale(x, y, z) -> np.ndarray:
    return np.diag([x, y, z, 1.0])


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Camera-to-world matrix: the camera looks down its local -Z."""
    eye, target, up = (np.asarray(v, dtype=np.float64) for v in (eye, target, up))
    f = target - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = r, u, -f, eye
    return m


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    m = np.eye(4)
    m[:3, :3] = [[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                 [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                 [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]]
    return m


# ----------------------------------------------------------------- meshes

def quad(p0, p1, p2, p3) -> Mesh:
    """Two triangles (p0, p1, p2), (p0, p2, p3)."""
    pos = np.array([p0, p1, p2, p3], dtype=np.float32)
    return Mesh(pos, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))


def box_mesh(size=1.0) -> Mesh:
    h = size / 2.0
    v = np.array([[-h, -h, -h], [h, -h, -h], [h, h, -h], [-h, h, -h],
                  [-h, -h, h], [h, -h, h], [h, h, h], [-h, h, h]], dtype=np.float32)
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 4, 7, 3), (1, 2, 6, 5), (0, 1, 5, 4), (3, 7, 6, 2)]
    idx = []
    for a, b, c, d in faces:
        idx += [(a, b, c), (a, c, d)]
    return Mesh(v, np.array(idx, dtype=np.uint32))


def geodesic_sphere(frequency: int) -> Mesh:
    """Icosahedron with each face split into frequency^2 triangles, projected
    to the unit sphere; smooth normals are the positions."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                      [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    n = frequency
    positions = []
    indices = []
    for a, b, c in faces:
        A, B, C = verts[a], verts[b], verts[c]
        base = len(positions)
        row_start = []
        for i in range(n + 1):
            row_start.append(len(positions) - base)
            for j in range(n + 1 - i):
                p = A + (B - A) * (i / n) + (C - A) * (j / n)
                positions.append(p / np.linalg.norm(p))
        for i in range(n):
            for j in range(n - i):
                v0 = base + row_start[i] + j
                v1 = base + row_start[i + 1] + j
                v2 = base + row_start[i] + j + 1
                indices.append((v0, v1, v2))
                if j < n - i - 1:
                    v3 = base + row_start[i + 1] + j + 1
                    indices.append((v2, v1, v3))
    pos = np.array(positions, dtype=np.float32)
    return Mesh(pos, np.array(indices, dtype=np.uint32), normals=pos.copy())


# --------------------------------------------------------------- workloads

def _materials(graphs: list[ShaderGraph], sampling: int = _abi.EMISSION_AUTOMATIC) -> list[CompiledMaterial]:
    out = []
    for g in graphs:
        program, block = compile_surface_program(g)
        out.append(CompiledMaterial(g, program, block, sampling))
    return out


def cornell_box() -> Scene:
    """Closed box of 5 axis-aligned quads (2x2x2) + a cube rotated 20 degrees
    about Y; albedos 0.73 / 0.65 / 0.12 (grey, red, green); a 0.5 x 0.5
    emissive quad of strength 15 under the ceiling; 40 degree pinhole."""
    white = (0.73, 0.73, 0.73)
    red = (0.65, 0.05, 0.05)
    green = (0.12, 0.45, 0.15)
    mats = _materials([diffuse_material(white), diffuse_material(red), diffuse_material(green),
                       emission_material((1.0, 1.0, 1.0), 15.0)])
    meshes = [
        quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)),    # floor, normal +y
        quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)),    # ceiling, normal -y
        quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)),  # back wall, normal +z
        quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)),  # left wall, normal +x
        quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)),      # right wall, normal -x
        box_mesh(0.6),
        quad((-0.25, 1.98, -0.25), (0.25, 1.98, -0.25), (0.25, 1.98, 0.25), (-0.25, 1.98, 0.25)),  # light
    ]
    cube_xf = translate(0.3, 0.3, -0.2) @ rotate_y(math.radians(20.0))
    instances = [Instance(0, 0), Instance(1, 0), Instance(2, 0), Instance(3, 1), Instance(4, 2),
                 Instance(5, 0, cube_xf), Instance(6, 3)]
    cam = Camera(look_at((0.0, 1.0, 3.9), (0.0, 1.0, 0.0)), math.radians(40.0), math.radians(40.0), 0)
    return Scene(meshes, instances, mats, [], cam, background=(0.0, 0.0, 0.0))


def procedural_scene(seed: int = 0, frequencies=(10, 14, 18, 22, 27, 32, 38, 44), instances_per_mesh: int = 8,
                     material_count: int = 32, lights_per_type: int = 6, light_types=None) -> Scene:
    """64 seeded affine instances of 8 geodesic spheres (2k-40k triangles,
    ~1M instanced triangles, smooth normals), 32 random closure graphs over
    diffuse / emission / transparent / add / mix, point / spot / sun lights
    and a constant world colour."""
    rng = np.random.default_rng(seed)
    meshes = [geodesic_sphere(f) for f in frequencies]
    graphs = [random_material(rng, emission_probability=0.05) for _ in range(material_count)]
    mats = _materials(graphs)
    instances = []
    for mi in range(len(meshes)):
        for _ in range(instances_per_mesh):
            s = rng.uniform(0.6, 1.8)
            sx, sy, sz = s * rng.uniform(0.8, 1.25, 3)
            t = rng.uniform((-9, 0.5, -9), (9, 6, 9))
            xf = translate(*t) @ random_rotation(rng) @ scale(sx, sy, sz)
            instances.append(Instance(mi, int(rng.integers(0, material_count)), xf))
    if light_types is None:
        light_types = (_abi.LIGHT_POINT, _abi.LIGHT_SPOT, _abi.LIGHT_DISTANT, _abi.LIGHT_AREA)
    lights = []
    for lt in light_types:
        for _ in range(lights_per_type):
            color = tuple(float(c) for c in rng.uniform(0.5, 1.0, 3))
            if lt == _abi.LIGHT_DISTANT:
                d = rng.normal(size=3)
                d[1] = -abs(d[1]) - 0.5
                d /= np.linalg.norm(d)
                lights.append(Light(lt, color, float(rng.uniform(0.5, 2.0)), axis_z=tuple(d.tolist()),
                                    angle=float(math.radians(rng.uniform(0.5, 5.0)))))
            else:
                pos = tuple(rng.uniform((-10, 7, -10), (10, 12, 10)).tolist())
                xf = look_at(pos, (float(rng.uniform(-4, 4)), 0.0, float(rng.uniform(-4, 4))))
                flags = _abi.LIGHT_FLAG_NORMALIZE
                if lt == _abi.LIGHT_AREA and rng.random() < 0.5:
                    flags |= _abi.LIGHT_FLAG_ELLIPSE
                # half of the point / spot lamps have a finite radius, as a
                # disk or (LightDesc::is_sphere) a sphere
                radius = float(rng.uniform(0.1, 0.5)) if rng.random() < 0.5 else 0.0
                if lt in (_abi.LIGHT_POINT, _abi.LIGHT_SPOT) and radius > 0.0 and rng.random() < 0.5:
                    flags |= _abi.LIGHT_FLAG_SPHERE
                lights.append(Light(lt, color, float(rng.uniform(200.0, 800.0)), position=pos, radius=radius,
                                    axis_x=tuple(xf[:3, 0].tolist()), axis_y=tuple(xf[:3, 1].tolist()),
                                    axis_z=tuple(xf[:3, 2].tolist()),
                                    spot_angle=float(math.radians(rng.uniform(30, 90))),
                                    spot_smooth=float(rng.uniform(0.0, 0.5)),
                                    size_u=float(rng.uniform(0.5, 3.0)), size_v=float(rng.uniform(0.5, 3.0)),
                                    flags=flags))
    cam = Camera(look_at((0.0, 9.0, 24.0), (0.0, 2.0, 0.0)), math.radians(40.0), math.radians(40.0), 0)
    return Scene(meshes, instances, mats, lights, cam, background=(0.05, 0.06, 0.08))


def many_light_scene(seed: int = 0, boxes: int = 200, emitters: int = 10000, emission_materials: int = 10000) -> Scene:
    """Ground plane + 200 random boxes (2.4k triangles) + emissive triangles
    scattered uniformly in a 20^3 volume with log-uniform strengths in
    [1e-2, 1e2]; Lambertian albedo uniform in [0.2, 0.8]."""
    rng = np.random.default_rng(seed)
    mats_graphs = [diffuse_material(tuple(float(a) for a in rng.uniform(0.2, 0.8, 3))) for _ in range(16)]
    strengths = 10.0 ** rng.uniform(-2.0, 2.0, emission_materials)
    for s in strengths:
        mats_graphs.append(emission_material(tuple(float(c) for c in rng.uniform(0.6, 1.0, 3)), float(s)))
    mats = _materials(mats_graphs)
    meshes = [quad((-30, 0, -30), (-30, 0, 30), (30, 0, 30), (30, 0, -30)), box_mesh(1.0)]
    instances = [Instance(0, 0)]
    for _ in range(boxes):
        xf = translate(*rng.uniform((-10, 0.5, -10), (10, 3, 10))) @ rotate_y(float(rng.uniform(0, 2 * math.pi))) \
            @ scale(*rng.uniform(0.3, 2.0, 3))
        instances.append(Instance(1, int(rng.integers(0, 16)), xf))
    centers = rng.uniform((-10, 0.5, -10), (10, 20.5, 10), (emitters, 3))
    offsets = rng.normal(scale=0.15, size=(emitters, 3, 3))
    pos = (centers[:, None, :] + offsets).reshape(-1, 3).astype(np.float32)
    idx = np.arange(emitters * 3, dtype=np.uint32).reshape(-1, 3)
    tri_mats = (16 + rng.integers(0, emission_materials, emitters)).astype(np.uint32)
    meshes.append(Mesh(pos, idx, materials=tri_mats))
    instances.append(Instance(2, 16))
    cam = Camera(look_at((0.0, 12.0, 32.0), (0.0, 5.0, 0.0)), math.radians(45.0), math.radians(45.0), 0)
    return Scene(meshes, instances, mats, [], cam, background=(0.0, 0.0, 0.0))


def small_test_scene(seed: int = 0, transparent: bool = True, lights: bool = True) -> Scene:
    """A few-hundred-triangle scene exercising every closure, instance
    transforms, emissive meshes and point / spot / sun lights."""
    rng = np.random.default_rng(seed)
    graphs = [diffuse_material((0.7, 0.7, 0.7)), emission_material((1.0, 0.9, 0.8), 6.0)]
    for _ in range(6):
        graphs.append(random_material(rng, emission_probability=0.1,
                                      transparent_probability=0.3 if transparent else 0.0))
    mats = _materials(graphs)
    meshes = [quad((-4, 0, -4), (-4, 0, 4), (4, 0, 4), (4, 0, -4)), geodesic_sphere(3), box_mesh(1.0),
              quad((-0.5, 0, -0.5), (0.5, 0, -0.5), (0.5, 0, 0.5), (-0.5, 0, 0.5))]
    instances = [Instance(0, 0), Instance(3, 1, translate(0.0, 3.5, 0.0) @ rotate_y(0.3) @ np.diag([1, -1, 1, 1]))]
    for i in range(6):
        xf = translate(*rng.uniform((-2.5, 0.5, -2.5), (2.5, 2.0, 2.5))) @ random_rotation(rng) \
            @ scale(*rng.uniform(0.4, 1.0, 3))
        instances.append(Instance(1 + (i % 2), 2 + i, xf))
    ls = []
    if lights:
        ls = [Light(_abi.LIGHT_POINT, (1.0, 0.9, 0.8), 80.0, position=(2.0, 4.0, 1.0), radius=0.3),
              Light(_abi.LIGHT_SPOT, (0.8, 0.9, 1.0), 120.0, position=(-2.0, 4.5, 2.0), radius=0.25,
                    axis_x=(1, 0, 0), axis_y=(0, 0, 1), axis_z=(0, 1, 0), spot_angle=math.radians(70),
                    spot_smooth=0.3),
              Light(_abi.LIGHT_DISTANT, (1.0, 1.0, 0.9), 1.5, axis_z=(0.3, -0.9, 0.2), angle=math.radians(3.0)),
              Light(_abi.LIGHT_AREA, (0.9, 1.0, 0.9), 60.0, position=(3.0, 3.0, -1.0), axis_x=(1, 0, 0),
                    axis_y=(0, 0, 1), axis_z=(0, 1, 0), size_u=1.5, size_v=0.8),
              Light(_abi.LIGHT_AREA, (1.0, 0.8, 0.9), 40.0, position=(-3.0, 2.5, -1.5), axis_x=(0, 0, 1),
                    axis_y=(0, 1, 0), axis_z=(1, 0, 0), size_u=1.0, size_v=1.2,
                    flags=_abi.LIGHT_FLAG_NORMALIZE | _abi.LIGHT_FLAG_ELLIPSE)]
    cam = Camera(look_at((0.0, 3.0, 9.0), (0.0, 1.0, 0.0)), math.radians(40.0), math.radians(40.0), 0)
    return Scene(meshes, instances, mats, ls, cam, background=(0.1, 0.12, 0.15))


def lamp_scene(seed: int = 0) -> Scene:
    """Lamps in view: rectangle and ellipse area lamps (two stacked along the
    view axis, one facing away), finite-radius point and spot disks, a delta
    point and a sun, over a floor with boxes and a transparent pane; camera
    and BSDF rays hit the lamps directly."""
    rng = np.random.default_rng(seed)
    pane = ShaderGraph()
    pane.set_output(pane.transparent_bsdf((0.8, 0.9, 0.8)))
    graphs = [diffuse_material((0.7, 0.7, 0.7)), pane]
    for _ in range(3):
        graphs.append(random_material(rng, emission_probability=0.0, transparent_probability=0.2))
    mats = _materials(graphs)
    meshes = [quad((-6, 0, -6), (-6, 0, 6), (6, 0, 6), (6, 0, -6)), box_mesh(1.0),
              quad((-1, 0, 0), (1, 0, 0), (1, 2, 0), (-1, 2, 0))]
    instances = [Instance(0, 0), Instance(2, 1, translate(0.5, 0.0, 1.5))]
    for k in range(4):
        xf = translate(*rng.uniform((-3, 0.5, -3), (3, 1.5, 1))) @ rotate_y(float(rng.uniform(0, 6.28)))
        instances.append(Instance(1, 2 + (k % 3), xf))
    ls = [
        Light(_abi.LIGHT_AREA, (1.0, 0.9, 0.8), 30.0, position=(-1.5, 2.0, -2.0), size_u=1.2, size_v=0.8,
              axis_x=(1, 0, 0), axis_y=(0, 1, 0), axis_z=(0, 0, -1)),
        Light(_abi.LIGHT_AREA, (0.8, 0.9, 1.0), 25.0, position=(-1.3, 2.1, -3.0), size_u=1.0, size_v=1.0,
              axis_x=(1, 0, 0), axis_y=(0, 1, 0), axis_z=(0, 0, -1),
              flags=_abi.LIGHT_FLAG_NORMALIZE | _abi.LIGHT_FLAG_ELLIPSE),
        Light(_abi.LIGHT_AREA, (0.9, 1.0, 0.9), 40.0, position=(1.8, 1.5, -1.0), size_u=0.9, size_v=0.6,
              axis_x=(1, 0, 0), axis_y=(0, 1, 0), axis_z=(0, 0, 1)),
        Light(_abi.LIGHT_AREA, (1.0, 1.0, 1.0), 20.0, position=(0.0, 3.5, 0.0), size_u=2.0, size_v=2.0,
              axis_x=(1, 0, 0), axis_y=(0, 0, 1), axis_z=(0, 1, 0), flags=0),
        Light(_abi.LIGHT_POINT, (1.0, 0.8, 0.6), 60.0, position=(2.5, 2.5, -2.0), radius=0.35),
        Light(_abi.LIGHT_SPOT, (0.6, 0.8, 1.0), 90.0, position=(-2.5, 3.0, 0.5), radius=0.3,
              axis_x=(1, 0, 0), axis_y=(0, 0, 1), axis_z=(0.3, 1, 0.2), spot_angle=math.radians(80), spot_smooth=0.4),
        Light(_abi.LIGHT_POINT, (0.9, 0.9, 1.0), 15.0, position=(0.5, 1.0, -0.5)),
        Light(_abi.LIGHT_DISTANT, (1.0, 1.0, 0.9), 0.8, axis_z=(0.2, -0.9, -0.3), angle=math.radians(4.0)),
        Light(_abi.LIGHT_AREA, (1.0, 0.5, 0.5), 10.0, position=(0.0, 1.2, -4.0), size_u=1.0, size_v=1.0,
              axis_x=(1, 0, 0), axis_y=(0, 1, 0), axis_z=(0, 0, -1), use_mis=False),
        # sphere lamps (LightDesc::is_sphere)
        Light(_abi.LIGHT_POINT, (0.7, 1.0, 0.8), 50.0, position=(-0.8, 2.8, -1.5), radius=0.4,
              flags=_abi.LIGHT_FLAG_NORMALIZE | _abi.LIGHT_FLAG_SPHERE),
        Light(_abi.LIGHT_SPOT, (1.0, 0.9, 0.6), 70.0, position=(2.2, 3.2, 1.0), radius=0.35,
              axis_x=(1, 0, 0), axis_y=(0, 0, 1), axis_z=(-0.3, 1, -0.2), spot_angle=math.radians(60), spot_smooth=0.2,
              flags=_abi.LIGHT_FLAG_NORMALIZE | _abi.LIGHT_FLAG_SPHERE),
    ]
    cam = Camera(look_at((0.0, 2.0, 7.0), (0.0, 1.5, -1.0)), math.radians(45.0), math.radians(45.0), 0)
    return Scene(meshes, instances, mats, ls, cam, background=(0.05, 0.05, 0.08))


def glossy_scene(seed: int = 0) -> Scene:
    """The small test scene's geometry and lamps with glossy materials: GGX
    and Beckmann at roughness 0 (mirror), 0.1, 0.35 and 0.6 on the spheres
    and boxes (smooth-normal spheres exercise the specular-reflection normal
    correction), a glossy floor, and random diffuse + glossy, glossy +
    transparent and value-linked-roughness mixtures; one material turns the
    bump-map correction off."""
    rng = np.random.default_rng(seed)
    graphs = [glossy_material((0.8, 0.8, 0.8), 0.25), emission_material((1.0, 0.9, 0.8), 6.0),
              glossy_material((0.9, 0.8, 0.6), 0.0), glossy_material((0.6, 0.8, 0.9), 0.35, "BECKMANN"),
              glossy_material((0.9, 0.9, 0.9), 0.1), glossy_material((0.7, 0.9, 0.7), 0.6, "BECKMANN")]
    for _ in range(2):
        graphs.append(glossy_mixture_material(rng))
    base = small_test_scene(seed=seed)
    base.materials = _materials(graphs)
    base.materials[3].use_bump_map_correction = False
    return base


def glass_scene(seed: int = 0) -> Scene:
    """The small test scene's geometry and lamps with dielectric materials:
    smooth (singular) and rough GGX glass, Beckmann glass, a tinted glass,
    smooth and rough refraction, and refraction mixed with diffuse; the
    spheres are closed, so paths enter and leave them (back-facing hits with
    the inverted IOR) and reach total internal reflection."""
    from .materials import ShaderGraph as _G
    graphs = [diffuse_material((0.7, 0.7, 0.7)), emission_material((1.0, 0.9, 0.8), 6.0),
              glass_material((1.0, 1.0, 1.0), 0.0, 1.5), glass_material((0.95, 0.95, 1.0), 0.2, 1.45),
              glass_material((0.8, 1.0, 0.85), 0.3, 1.33, "BECKMANN"), glass_material((1.0, 0.7, 0.5), 0.0, 1.6)]
    g = _G()
    g.set_output(g.refraction_bsdf((0.9, 0.95, 1.0), 0.0, 1.4))
    graphs.append(g)
    g = _G()
    g.set_output(g.mix_shader(0.3, g.refraction_bsdf((1.0, 1.0, 1.0), 0.25, 1.5, "BECKMANN"),
                              g.diffuse_bsdf((0.6, 0.3, 0.2))))
    graphs.append(g)
    base = small_test_scene(seed=seed)
    base.materials = _materials(graphs)
    return base


def value_graph_scene(seed: int = 0) -> Scene:
    """The small test scene's geometry and lamps with materials whose closure
    inputs are linked to value nodes (RGB / Value nodes through colour
    blends, float math, conversions, separate / combine RGB into rough
    diffuse colours, mix factors and emission strengths), plus rough and
    smooth diffuse walls."""
    rng = np.random.default_rng(seed)
    graphs = [diffuse_material((0.7, 0.7, 0.7), 0.5), emission_material((1.0, 0.9, 0.8), 6.0)]
    for _ in range(6):
        graphs.append(value_graph_material(rng))
    base = small_test_scene(seed=seed)
    base.materials = _materials(graphs)
    return base


def _f32_view(eye, target) -> np.ndarray:
    """Camera-to-world matrix looking from `eye` at `target` (+y up, camera
    space -z forward), evaluated in float32 in the order a C++ float
    implementation takes: unit(v) = v * (1 / sqrt(max(dot(v, v), 1e-20)))."""
    f = np.float32

    def unit(v):
        d = f(v[0] * v[0]) + f(v[1] * v[1])
        d = f(d + f(v[2] * v[2]))
        s = f(f(1.0) / f(np.sqrt(max(d, f(1e-20)))))
        return [f(v[0] * s), f(v[1] * s), f(v[2] * s)]

    def cross(a, b):
        return [f(f(a[1] * b[2]) - f(a[2] * b[1])), f(f(a[2] * b[0]) - f(a[0] * b[2])),
                f(f(a[0] * b[1]) - f(a[1] * b[0]))]

    e = [f(v) for v in eye]
    t = [f(v) for v in target]
    forward = unit([f(t[i] - e[i]) for i in range(3)])
    right = unit(cross(forward, [f(0), f(1), f(0)]))
    back = [-forward[0], -forward[1], -forward[2]]
    up = unit(cross(back, right))
    m = np.eye(4, dtype=np.float32)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = right, up, back, e
    return m


def luisa_demo_scene(variant: int = 0) -> Scene:
    """The Cornell-style room of the reference's Luisa demo
    (examples/render_luisa_demo.cpp:203-305) in this scene model: a floor and
    three walls in one mesh with per-triangle materials, a cube scaled to a
    block, rough diffuse plaster / red / green / blue, a 1.8 m square area
    light under the open ceiling and a background light, 47 degree camera.
    Variant 1 (or True): the block's colour is an RGB-node mix and its
    roughness float math; variant 2: the block is a GGX Glossy BSDF and the
    plaster a mix of rough diffuse and Beckmann glossy; variant 4: the block
    is a rough GGX Glass BSDF (IOR 1.45) and the plaster a mix of rough
    diffuse and Beckmann Refraction (IOR 1.3) -- as
    tests/adapter/adapter_probe.cpp builds them."""
    f = np.float32
    variant = int(variant)
    graphs = [diffuse_material((0.72, 0.72, 0.72), 0.35), diffuse_material((0.72, 0.06, 0.035), 0.45),
              diffuse_material((0.04, 0.54, 0.12), 0.45)]
    if variant == 2:
        g = ShaderGraph()
        g.set_output(g.mix_shader(0.25, g.diffuse_bsdf((0.72, 0.72, 0.72), 0.35),
                                  g.glossy_bsdf((0.9, 0.9, 0.85), 0.2, "BECKMANN")))
        graphs[0] = g
    if variant == 4:
        g = ShaderGraph()
        g.set_output(g.mix_shader(0.3, g.diffuse_bsdf((0.72, 0.72, 0.72), 0.35),
                                  g.refraction_bsdf((0.9, 0.9, 0.85), 0.2, 1.3, "BECKMANN")))
        graphs[0] = g
    if variant == 1:
        g = ShaderGraph()
        color = g.mix_color(0.3, g.rgb((0.035, 0.18, 0.85)), g.rgb((0.9, 0.5, 0.1)))
        g.set_output(g.diffuse_bsdf(color, g.math("clamp", g.math("multiply", g.value(0.6), 0.5))))
        graphs.append(g)
    elif variant == 2:
        graphs.append(glossy_material((0.035, 0.18, 0.85), 0.3, "GGX"))
    elif variant == 4:
        graphs.append(glass_material((0.9, 0.95, 1.0), 0.15, 1.45, "GGX"))
    else:
        graphs.append(diffuse_material((0.035, 0.18, 0.85), 0.16))
    mats = _materials(graphs)

    def quads(qs):
        pos, idx = [], []
        for q in qs:
            b = len(pos)
            pos += q
            idx += [(b, b + 1, b + 2), (b, b + 2, b + 3)]
        return np.array(pos, np.float32), np.array(idx, np.uint32)

    rp, ri = quads([[(-3, 0, 2.5), (3, 0, 2.5), (3, 0, -3), (-3, 0, -3)],
                    [(-3, 0, -3), (3, 0, -3), (3, 4.5, -3), (-3, 4.5, -3)],
                    [(-3, 0, 2.5), (-3, 0, -3), (-3, 4.5, -3), (-3, 4.5, 2.5)],
                    [(3, 0, -3), (3, 0, 2.5), (3, 4.5, 2.5), (3, 4.5, -3)]])
    cp, ci = quads([[(-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)],
                    [(1, -1, -1), (-1, -1, -1), (-1, 1, -1), (1, 1, -1)],
                    [(-1, -1, -1), (-1, -1, 1), (-1, 1, 1), (-1, 1, -1)],
                    [(1, -1, 1), (1, -1, -1), (1, 1, -1), (1, 1, 1)],
                    [(-1, 1, 1), (1, 1, 1), (1, 1, -1), (-1, 1, -1)]])
    meshes = [Mesh(rp, ri, materials=np.array([0, 0, 0, 0, 1, 1, 2, 2], np.uint32)), Mesh(cp, ci)]
    block = np.eye(4, dtype=np.float32)
    block[0, 0], block[1, 1], block[2, 2] = f(0.72), f(1.15), f(0.72)
    block[:3, 3] = [f(0.35), f(1.15), f(-0.55)]
    instances = [Instance(0, 0), Instance(1, 3, block)]
    pi = f(3.14159265358979323846)
    fov = f(f(f(47.0) * pi) / f(180.0))
    cam = Camera(_f32_view((0.0, 2.05, 7.0), (0.0, 1.5, -0.8)), float(fov), float(fov), 2, near_clip=1.0e-3,
                 far_clip=100.0)
    light = Light(_abi.LIGHT_AREA, (1.0, 0.82, 0.62), 18.0, position=(-0.4, 4.25, -0.6), axis_x=(1, 0, 0),
                  axis_y=(0, 0, 1), axis_z=(0, 1, 0), radius=1.8, size_u=1.8, size_v=1.8, spread=float(pi),
                  spot_smooth=0.15, flags=_abi.LIGHT_FLAG_NORMALIZE | _abi.LIGHT_FLAG_SPHERE)
    return Scene(meshes, instances, mats, [light], cam, background=(0.008, 0.012, 0.025))


def render_settings(width: int, height: int, max_bounces: int = 4, seed: int = 0, **overrides) -> _abi.RenderSettings:
    s = _abi.default_settings()
    s.full_width, s.full_height = width, height
    s.max_bounces = max_bounces
    s.seed = seed
    for k, v in overrides.items():
        setattr(s, k, v)
    return s


class SceneDatabase:
    """Atomic snapshot store: apply() validates the whole delta and commits a
    new revision, or raises and keeps the previous snapshot."""

    def __init__(self, scene: Scene):
        self.snapshot = scene

    def apply(self, material_graphs: dict[int, ShaderGraph] | None = None,
              instance_transforms: dict[int, np.ndarray] | None = None) -> Scene:
        nxt = copy.copy(self.snapshot)
        nxt.materials = list(self.snapshot.materials)
        nxt.instances = list(self.snapshot.instances)
        for index, graph in (material_graphs or {}).items():
            if not 0 <= index < len(nxt.materials):
                raise ValueError(f"material {index} does not exist")
            program, block = compile_surface_program(graph)
            nxt.materials[index] = CompiledMaterial(graph, program, block, nxt.materials[index].emission_sampling)
        for index, xf in (instance_transforms or {}).items():
            if not 0 <= index < len(nxt.instances):
                raise ValueError(f"instance {index} does not exist")
            xf = np.asarray(xf, dtype=np.float64)
            if xf.shape != (4, 4) or not np.isfinite(xf).all():
                raise ValueError("instance transform must be a finite 4x4 matrix")
            nxt.instances[index] = dataclasses.replace(nxt.instances[index], transform=xf)
        nxt.revision = self.snapshot.revision + 1
        self.snapshot = nxt
        return nxt
