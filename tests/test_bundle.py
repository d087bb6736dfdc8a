"""Blender scene bundles through the reference's importer into the CUDA
backend's adapter (not gpu-marked).

The reference's load_blender_scene_bundle (src/adapter/blender_scene.cpp:285)
reads the directory its exporter writes; callers such as
examples/render_blender_scene.cpp hand the SceneSnapshot it returns to a
RendererBackend.  Here the importer is compiled where it lies against the
yyjson-compatible reader tests/adapter/yyjson.h, with the reference's own
importer tests (tests/test_blender_import.cpp, test_blender_muted_node.cpp,
test_blender_curve_import.cpp) linked against it to pin that reader.  A
Cornell-style room written as a bundle (tests/adapter/blender_bundle.py:
Diffuse, RGB-fed Diffuse, Mix of Diffuse and GGX Glossy by a Value node,
Emission, a point light, a Background world) is imported, compiled by the
reference's MaterialLibrary and flattened by CudaPathTracerBackend's
flatten(); the flattened scene must hold exactly the room, and the oracle
must render it.  The GPU render of the same bundle is in
tests/test_bundle_gpu.py.

Needs oracle/_ref (`make -C oracle adapter`, built where the reference tree
is present); skipped without it."""

import ctypes
import math
import pathlib
import subprocess
import sys

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes

ROOT = pathlib.Path(__file__).resolve().parent.parent
REF_BUILD = ROOT / "oracle" / "_ref"
PROBE = REF_BUILD / "libpsycles_adapter_probe.so"
sys.path.insert(0, str(ROOT / "tests" / "adapter"))
import blender_bundle as bundle  # noqa: E402

pytestmark = pytest.mark.skipif(not PROBE.exists(), reason="adapter probe not built (make -C oracle adapter)")


def bundle_probe():
    from test_adapter import probe
    lib = probe()
    lib.probe_bundle_flatten.restype = ctypes.c_void_p
    lib.probe_bundle_flatten.argtypes = [ctypes.c_char_p, ctypes.POINTER(_abi.RenderSettings),
                                         ctypes.POINTER(ctypes.c_uint32), ctypes.c_char_p, ctypes.c_size_t]
    return lib


class FlattenedBundle:
    """A bundle imported, compiled and flattened by the probe; `.pointer`
    as scenes.SceneDescHandle, `.settings` the psy_render_settings the
    adapter makes of the bundle's render settings."""

    def __init__(self, directory):
        self.lib = bundle_probe()
        self.settings = _abi.RenderSettings()
        samples = ctypes.c_uint32(0)
        err = ctypes.create_string_buffer(512)
        self.handle = self.lib.probe_bundle_flatten(str(directory).encode(), ctypes.byref(self.settings),
                                                    ctypes.byref(samples), err, 512)
        self.error = err.value.decode()
        self.samples = samples.value
        if self.handle:
            self.desc = self.lib.probe_flat_desc(self.handle).contents
            self.pointer = ctypes.pointer(self.desc)

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.probe_flat_destroy(self.handle)


def arr(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0)


@pytest.mark.parametrize("name", ["blender_import", "blender_muted_node", "blender_curve_import"])
def test_reference_importer_tests_pass_on_this_reader(name):
    exe = REF_BUILD / f"test_{name}"
    if not exe.exists():
        pytest.skip("reference importer tests not built")
    done = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert done.returncode == 0, done.stdout[-2000:] + done.stderr[-2000:]


@pytest.mark.parametrize("world_tree", [True, False])
def test_bundle_flattens_to_the_room(tmp_path, world_tree):
    flat = FlattenedBundle(bundle.write_bundle(tmp_path / "room", world_tree=world_tree))
    assert flat.handle, flat.error
    d = flat.desc
    assert (d.mesh_count, d.instance_count, d.material_count, d.light_count) == (3, 3, 4, 1)
    # meshes: the room with one material per triangle, the cube and the lamp quad
    for i, (positions, indices, materials) in enumerate(bundle.room_desc_arrays()):
        m = d.meshes[i]
        assert (m.vertex_count, m.triangle_count, m.smooth) == (positions.shape[0], indices.shape[0], 0)
        assert np.array_equal(arr(m.positions, m.vertex_count * 3), positions.reshape(-1))
        assert np.array_equal(arr(m.indices, m.triangle_count * 3), indices.reshape(-1))
        if materials is None:
            assert not m.materials
        else:
            # White, Red, Green are materials 0, 1, 2 (MaterialId order)
            assert np.array_equal(arr(m.materials, m.triangle_count), materials)
    xfs = [np.eye(4), bundle.cube_transform(), np.eye(4)]
    for i, (mesh, material) in enumerate(((0, 0), (1, 0), (2, 3))):
        inst = d.instances[i]
        assert (inst.mesh, inst.material, inst.visibility) == (mesh, material, _abi.VIS_ALL)
        assert np.array_equal(np.array(inst.object_to_world[:], np.float32),
                              np.array(scenes._column_major(xfs[i]), np.float32))
    # materials: the closure trees the reference compiler made of the nodes
    ops = [[d.materials[k].closures[j].op for j in range(d.materials[k].closure_count)] for k in range(4)]
    assert ops[0] == [_abi.CLOSURE_DIFFUSE]
    assert ops[1] == [_abi.CLOSURE_DIFFUSE]
    red = d.materials[1].closures[0]
    assert red.color & _abi.INPUT_VALUE, "the RGB node feeds the colour through the value stream"
    assert sorted(ops[2]) == sorted([_abi.CLOSURE_DIFFUSE, _abi.CLOSURE_GLOSSY, _abi.CLOSURE_MIX])
    assert ops[3] == [_abi.CLOSURE_EMISSION]
    # the lamp: LightDesc of the bundle's point light
    lamp, want = d.lights[0], bundle.lamp_expectation()
    for key in ("type", "flags", "max_bounces"):
        assert getattr(lamp, key) == want[key], key
    for key in ("power", "radius", "size_u", "size_v", "spot_angle", "spot_smooth", "spread"):
        assert getattr(lamp, key) == np.float32(want[key]), key
    assert np.array_equal(np.array(lamp.position[:], np.float32), np.array(want["position"], np.float32))
    assert np.array_equal(np.array(lamp.color[:], np.float32), np.array(want["color"], np.float32))
    # the camera, as the scene model's camera_desc of the same view
    want_cam = scenes.camera_desc(scenes.Camera(bundle.camera_transform(), math.radians(40.0),
                                                math.radians(40.0), 2))
    assert bytes(d.camera) == bytes(want_cam)
    # the world: Background colour x strength, or the importer's emission
    # graph of the world colour at strength 1
    strength = np.float32(bundle.WORLD_STRENGTH if world_tree else 1.0)
    want_bg = np.array(bundle.WORLD_COLOR, np.float32) * strength
    assert np.array_equal(np.array(d.background[:], np.float32), want_bg)
    # render settings: the bundle's seed, filter and bounce limit
    s = flat.settings
    assert (s.full_width, s.full_height, s.seed, s.max_bounces) == (bundle.WIDTH, bundle.HEIGHT, bundle.SEED,
                                                                    bundle.MAX_BOUNCES)
    assert s.pixel_filter == 2 and s.filter_width == np.float32(1.5)  # Blackman-Harris
    assert flat.samples == 16


def test_oracle_renders_the_flattened_bundle(tmp_path):
    flat = FlattenedBundle(bundle.write_bundle(tmp_path / "room"))
    assert flat.handle, flat.error
    film = OracleFilm(flat.settings)
    film.render(flat, 0, 2, 2)
    img = film.resolve(_abi.PASS_COMBINED)
    assert img.shape == (bundle.HEIGHT, bundle.WIDTH, 4)
    assert np.all(np.isfinite(img)) and float(img[..., :3].mean()) > 0.01
    # the red and green walls tint the left and right thirds
    left, right = img[:, : bundle.WIDTH // 6, :3].mean((0, 1)), img[:, -bundle.WIDTH // 6:, :3].mean((0, 1))
    assert left[0] > left[1] and right[1] > right[0]


def test_bundle_errors_are_reported(tmp_path):
    bad = bundle.write_bundle(tmp_path / "schema", schema="psycles.blender-scene.v0")
    f = FlattenedBundle(bad)
    assert not f.handle and "unsupported Blender scene bundle schema" in f.error
    broken = bundle.write_bundle(tmp_path / "broken")
    (broken / "scene.json").write_text((broken / "scene.json").read_text()[:-10])
    f = FlattenedBundle(broken)
    assert not f.handle and "failed to parse" in f.error
    missing = bundle.write_bundle(tmp_path / "missing")
    (missing / "geometry.bin").unlink()
    f = FlattenedBundle(missing)
    assert not f.handle and "geometry.bin" in f.error
