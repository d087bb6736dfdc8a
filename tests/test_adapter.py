"""The compiled drop-in adapter (psycles_b200/adapter) on a real Psycles
SceneSnapshot (not gpu-marked).

tests/adapter/adapter_probe.cpp builds the Cornell-style room of the
reference's Luisa demo (examples/render_luisa_demo.cpp:203-305) with the
reference's own contract API, compiles its materials with the reference's
own MaterialLibrary::update and flattens it with the adapter's flatten().
The flattened psy_scene_desc must equal what this package's scene model
builds for the same room (luisa_demo_scene) -- geometry, instances, lamp,
camera and background field for field -- and render, through the oracle,
to the same passes: bit for bit for the plain materials, and for the
variant whose block colour and roughness the reference compiler lowers to a
value stream (RGB nodes through a colour mix, float math).

Needs oracle/_ref/libpsycles_adapter_probe.so (`make -C oracle adapter`,
built from the reference tree where it is present); skipped without it."""

import ctypes
import pathlib

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes

ROOT = pathlib.Path(__file__).resolve().parent.parent
PROBE = ROOT / "oracle" / "_ref" / "libpsycles_adapter_probe.so"

pytestmark = pytest.mark.skipif(not PROBE.exists(), reason="adapter probe not built (make -C oracle adapter)")


def probe():
    _abi.load()  # libpsycles_cuda.so first, so the probe resolves it
    lib = ctypes.CDLL(str(PROBE))
    lib.probe_demo_flatten.restype = ctypes.c_void_p
    lib.probe_demo_flatten.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    lib.probe_flat_desc.restype = ctypes.POINTER(_abi.SceneDesc)
    lib.probe_flat_desc.argtypes = [ctypes.c_void_p]
    lib.probe_flat_destroy.argtypes = [ctypes.c_void_p]
    return lib


class Flattened:
    """The adapter's flattened demo snapshot (variant 0 plain, 1 value-graph
    block, 2 glossy, 4 glass and refraction); `.pointer` as
    scenes.SceneDescHandle."""

    def __init__(self, variant):
        self.lib = probe()
        err = ctypes.create_string_buffer(512)
        self.handle = self.lib.probe_demo_flatten(int(variant), err, 512)
        assert self.handle, err.value.decode()
        self.desc = self.lib.probe_flat_desc(self.handle).contents
        self.pointer = ctypes.pointer(self.desc)

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.probe_flat_destroy(self.handle)


def arr(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0)


def test_flattened_snapshot_equals_scene_model():
    flat = Flattened(False)  # owns the arrays the descriptor points into
    a = flat.desc
    handle = scenes.luisa_demo_scene(False).to_desc()
    b = handle.desc
    assert (a.mesh_count, a.instance_count, a.material_count, a.light_count) == \
        (b.mesh_count, b.instance_count, b.material_count, b.light_count) == (2, 2, 4, 1)
    for i in range(a.mesh_count):
        ma, mb = a.meshes[i], b.meshes[i]
        assert (ma.vertex_count, ma.triangle_count, ma.smooth) == (mb.vertex_count, mb.triangle_count, mb.smooth)
        assert np.array_equal(arr(ma.positions, 3 * ma.vertex_count), arr(mb.positions, 3 * mb.vertex_count))
        assert np.array_equal(arr(ma.indices, 3 * ma.triangle_count), arr(mb.indices, 3 * mb.triangle_count))
        assert bool(ma.materials) == bool(mb.materials)
        if ma.materials:
            assert np.array_equal(arr(ma.materials, ma.triangle_count), arr(mb.materials, mb.triangle_count))
    for i in range(a.instance_count):
        ia, ib = a.instances[i], b.instances[i]
        assert list(ia.object_to_world) == list(np.float32(ib.object_to_world))
        assert (ia.mesh, ia.material, ia.visibility) == (ib.mesh, ib.material, ib.visibility)
    la, lb = a.lights[0], b.lights[0]
    for name, _ in _abi.LightDesc._fields_:
        va, vb = getattr(la, name), getattr(lb, name)
        if hasattr(va, "__len__"):
            assert list(va) == list(np.float32(list(vb))), name
        else:
            assert np.float32(va) == np.float32(vb), name
    assert list(a.camera.camera_to_world) == list(b.camera.camera_to_world)
    for name in ("field_of_view", "horizontal_field_of_view", "sensor_fit", "near_clip", "far_clip", "projection"):
        assert np.float32(getattr(a.camera, name)) == np.float32(getattr(b.camera, name)), name
    assert list(a.background) == list(np.float32(list(b.background)))
    # the materials: one rough diffuse closure each, colour and roughness as authored
    for i in range(a.material_count):
        ma, mb = a.materials[i], b.materials[i]
        ca, cb = ma.closures[ma.root], mb.closures[mb.root]
        assert ca.op == cb.op == _abi.CLOSURE_DIFFUSE
        assert not ca.color & _abi.INPUT_VALUE and not ca.roughness & _abi.INPUT_VALUE  # unlinked sockets
        col_a = arr(ma.vectors, 3 * ma.vector_count).reshape(-1, 3)[ca.color]
        col_b = arr(mb.vectors, 3 * mb.vector_count).reshape(-1, 3)[cb.color]
        assert np.array_equal(col_a, col_b)
        assert arr(ma.scalars, ma.scalar_count)[ca.roughness] == arr(mb.scalars, mb.scalar_count)[cb.roughness]


@pytest.mark.parametrize("graph_material", [0, 1, 2, 4])
def test_flattened_snapshot_renders_as_scene_model(graph_material):
    flat = Flattened(graph_material)
    model = scenes.luisa_demo_scene(graph_material)
    if graph_material == 1:
        block = flat.desc.materials[3]
        assert block.value_count > 0  # the reference compiler emitted a value stream
        c = block.closures[block.root]
        assert c.color & _abi.INPUT_VALUE and c.roughness & _abi.INPUT_VALUE
    if graph_material == 2:
        # the reference compiler's glossy closures: GGX block, Beckmann in the plaster mix
        block = flat.desc.materials[3]
        c = block.closures[block.root]
        assert (c.op, c.a) == (_abi.CLOSURE_GLOSSY, _abi.GLOSSY_GGX)
        plaster = flat.desc.materials[0]
        ops = {(plaster.closures[k].op, plaster.closures[k].a) for k in range(plaster.closure_count)}
        assert (_abi.CLOSURE_GLOSSY, _abi.GLOSSY_BECKMANN) in ops and plaster.flags == 0
    if graph_material == 4:
        # the reference compiler's dielectric closures: GGX glass block (IOR in a
        # scalar slot), Beckmann refraction in the plaster mix
        block = flat.desc.materials[3]
        c = block.closures[block.root]
        assert (c.op, c.a) == (_abi.CLOSURE_GLASS, _abi.GLOSSY_GGX)
        assert not c.scalar & _abi.INPUT_VALUE
        assert arr(block.scalars, block.scalar_count)[c.scalar] == np.float32(1.45)
        plaster = flat.desc.materials[0]
        ops = {(plaster.closures[k].op, plaster.closures[k].a) for k in range(plaster.closure_count)}
        assert (_abi.CLOSURE_REFRACTION, _abi.GLOSSY_BECKMANN) in ops
    st = scenes.render_settings(64, 48, max_bounces=4)
    fa, fb = OracleFilm(st), OracleFilm(st)
    fa.render(flat, 0, 4, 4)
    fb.render(model.to_desc(), 0, 4, 4)
    for kind in (_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO):
        ra, rb = fa.resolve(kind), fb.resolve(kind)
        assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32)), kind
    assert fa.resolve(_abi.PASS_COMBINED)[..., :3].mean() > 0.0


def test_pfm_writer_equals_the_reference_writer(tmp_path):
    from psycles_b200.backend import write_pfm
    lib = probe()
    lib.probe_write_pfm.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                    ctypes.c_char_p]
    rng = np.random.default_rng(0)
    for channels in (4, 3, 1):
        img = rng.uniform(-1.0, 4.0, (5, 7, channels)).astype(np.float32)
        ref, ours = tmp_path / f"ref{channels}.pfm", tmp_path / f"ours{channels}.pfm"
        assert lib.probe_write_pfm(7, 5, channels, img.ctypes.data, str(ref).encode()) == 0
        write_pfm(img, ours)
        assert ref.read_bytes() == ours.read_bytes(), channels


def test_multiscatter_glossy_is_refused():
    """MULTI_GGX needs Cycles' tabulated energy-preservation tables, which
    are not in the CUDA path: flatten() refuses the material with a
    diagnostic instead of rendering it as plain GGX."""
    lib = probe()
    err = ctypes.create_string_buffer(512)
    assert not lib.probe_demo_flatten(3, err, 512)
    assert "Multiscatter GGX" in err.value.decode()
