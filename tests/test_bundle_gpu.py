"""A Blender scene bundle rendered on the GPU through the reference's
importer and the compiled drop-in adapter (gpu-marked).

tests/adapter/adapter_probe.cpp's probe_bundle_render does what
examples/render_blender_scene.cpp:232-420 does with the Luisa backend:
load_blender_scene_bundle(directory), compile_scene(*imported.scene),
create_session with the bundle's own render settings (seed, Blackman-Harris
filter of width 1.5, bounce limits), render_samples(SampleRange, OutputSink&)
in several sample ranges into io::MemoryOutputSink.  The passes must match the
oracle's render of the adapter's flattened scene with the same settings
(relative RMSE 1e-3, at most 1 % of pixels differing in any bit) for the room
of tests/adapter/blender_bundle.py with a Background world tree and with the
importer's world emission graph."""

import ctypes
import pathlib
import sys

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi
from _parity import rel_rmse

ROOT = pathlib.Path(__file__).resolve().parent.parent
PROBE = ROOT / "oracle" / "_ref" / "libpsycles_adapter_probe.so"
sys.path.insert(0, str(ROOT / "tests" / "adapter"))
import blender_bundle as bundle  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not PROBE.exists(), reason="adapter probe not built (make -C oracle adapter)")]


@pytest.mark.parametrize("world_tree", [True, False])
def test_bundle_renders_through_the_contract(tmp_path, world_tree):
    from test_bundle import FlattenedBundle, bundle_probe
    lib = bundle_probe()
    f = ctypes.c_void_p
    lib.probe_bundle_render.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, f, f, f, f,
                                        ctypes.c_char_p, ctypes.c_size_t]
    directory = bundle.write_bundle(tmp_path / "room", world_tree=world_tree)
    w, h, spp = bundle.WIDTH, bundle.HEIGHT, 8
    out = {k: np.zeros((h, w, 4), np.float32) for k in ("combined", "normal", "albedo")}
    count = np.zeros((h, w, 1), np.float32)
    err = ctypes.create_string_buffer(512)
    rc = lib.probe_bundle_render(0, str(directory).encode(), spp, 3, out["combined"].ctypes.data,
                                 out["normal"].ctypes.data, out["albedo"].ctypes.data, count.ctypes.data, err, 512)
    assert rc == 0, err.value.decode()
    flat = FlattenedBundle(directory)
    assert flat.handle, flat.error
    film = OracleFilm(flat.settings)
    film.render(flat, 0, spp, spp)
    for kind, got in ((_abi.PASS_COMBINED, out["combined"]), (_abi.PASS_NORMAL, out["normal"]),
                      (_abi.PASS_ALBEDO, out["albedo"])):
        ref = film.resolve(kind)
        assert rel_rmse(got, ref) <= 1e-3, kind
        assert np.mean(got.view(np.uint32) != ref.view(np.uint32)) <= 0.01, kind
    assert np.all(count == spp)
