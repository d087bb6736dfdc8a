"""Rendering a real Psycles SceneSnapshot through the compiled drop-in
adapter on the GPU (gpu-marked).

tests/adapter/adapter_probe.cpp drives CudaPathTracerBackend exactly as a
reference caller (examples/render_luisa_demo.cpp:367-415) drives
LuisaPathTracerBackend: compile_scene(snapshot), create_session(scene,
settings), render_samples(SampleRange, OutputSink&) into the reference's
io::MemoryOutputSink in several sample ranges, then io::write_pfm.  The
passes must match the oracle's render of the adapter's flattened snapshot
(relative RMSE 1e-3, at most 1 % of pixels differing in any bit), the PFM
must hold the Combined pass, and an unsupported pass must be refused with a
null session.  The plain demo materials, the variant whose block the
reference compiler lowers to a value stream, the glossy variant (GGX
block, diffuse + Beckmann plaster) and the dielectric variant (rough GGX
glass block, diffuse + Beckmann refraction plaster) are rendered."""

import ctypes
import pathlib

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from _parity import rel_rmse

ROOT = pathlib.Path(__file__).resolve().parent.parent
PROBE = ROOT / "oracle" / "_ref" / "libpsycles_adapter_probe.so"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not PROBE.exists(), reason="adapter probe not built (make -C oracle adapter)")]


@pytest.mark.parametrize("graph_material", [0, 1, 2, 4])
def test_snapshot_renders_through_the_contract(tmp_path, graph_material):
    from test_adapter import Flattened, probe
    lib = probe()
    f = ctypes.c_void_p
    lib.probe_demo_render.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint32, f, f, f, f, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
    w, h, spp = 96, 72, 8
    out = {k: np.zeros((h, w, 4), np.float32) for k in ("combined", "normal", "albedo")}
    count = np.zeros((h, w, 1), np.float32)
    pfm = tmp_path / "combined.pfm"
    err = ctypes.create_string_buffer(512)
    rc = lib.probe_demo_render(0, graph_material, w, h, spp, 3, out["combined"].ctypes.data,
                               out["normal"].ctypes.data, out["albedo"].ctypes.data, count.ctypes.data,
                               str(pfm).encode(), err, 512)
    assert rc == 0, err.value.decode()
    flat = Flattened(graph_material)
    st = scenes.render_settings(w, h, max_bounces=4)
    film = OracleFilm(st)
    film.render(flat, 0, spp, spp)
    for kind, got in ((_abi.PASS_COMBINED, out["combined"]), (_abi.PASS_NORMAL, out["normal"]),
                      (_abi.PASS_ALBEDO, out["albedo"])):
        ref = film.resolve(kind)
        assert rel_rmse(got, ref) <= 1e-3, kind
        assert np.mean(got.view(np.uint32) != ref.view(np.uint32)) <= 0.01, kind
    assert np.all(count == spp)
    # io::write_pfm: "PF", width height, -1.0, RGB rows bottom to top
    data = pfm.read_bytes()
    header = f"PF\n{w} {h}\n-1.0\n".encode()
    assert data.startswith(header)
    pixels = np.frombuffer(data[len(header):], "<f4").reshape(h, w, 3)
    assert np.array_equal(pixels[::-1], out["combined"][..., :3])
