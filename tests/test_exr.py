"""Multi-layer OpenEXR output (not gpu-marked).

psycles_b200.exr writes io::write_multilayer_exr's file
(src/io/openexr.cpp:150-349) without OpenImageIO: channel names
`<view layer>.<pass>.<component>` with the reference's component rule,
full-float scanlines, ZIP compression, and the reference's argument checks
and messages.  The container and the ZIP scheme are checked against the
OpenEXR library that OpenCV links (where that build has OpenEXR): it must
decode the files bit for bit, for compressed and for raw-stored chunks."""

import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

from psycles_b200 import _abi
from psycles_b200.backend import DEFAULT_PASSES, MemoryOutputSink, PassRequest, PassTile
from psycles_b200.exr import component_name, read_exr, write_exr, write_multilayer_exr

ROOT = pathlib.Path(__file__).resolve().parent.parent


def tile(kind, name, pixels):
    h, w = pixels.shape[:2]
    return PassTile(PassRequest(kind, name, pixels.shape[2]), (0, 0, w, h), (w, h), pixels)


def _opencv_has_openexr() -> bool:
    try:
        import cv2
    except ImportError:
        return False
    return "OpenEXR:" in cv2.getBuildInformation() and "OpenEXR:                     NO" not in cv2.getBuildInformation()


@pytest.mark.skipif(not _opencv_has_openexr(), reason="OpenCV without OpenEXR")
def test_openexr_library_decodes_the_files(tmp_path):
    rng = np.random.default_rng(1)
    cases = []
    for k, (h, w) in enumerate([(37, 53), (16, 8), (1, 1), (100, 3)]):
        noisy = rng.uniform(-2.0, 5.0, (h, w, 4)).astype(np.float32)  # raw-stored chunks
        noisy[0, 0, 0] = np.inf
        smooth = np.broadcast_to(np.linspace(0, 1, w, dtype=np.float32)[None, :, None], (h, w, 3)).copy()
        for name, img in ((f"noisy{k}", noisy), (f"smooth{k}", smooth)):
            path = tmp_path / f"{name}.exr"
            write_exr(path, w, h, [(c, img[..., i]) for i, c in enumerate("RGBA"[:img.shape[2]])])
            np.save(tmp_path / f"{name}.npy", img)
            cases.append(name)
    script = (
        "import sys, numpy as np, cv2\n"
        "d = sys.argv[1]\n"
        "for n in sys.argv[2:]:\n"
        "    r = cv2.imread(f'{d}/{n}.exr', cv2.IMREAD_UNCHANGED)\n"
        "    ref = np.load(f'{d}/{n}.npy')\n"
        "    order = [2, 1, 0, 3][:ref.shape[2]]\n"
        "    assert r is not None and r.dtype == np.float32, n\n"
        "    assert np.array_equal(r.reshape(ref.shape)[..., order], ref), n\n"
        "print('ok')\n")
    env = dict(os.environ, OPENCV_IO_ENABLE_OPENEXR="1")
    out = subprocess.run([sys.executable, "-c", script, str(tmp_path), *cases], env=env, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr


def test_component_names_follow_the_reference():
    assert [component_name(_abi.PASS_COMBINED, 4, c) for c in range(4)] == list("RGBA")
    assert [component_name(_abi.PASS_NORMAL, 4, c) for c in range(4)] == ["X", "Y", "Z", "A"]
    assert component_name(1, 1, 0) == "Z"  # depth
    assert [component_name(_abi.PASS_SAMPLE_COUNT, 1, 0)] == ["X"]
    assert [component_name(_abi.PASS_ALBEDO, 2, c) for c in range(2)] == ["X", "Y"]
    assert [component_name(_abi.PASS_ALBEDO, 3, c) for c in range(3)] == list("RGB")
    assert [component_name(_abi.PASS_ALBEDO, 6, c) for c in range(6)] == [f"C{i}" for i in range(6)]


def test_multilayer_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    h, w = 45, 70
    sink = MemoryOutputSink()
    for req in DEFAULT_PASSES:
        sink.write(tile(req.kind, req.name, rng.uniform(-1, 3, (h, w, req.channels)).astype(np.float32)))
    path = tmp_path / "passes.exr"
    sink.write_multilayer_exr(path)
    ch = read_exr(path)
    names = sorted(ch)
    assert "ViewLayer.Combined.A" in names and "ViewLayer.Normal.X" in names and "ViewLayer.Sample Count.X" in names
    assert "ViewLayer.Denoising Normal.R" in names  # only the normal pass takes X / Y / Z
    assert len(names) == sum(r.channels for r in DEFAULT_PASSES)
    for kind, t in sink.tiles.items():
        n = t.pixels.shape[2]
        for c in range(n):
            got = ch[f"ViewLayer.{t.pass_.name}.{component_name(kind, n, c)}"]
            assert np.array_equal(got, t.pixels[..., c])
    # the channel list is sorted by name and the header names the ZIP compression
    data = path.read_bytes()
    assert data[:4] == bytes([0x76, 0x2F, 0x31, 0x01])
    positions = [data.index(n.encode() + b"\0") for n in names]
    assert positions == sorted(positions)


def test_long_channel_names_set_the_long_name_flag(tmp_path):
    px = np.ones((4, 4, 3), np.float32)
    path = tmp_path / "long.exr"
    write_multilayer_exr([tile(_abi.PASS_ALBEDO, "A pass name well beyond the short limit", px)], path, "Layer")
    version = int.from_bytes(path.read_bytes()[4:8], "little")
    assert version & 0xFF == 2 and version & 0x400
    assert np.array_equal(read_exr(path)["Layer.A pass name well beyond the short limit.B"], px[..., 2])


def test_argument_checks_carry_the_reference_messages(tmp_path):
    px = np.zeros((4, 5, 4), np.float32)
    good = tile(_abi.PASS_COMBINED, "Combined", px)
    cases = [
        (([], tmp_path / "a.exr"), {}, "no render passes were supplied"),
        (([good], tmp_path / "a.exr"), {"view_layer": ""}, "the OpenEXR view-layer name is empty"),
        (([good], tmp_path / "a.pfm"), {}, "the output path does not have an .exr extension"),
        (([tile(0, "Combined", np.zeros((0, 5, 4), np.float32))], tmp_path / "a.exr"), {},
         "the render extent is invalid for OpenEXR"),
        (([good, tile(4, "Albedo", np.zeros((4, 6, 4), np.float32))], tmp_path / "a.exr"), {},
         "all OpenEXR passes must have the same extent"),
        (([good, tile(4, "Albedo", np.zeros((4, 5, 0), np.float32))], tmp_path / "a.exr"), {},
         "an OpenEXR pass has no channels"),
        (([tile(0, "", px)], tmp_path / "a.exr"), {}, "an OpenEXR pass has an empty name"),
        (([good, tile(0, "Combined", px)], tmp_path / "a.exr"), {},
         "duplicate OpenEXR channel name: ViewLayer.Combined.R"),
    ]
    for args, kwargs, message in cases:
        with pytest.raises(ValueError) as e:
            write_multilayer_exr(*args, **kwargs)
        assert str(e.value) == message
    write_multilayer_exr([good], tmp_path / "upper.EXR")
    assert (tmp_path / "upper.EXR").exists()
