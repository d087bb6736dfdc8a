"""The flat light distribution's pick on the device against the oracle.

The device's binary search over the cumulative distribution must pick what
the oracle's search picks (src/luisa/path_tracer_light_distribution.cpp:12-55)
for every random number: the power-of-two fractions k / 2^bits and their
neighbours one ulp away (the Cornell box's two equal emitters put a CDF
value on 1/2), 0, the largest float below 1, 1, NaN, and uniform numbers.
The not-gpu test checks that the oracle's picks step through the
distribution in order."""

import ctypes

import numpy as np
import pytest

from oracle.oracle import OracleScene
from psycles_b200 import _abi, scenes


def _numbers(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    edges = []
    for bits in range(1, 21):
        k = np.unique(np.concatenate([np.arange(0, min(1 << bits, 64)), rng.integers(0, 1 << bits, 256)]))
        edges.append((k / float(1 << bits)).astype(np.float32))
    e = np.concatenate(edges)
    near = np.concatenate([e, np.nextafter(e, np.float32(0)), np.nextafter(e, np.float32(1))])
    special = np.array([0.0, np.nextafter(np.float32(1), np.float32(0)), 1.0, np.nan, -0.0], np.float32)
    return np.concatenate([near, special, rng.random(200000, dtype=np.float32)]).astype(np.float32)


def _cases():
    return {"procedural": lambda: scenes.procedural_scene(seed=0),
            "many_light": lambda: scenes.many_light_scene(seed=0),
            "cornell": scenes.cornell_box}


@pytest.mark.parametrize("which", ["procedural", "many_light", "cornell"])
def test_oracle_pick_is_the_cdf_search(which):
    """The oracle's picks of increasing numbers step through the
    distribution's entries in order (triangles, then lights), each with a
    positive selection pdf."""
    osc = OracleScene(_cases()[which]().to_desc())
    u = np.sort(np.random.default_rng(3).random(50000, dtype=np.float32))
    kind, index, pdf = osc.distribution_sample(u)
    key = kind.astype(np.int64) * (1 << 32) + index
    # sorted numbers pick entries in distribution order (triangles, then lights)
    assert np.all(np.diff(key) >= 0)
    assert np.all(pdf > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["procedural", "many_light", "cornell"])
def test_device_pick_matches_oracle(backend, which):
    scene = _cases()[which]()
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    osc = OracleScene(scene.to_desc())
    u = _numbers(5)
    o_kind, o_index, o_pdf = osc.distribution_sample(u)
    n = u.size
    d_kind = np.zeros(n, np.uint32)
    d_index = np.zeros(n, np.uint32)
    d_pdf = np.zeros(n, np.float32)
    _abi.check(backend.context.lib.psy_debug_light_distribution(
        comp.scene.handle, _abi.ptr(u), n, _abi.ptr(d_kind, ctypes.c_uint32), _abi.ptr(d_index, ctypes.c_uint32),
        _abi.ptr(d_pdf)))
    assert np.array_equal(d_kind, o_kind)
    assert np.array_equal(d_index, o_index)
    assert np.array_equal(d_pdf.view(np.uint32), o_pdf.view(np.uint32))
