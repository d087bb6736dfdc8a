"""The allocation-free render entry point (psy_session_render_samples_static).

Some callers cannot allocate device memory while they render -- a plugin
held to its host application's fixed memory budget, or a viewport thread
that must not stall on an allocation.  This entry point renders from static
device arrays instead.  The test calls it through the C ABI twice in a row
and checks each result against psy_session_render_samples on the same
scene, with the parity tolerance of the other GPU tests (relative RMSE
1e-3).  It lives in a file of its own that pytest collects last.
"""

import ctypes

import numpy as np
import pytest

from psycles_b200 import _abi, scenes
from psycles_b200.backend import CudaPathTracerBackend, SampleRange

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


def rel_rmse(a, b):
    ref = float(np.sqrt(np.mean(np.square(b.astype(np.float64)))))
    return float(np.sqrt(np.mean(np.square(a.astype(np.float64) - b.astype(np.float64))))) / max(ref, 1e-12)


def test_static_render_matches_allocating_render_twice():
    backend = CudaPathTracerBackend(0)
    lib = backend.context.lib
    scene = scenes.small_test_scene(seed=2)
    settings = scenes.render_settings(80, 60, max_bounces=6)
    compiled = backend.compile_scene(scene).scene
    regular = backend.create_session(compiled, settings)
    static = backend.create_session(compiled, scenes.render_settings(80, 60, max_bounces=6))
    for first, count in ((0, 3), (3, 5)):
        assert regular.render_samples(SampleRange(first, count, 0, 8)), regular.diagnostics
        status = lib.psy_session_render_samples_static(static.handle, first, count, 0, 8)
        assert status == _abi.PSY_OK, lib.psy_last_error().decode()
        assert static.rendered_samples() == regular.rendered_samples() == first + count
        for kind in PASSES:
            a, b = static.read_pass(kind), regular.read_pass(kind)
            assert rel_rmse(a, b) <= 1e-3, (first, kind)


def test_static_render_limits_are_reported():
    backend = CudaPathTracerBackend(0)
    lib = backend.context.lib
    compiled = backend.compile_scene(scenes.cornell_box()).scene
    big = backend.create_session(compiled, scenes.render_settings(512, 256))
    assert lib.psy_session_render_samples_static(big.handle, 0, 1, 0, 4) == 5
    assert b"65536 pixels" in lib.psy_last_error()
    small = backend.create_session(compiled, scenes.render_settings(64, 64))
    assert lib.psy_session_render_samples_static(small.handle, 0, 1, 0, 1024) == 5
    assert b"256 total samples" in lib.psy_last_error()
