"""The allocation-free render entry point (psy_session_render_samples_static).

Some callers cannot allocate device memory while they render -- a plugin
held to its host application's fixed device-memory budget, or a viewport
thread that must not stall on an allocation's implicit synchronisation.
This entry point renders from static device arrays instead.  The test calls
it through the C ABI twice in a row and checks each result against
psy_session_render_samples on the same scene: the same kernels run in the
same sample order, so every pass must be bit-identical.  It also checks that
a call after the first (which sets up the static table) leaves the device's
free memory unchanged.  It lives in a file of its own that pytest collects
last.
"""

import ctypes

import numpy as np
import pytest

from psycles_b200 import _abi, scenes
from psycles_b200.backend import CudaPathTracerBackend, SampleRange

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


def device_free_bytes() -> int:
    """cudaMemGetInfo of the current device, through the CUDA runtime the
    library itself loaded."""
    rt = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def test_static_render_matches_allocating_render_twice():
    backend = CudaPathTracerBackend(0)
    lib = backend.context.lib
    scene = scenes.small_test_scene(seed=2)
    settings = scenes.render_settings(80, 60, max_bounces=6)
    compiled = backend.compile_scene(scene).scene
    regular = backend.create_session(compiled, settings)
    static = backend.create_session(compiled, scenes.render_settings(80, 60, max_bounces=6))
    free_after = []
    for first, count in ((0, 3), (3, 5)):
        assert regular.render_samples(SampleRange(first, count, 0, 8)), regular.diagnostics
        free_before = device_free_bytes()
        status = lib.psy_session_render_samples_static(static.handle, first, count, 0, 8)
        assert status == _abi.PSY_OK, lib.psy_last_error().decode()
        free_after.append((free_before, device_free_bytes()))
        assert static.rendered_samples() == regular.rendered_samples() == first + count
        for kind in PASSES:
            a, b = static.read_pass(kind), regular.read_pass(kind)
            assert a.shape == b.shape
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (first, kind)
    # the second call allocates nothing on the device (free memory may only
    # grow, when the stream's pool returns memory at the call's final
    # synchronisation)
    before, after = free_after[1]
    assert after >= before, (before, after)


def test_static_render_limits_are_reported():
    backend = CudaPathTracerBackend(0)
    lib = backend.context.lib
    compiled = backend.compile_scene(scenes.cornell_box()).scene
    big = backend.create_session(compiled, scenes.render_settings(512, 256))
    assert lib.psy_session_render_samples_static(big.handle, 0, 1, 0, 4) == _abi.PSY_ERROR_RANGE
    assert b"65536 pixels" in lib.psy_last_error()
    small = backend.create_session(compiled, scenes.render_settings(64, 64))
    assert lib.psy_session_render_samples_static(small.handle, 0, 1, 0, 1024) == _abi.PSY_ERROR_RANGE
    assert b"256 total samples" in lib.psy_last_error()
