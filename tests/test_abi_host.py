"""C ABI surface and host precompute of libpsycles_cuda.so, without a GPU:
every symbol include/psycles_cuda.h declares is exported, and the host
tables (Sobol LUT, pixel filter, default settings) equal the oracle's."""

import ctypes
import pathlib
import re

import numpy as np
import pytest

from psycles_b200 import _abi

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _declared_symbols():
    text = (ROOT / "include" / "psycles_cuda.h").read_text()
    return sorted(set(re.findall(r"\b(psy_[a-z0-9_]+)\s*\(", text)))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    assert {n for n, _, _ in _abi.SIGNATURES} <= set(declared)


def test_abi_version():
    assert _abi.load().psy_abi_version() == 2


def test_sobol_table_matches_oracle(oracle_lib, golden):
    lib = _abi.load()
    for size in (256, 1024):
        a = np.zeros(size * 256 * 4, np.float32)
        b = np.zeros_like(a)
        _abi.check(lib.psy_sobol_generate_table(size, _abi.ptr(a)))
        oracle_lib.oracle_sobol_table(size, _p(b))
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert lib.psy_sobol_generate_table(300, _abi.ptr(np.zeros(4, np.float32))) == 1


def test_sequence_sizes_match_oracle(oracle_lib):
    lib = _abi.load()
    for n in (0, 1, 2, 16, 64, 255, 256, 257, 1000, 8192, 9000):
        assert lib.psy_sobol_sequence_size_for_samples(n) == oracle_lib.oracle_sobol_sequence_size(n)


@pytest.mark.parametrize("filt", [0, 1, 2])
@pytest.mark.parametrize("width", [0.5, 1.0, 1.5, 2.5])
def test_pixel_filter_matches_oracle(oracle_lib, filt, width):
    lib = _abi.load()
    a = np.zeros(1024, np.float32)
    b = np.zeros(1024, np.float32)
    _abi.check(lib.psy_pixel_filter_table(filt, width, _abi.ptr(a)))
    oracle_lib.oracle_pixel_filter_table(filt, ctypes.c_float(width), _p(b))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_default_settings_match_contract():
    lib = _abi.load()
    c = _abi.RenderSettings()
    lib.psy_render_settings_default(ctypes.byref(c))
    p = _abi.default_settings()
    assert bytes(c) == bytes(p)
    assert c.max_bounces == 12 and c.transparent_max_bounces == 8 and abs(c.light_sampling_threshold - 0.01) < 1e-9


def test_calls_without_device_fail_cleanly():
    lib = _abi.load()
    assert lib.psy_scene_compile(None, None, None) == 1
    assert lib.psy_session_render_samples(None, 0, 1, 0, 1) == 1
    assert b"null" in lib.psy_last_error()
