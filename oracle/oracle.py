"""TEST INFRASTRUCTURE ONLY -- Python handle on the CPU oracle
(oracle/liboracle.so, built by `make -C oracle`).  Used by tests/, the smoke
check and bench.py's CPU-baseline leg as the checker; the product never
imports it."""

from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libpsycles_ref.so"

_lib = None


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        vp = ctypes.c_void_p
        lib.oracle_render.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp, vp,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
        lib.oracle_render.restype = ctypes.c_int
        lib.oracle_resolve_pass.argtypes = [ctypes.c_uint32, vp, vp, ctypes.c_uint64, ctypes.c_float, vp]
        lib.oracle_sobol_fingerprint.restype = ctypes.c_uint64
        lib.oracle_scene_create.restype = vp
        lib.oracle_scene_create.argtypes = [vp, ctypes.c_int]
        lib.oracle_scene_destroy.argtypes = [vp]
        lib.oracle_scene_closest.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        lib.oracle_pixel_filter_table.argtypes = [ctypes.c_uint32, ctypes.c_float, vp]
        lib.oracle_sample_cosine_hemisphere.argtypes = [vp, vp, vp, vp]
        lib.oracle_next_surface.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleFilm:
    """Film sums of the oracle for one window, accumulated over calls."""

    def __init__(self, settings):
        self.settings = settings
        w = settings.window_width or settings.full_width
        h = settings.window_height or settings.full_height
        self.shape = (h, w)
        n = w * h
        self.combined = np.zeros(4 * n, np.float32)
        self.normal = np.zeros(4 * n, np.float32)
        self.albedo = np.zeros(4 * n, np.float32)
        self.count = np.zeros(n, np.uint32)

    def render(self, desc_handle, first: int, count: int, total: int, threads: int = 0, brute_force: bool = False,
               trace: tuple[int, int, int] | None = None):
        lib = load()
        t = None
        tx = ty = ts = -1
        if trace is not None:
            from psycles_b200 import _abi
            t = _abi.PathTrace()
            tx, ty, ts = trace
        st = lib.oracle_render(ctypes.cast(desc_handle.pointer, ctypes.c_void_p),
                               ctypes.cast(ctypes.byref(self.settings), ctypes.c_void_p), first, count, total,
                               _p(self.combined), _p(self.normal), _p(self.albedo), _p(self.count), threads,
                               1 if brute_force else 0, tx, ty, ts,
                               ctypes.cast(ctypes.byref(t), ctypes.c_void_p) if t is not None else None)
        if st != 0:
            raise RuntimeError("oracle_render failed")
        return t

    def resolve(self, kind: int) -> np.ndarray:
        """The pass as write_passes would hand it to the sink."""
        lib = load()
        h, w = self.shape
        n = h * w
        if kind == 20:
            out = np.zeros(n, np.float32)
            lib.oracle_resolve_pass(kind, None, _p(self.count), n, ctypes.c_float(1.0), _p(out))
            return out.reshape(h, w, 1)
        src = {0: self.combined, 2: self.normal, 18: self.normal, 4: self.albedo, 19: self.albedo}[kind]
        out = np.zeros(4 * n, np.float32)
        lib.oracle_resolve_pass(kind, _p(src), _p(self.count), n, ctypes.c_float(self.settings.film_exposure), _p(out))
        return out.reshape(h, w, 4)


class OracleScene:
    """Prepared oracle scene for traversal queries."""

    def __init__(self, desc_handle, brute_force: bool = False):
        self.lib = load()
        self.handle = self.lib.oracle_scene_create(ctypes.cast(desc_handle.pointer, ctypes.c_void_p),
                                                   1 if brute_force else 0)

    def closest(self, rays: np.ndarray, visibility: int = 63):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        tuv = np.zeros((rays.shape[0], 3), np.float32)
        ids = np.zeros((rays.shape[0], 2), np.uint32)
        self.lib.oracle_scene_closest(self.handle, _p(rays), rays.shape[0], visibility, _p(tuv), _p(ids))
        return tuv, ids

    def __del__(self):
        try:
            self.lib.oracle_scene_destroy(self.handle)
        except Exception:
            pass
