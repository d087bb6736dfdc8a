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
        lib.oracle_render_prepared.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                               ctypes.c_uint32, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, vp]
        lib.oracle_render_prepared.restype = ctypes.c_int
        lib.oracle_resolve_pass.argtypes = [ctypes.c_uint32, vp, vp, ctypes.c_uint64, ctypes.c_float, vp]
        lib.oracle_sobol_fingerprint.restype = ctypes.c_uint64
        lib.oracle_scene_create.restype = vp
        lib.oracle_scene_create.argtypes = [vp, ctypes.c_int]
        lib.oracle_scene_destroy.argtypes = [vp]
        lib.oracle_scene_closest.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        lib.oracle_light_tree_query.argtypes = [vp, vp, vp, ctypes.c_uint32, vp, vp, vp]
        lib.oracle_light_tree_query.restype = ctypes.c_int
        lib.oracle_light_tree_triangle_emitter.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32]
        lib.oracle_light_tree_triangle_emitter.restype = ctypes.c_uint32
        lib.oracle_scene_emitter_count.argtypes = [vp]
        lib.oracle_distribution_sample.argtypes = [vp, vp, ctypes.c_uint32, vp, vp, vp]
        lib.oracle_scene_emitter_count.restype = ctypes.c_uint32
        lib.oracle_pixel_filter_table.argtypes = [ctypes.c_uint32, ctypes.c_float, vp]
        lib.oracle_sample_cosine_hemisphere.argtypes = [vp, vp, vp, vp]
        lib.oracle_sample_visible_normal.argtypes = [ctypes.c_int, vp, vp, ctypes.c_float, vp, vp]
        lib.oracle_next_surface.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        lib.oracle_diffuse_intensity.argtypes = [vp, vp, ctypes.c_float, vp, vp, vp]
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

    def render_prepared(self, scene: "OracleScene", first: int, count: int, total: int, row_stride: int = 1,
                        threads: int = 0, trace: tuple[int, int, int] | None = None):
        """render() over a scene prepared once (OracleScene), rendering only
        the window rows whose index is a multiple of `row_stride`."""
        lib = load()
        t = None
        tx = ty = ts = -1
        if trace is not None:
            from psycles_b200 import _abi
            t = _abi.PathTrace()
            tx, ty, ts = trace
        st = lib.oracle_render_prepared(scene.handle, ctypes.cast(ctypes.byref(self.settings), ctypes.c_void_p),
                                        first, count, total, row_stride, _p(self.combined), _p(self.normal),
                                        _p(self.albedo), _p(self.count), threads, tx, ty, ts,
                                        ctypes.cast(ctypes.byref(t), ctypes.c_void_p) if t is not None else None)
        if st != 0:
            raise RuntimeError("oracle_render_prepared failed")
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

    def light_tree_query(self, queries: np.ndarray, pdf_emitters: np.ndarray):
        """(selected emitter, its selection pdf, reverse pdf of pdf_emitters)
        per shading point; queries are (position, u, normal, transmission)."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 8)
        e = np.ascontiguousarray(pdf_emitters, np.uint32)
        sel = np.zeros(q.shape[0], np.uint32)
        spdf = np.zeros(q.shape[0], np.float32)
        rpdf = np.zeros(q.shape[0], np.float32)
        if self.lib.oracle_light_tree_query(self.handle, _p(q), _p(e), q.shape[0], _p(sel), _p(spdf), _p(rpdf)) != 0:
            raise RuntimeError("scene has no usable light tree")
        return sel, spdf, rpdf

    def distribution_sample(self, u: np.ndarray):
        """(kind, index, selection pdf) of the flat light distribution's
        pick for each random number u."""
        u = np.ascontiguousarray(u, np.float32).reshape(-1)
        kind = np.zeros(u.size, np.uint32)
        index = np.zeros(u.size, np.uint32)
        pdf = np.zeros(u.size, np.float32)
        self.lib.oracle_distribution_sample(self.handle, _p(u), u.size, _p(kind), _p(index), _p(pdf))
        return kind, index, pdf

    def emitter_count(self) -> int:
        """Emissive triangles + analytic lights of the prepared scene."""
        return int(self.lib.oracle_scene_emitter_count(self.handle))

    def triangle_emitter(self, obj: int, prim: int) -> int:
        return int(self.lib.oracle_light_tree_triangle_emitter(self.handle, obj, prim))

    def __del__(self):
        try:
            self.lib.oracle_scene_destroy(self.handle)
        except Exception:
            pass


# ----------------------------------------------------------------- light tree

def light_tree_emitter_records(seed: int, count: int) -> np.ndarray:
    """Seeded emitter records (20 floats each, the layout of
    oracle_build_light_tree / ref_build_light_tree): triangle-, point-, spot-
    and distant-like measures, a few invalid ones, shared centroids for the
    tie-breaks, and identities in shuffled order."""
    rng = np.random.default_rng(seed)
    rec = np.zeros((count, 20), np.float32)
    kinds = rng.integers(0, 6, count)
    for i in range(count):
        k = int(kinds[i])
        c = rng.uniform(-10.0, 10.0, 3).astype(np.float32)
        if i > 2 and rng.uniform() < 0.1:
            c = rec[rng.integers(0, i), 14:17].copy()
        half = rng.uniform(0.0, 1.0, 3).astype(np.float32)
        axis = rng.normal(size=3)
        axis = (axis / np.linalg.norm(axis)).astype(np.float32)
        energy = np.float32(rng.uniform(0.01, 5.0))
        lo, hi, empty_b = c - half, c + half, 0.0
        theta_o, theta_e, distant = np.float32(np.pi / 2), np.float32(np.pi / 2), 0.0
        if k == 0:    # one-sided triangle
            theta_o = np.float32(0.0)
        elif k == 1:  # point light
            theta_o = np.float32(np.pi)
        elif k == 2:  # spot light
            theta_o, theta_e = np.float32(0.0), np.float32(rng.uniform(0.05, 1.5))
        elif k == 3:  # distant light
            lo, hi, empty_b, distant = np.zeros(3), np.zeros(3), 1.0, 1.0
            theta_o, theta_e = np.float32(0.0), np.float32(rng.uniform(0.0, 0.3))
        elif k == 4 and rng.uniform() < 0.3:  # emits nothing
            energy = np.float32(0.0)
        rec[i, 0:3], rec[i, 3:6], rec[i, 6] = lo, hi, empty_b
        rec[i, 7:10], rec[i, 10], rec[i, 11], rec[i, 12] = axis, theta_o, theta_e, 0.0
        rec[i, 13], rec[i, 14:17], rec[i, 17] = energy, c, distant
    rec[:, 18] = rng.permutation(count).astype(np.float32)
    return rec


def build_light_tree(lib: ctypes.CDLL, symbol: str, records: np.ndarray, max_leaf: int = 8) -> dict:
    """Runs oracle_build_light_tree or ref_build_light_tree on `records`."""
    n = records.shape[0]
    cap = 2 * n + 4
    node_m = np.zeros((cap, 14), np.float32)
    node_t = np.zeros((cap, 6), np.uint32)
    em_m = np.zeros((n, 14), np.float32)
    em_id = np.zeros(n, np.uint32)
    to_tree = np.zeros(n, np.uint32)
    to_leaf = np.zeros(n, np.uint32)
    root = ctypes.c_uint32(0)
    nodes = ctypes.c_uint32(0)
    fn = getattr(lib, symbol)
    fn.restype = ctypes.c_int
    rc = fn(_p(np.ascontiguousarray(records, np.float32)), ctypes.c_uint32(n), ctypes.c_uint32(max_leaf),
            ctypes.c_uint32(cap), _p(node_m), _p(node_t), _p(em_m), _p(em_id), _p(to_tree), _p(to_leaf),
            ctypes.byref(root), ctypes.byref(nodes))
    if rc != 0:
        raise RuntimeError(f"{symbol} failed with {rc}")
    k = nodes.value
    return {"node_measure": node_m[:k], "node_topology": node_t[:k], "emitter_measure": em_m,
            "emitter_ids": em_id, "to_tree": to_tree, "to_leaf": to_leaf, "root": root.value}


def light_tree_fingerprint(tree: dict) -> int:
    """FNV-1a 64 over every output word of a tree build."""
    h = 14695981039346656037
    parts = [tree["node_measure"].view(np.uint32), tree["node_topology"], tree["emitter_measure"].view(np.uint32),
             tree["emitter_ids"], tree["to_tree"], tree["to_leaf"], np.array([tree["root"]], np.uint32)]
    for part in parts:
        for b in np.ascontiguousarray(part).tobytes():
            h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h
