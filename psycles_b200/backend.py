"""Host mirror of the reference render contract over the C ABI.

Names and argument meaning follow include/psycles/contract/render.h:
RendererBackend.compile_scene -> SceneCompilation(scene, diagnostics);
create_session -> RenderSession or None; RenderSession.render_samples(
SampleRange, OutputSink) -> bool (False for a cancelled session, an empty or
out-of-range SampleRange, a changed total, or a failed dispatch), reset,
cancel; OutputSink.begin / write(PassTile) / end.  Every call goes through
libpsycles_cuda.so.
"""

from __future__ import annotations

import atexit
import ctypes
import dataclasses
import threading
import weakref

import numpy as np

from . import _abi
from .scenes import Scene

# Live native objects by kind.  At interpreter exit they are closed in
# dependency order (servers and batches, then sessions, scenes, contexts),
# before module teardown could free them in arbitrary order: a scene freed
# after its context would free device memory on a destroyed stream.
_LIVE = {kind: weakref.WeakSet() for kind in ("server", "batch", "session", "scene", "context")}


@atexit.register
def _close_all() -> None:
    for kind in ("server", "batch", "session", "scene", "context"):
        for obj in list(_LIVE[kind]):
            try:
                obj.close()
            except Exception:
                pass

PassKind = {
    "combined": _abi.PASS_COMBINED, "normal": _abi.PASS_NORMAL, "albedo": _abi.PASS_ALBEDO,
    "denoising_normal": _abi.PASS_DENOISING_NORMAL, "denoising_albedo": _abi.PASS_DENOISING_ALBEDO,
    "sample_count": _abi.PASS_SAMPLE_COUNT,
}


@dataclasses.dataclass
class PassRequest:
    kind: int = _abi.PASS_COMBINED
    name: str = ""
    channels: int = 4


@dataclasses.dataclass
class SampleRange:
    first: int = 0
    count: int = 0
    offset: int = 0
    total: int = 0


@dataclasses.dataclass
class PassTile:
    pass_: PassRequest
    window: tuple[int, int, int, int]
    full_extent: tuple[int, int]
    pixels: np.ndarray  # float32 [height, width, channels]


class OutputSink:
    def begin(self, settings) -> None:  # pragma: no cover - interface
        pass

    def write(self, tile: PassTile) -> None:  # pragma: no cover - interface
        raise NotImplementedError

    def end(self, cancelled: bool) -> None:  # pragma: no cover - interface
        pass


class MemoryOutputSink(OutputSink):
    """io::MemoryOutputSink (include/psycles/io/image.h:21): keeps the last tile per pass."""

    def __init__(self) -> None:
        self.tiles: dict[int, PassTile] = {}
        self.began = 0
        self.ended: bool | None = None

    def begin(self, settings) -> None:
        self.began += 1
        self.tiles = {}

    def write(self, tile: PassTile) -> None:
        self.tiles[tile.pass_.kind] = tile

    def end(self, cancelled: bool) -> None:
        self.ended = cancelled

    def pass_pixels(self, kind: int) -> np.ndarray:
        return self.tiles[kind].pixels

    def write_pfm(self, kind: int, path) -> None:
        """io::write_pfm of the pass (include/psycles/io/image.h:63)."""
        write_pfm(self.tiles[kind].pixels, path)

    def write_multilayer_exr(self, path, view_layer: str = "ViewLayer") -> None:
        """io::write_multilayer_exr of every pass the sink holds, in the order
        they were written (include/psycles/io/image.h:77-84)."""
        from .exr import write_multilayer_exr
        write_multilayer_exr(list(self.tiles.values()), path, view_layer)


def write_pfm(pixels: np.ndarray, path) -> None:
    """A pass image as a Portable Float Map, as io::write_pfm writes it
    (src/io/image.cpp:156-197): "PF" with the first three channels of a pass
    of three or more, else "Pf" with the first; scale -1.0 (little-endian
    floats); rows from the bottom of the image to the top.  `pixels` is
    [height, width, channels], top row first."""
    img = np.asarray(pixels, dtype=np.float32)
    if img.ndim == 2:
        img = img[..., None]
    h, w, c = img.shape
    if w == 0 or h == 0 or c == 0:
        raise ValueError("empty pass image")
    color = c >= 3
    body = img[::-1, :, :3] if color else img[::-1, :, :1]
    with open(path, "wb") as f:
        f.write(f"{'PF' if color else 'Pf'}\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(body, dtype="<f4").tobytes())


@dataclasses.dataclass
class RenderDiagnostic:
    message: str


class Context:
    """One CUDA device and its stream (psy_context)."""

    def __init__(self, device: int = 0):
        self.lib = _abi.load()
        h = ctypes.c_void_p()
        _abi.check(self.lib.psy_context_create(device, ctypes.byref(h)))
        self.handle = h
        _LIVE["context"].add(self)

    def close(self) -> None:
        if self.handle:
            self.lib.psy_context_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


class CompiledScene:
    def __init__(self, context: Context, handle: ctypes.c_void_p, scene: Scene):
        self.context = context
        self.handle = handle
        _LIVE["scene"].add(self)
        self.scene = scene
        self.lib = context.lib

    def source_revision(self) -> int:
        return int(self.lib.psy_scene_source_revision(self.handle))

    def build_stats(self) -> _abi.SceneBuildStats:
        """Phase times of compile_scene and of the latest light-tree build."""
        st = _abi.SceneBuildStats()
        _abi.check(self.lib.psy_scene_get_build_stats(self.handle, ctypes.byref(st)))
        return st

    def device_bytes(self) -> int:
        return int(self.lib.psy_scene_device_bytes(self.handle))

    def rebind_parameters(self, material: int, scalars: np.ndarray, vectors: np.ndarray) -> None:
        """Parameter-only edit: rewrites one material's parameter block on the device."""
        sc = np.ascontiguousarray(scalars, dtype=np.float32).reshape(-1)
        vc = np.ascontiguousarray(vectors, dtype=np.float32).reshape(-1)
        _abi.check(self.lib.psy_scene_rebind_parameters(self.handle, material, _abi.ptr(sc), sc.size,
                                                        _abi.ptr(vc), vc.size // 3))

    def close(self) -> None:
        if self.handle:
            self.lib.psy_scene_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class SceneCompilation:
    scene: CompiledScene | None
    diagnostics: list[RenderDiagnostic]

    def ok(self) -> bool:
        return self.scene is not None


class RenderSession:
    def __init__(self, compiled: CompiledScene, handle: ctypes.c_void_p, settings: _abi.RenderSettings,
                 passes: list[PassRequest]):
        self.compiled = compiled
        self.handle = handle
        _LIVE["session"].add(self)
        self.settings = settings
        self.passes = passes
        self.lib = compiled.lib
        self.diagnostics: list[RenderDiagnostic] = []
        self._lock = threading.Lock()

    @property
    def window(self) -> tuple[int, int, int, int]:
        s = self.settings
        return (s.window_x, s.window_y, s.window_width or s.full_width, s.window_height or s.full_height)

    def reset(self, settings: _abi.RenderSettings) -> None:
        _abi.check(self.lib.psy_session_reset(self.handle, ctypes.byref(settings)))
        self.settings = settings

    def cancel(self) -> None:
        self.lib.psy_session_cancel(self.handle)

    def set_camera(self, camera) -> None:
        """Renders through `camera` (a scenes.Camera; None restores the
        scene's) and clears the film."""
        from .scenes import camera_desc
        desc = camera_desc(camera) if camera is not None else None
        _abi.check(self.lib.psy_session_set_camera(self.handle, ctypes.byref(desc) if desc is not None else None))

    def render_samples(self, samples: SampleRange, output: OutputSink | None = None) -> bool:
        with self._lock:
            status = self.lib.psy_session_render_samples(self.handle, samples.first, samples.count,
                                                         samples.offset, samples.total)
            if status != _abi.PSY_OK:
                self.diagnostics.append(RenderDiagnostic(self.lib.psy_last_error().decode()))
                return False
            if output is not None:
                output.begin(self.settings)
                for p in self.passes:
                    output.write(PassTile(p, self.window, (self.settings.full_width, self.settings.full_height),
                                          self.read_pass(p.kind)))
                output.end(False)
            return True

    def read_pass(self, kind: int) -> np.ndarray:
        x, y, w, h = self.window
        ch = 1 if kind == _abi.PASS_SAMPLE_COUNT else 4
        out = np.zeros((h, w, ch), dtype=np.float32)
        channels = ctypes.c_uint32()
        _abi.check(self.lib.psy_session_read_pass(self.handle, kind, _abi.ptr(out), out.size, ctypes.byref(channels)))
        return out

    def rendered_samples(self) -> int:
        return int(self.lib.psy_session_rendered_samples(self.handle))

    def request_trace(self, x: int, y: int, sample: int) -> None:
        _abi.check(self.lib.psy_session_request_trace(self.handle, x, y, sample))

    def read_trace(self) -> _abi.PathTrace:
        t = _abi.PathTrace()
        _abi.check(self.lib.psy_session_read_trace(self.handle, ctypes.byref(t)))
        return t

    def stats(self) -> _abi.RenderStats:
        s = _abi.RenderStats()
        _abi.check(self.lib.psy_session_stats(self.handle, ctypes.byref(s)))
        return s

    def close(self) -> None:
        if self.handle:
            self.lib.psy_session_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


DEFAULT_PASSES = [PassRequest(_abi.PASS_COMBINED, "Combined"), PassRequest(_abi.PASS_NORMAL, "Normal"),
                  PassRequest(_abi.PASS_ALBEDO, "Albedo"),
                  PassRequest(_abi.PASS_DENOISING_NORMAL, "Denoising Normal"),
                  PassRequest(_abi.PASS_DENOISING_ALBEDO, "Denoising Albedo"),
                  PassRequest(_abi.PASS_SAMPLE_COUNT, "Sample Count", 1)]


class CudaPathTracerBackend:
    """contract::RendererBackend over libpsycles_cuda.so (one CUDA device)."""

    def __init__(self, device: int = 0, next_event_estimation: bool = True):
        self.context = Context(device)
        self.next_event_estimation = next_event_estimation

    def compile_scene(self, scene: Scene) -> SceneCompilation:
        desc = scene.to_desc()
        h = ctypes.c_void_p()
        status = self.context.lib.psy_scene_compile(self.context.handle, desc.pointer, ctypes.byref(h))
        if status != _abi.PSY_OK:
            return SceneCompilation(None, [RenderDiagnostic(self.context.lib.psy_last_error().decode())])
        return SceneCompilation(CompiledScene(self.context, h, scene), [])

    def create_session(self, compiled: CompiledScene, settings: _abi.RenderSettings,
                       passes: list[PassRequest] | None = None) -> RenderSession | None:
        settings.next_event_estimation = 1 if self.next_event_estimation else 0
        h = ctypes.c_void_p()
        status = self.context.lib.psy_session_create(compiled.handle, ctypes.byref(settings), ctypes.byref(h))
        if status != _abi.PSY_OK:
            return None
        return RenderSession(compiled, h, settings, list(passes or DEFAULT_PASSES))


class BatchRenderer:
    """Sample ranges of many sessions rendered in shared wavefronts
    (psy_batch_*).  Each session ends exactly as its own render_samples call
    would leave it; the batch only shares the path state and the launches."""

    def __init__(self, context: Context, path_capacity: int = 0, max_jobs: int = 0, use_graph: bool = True,
                 check_interval: int = 0):
        self.context = context
        self.lib = context.lib
        cfg = _abi.BatchConfig(path_capacity, max_jobs, 1 if use_graph else 0, check_interval)
        h = ctypes.c_void_p()
        _abi.check(self.lib.psy_batch_create(context.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        _LIVE["batch"].add(self)

    def render(self, work: list[tuple[RenderSession, SampleRange]]) -> bool:
        n = len(work)
        sessions = (ctypes.c_void_p * n)(*[s.handle for s, _ in work])
        cols = [np.array([getattr(r, f) for _, r in work], np.uint32) for f in ("first", "count", "offset", "total")]
        status = self.lib.psy_batch_render(self.handle, sessions, *[_abi.ptr(c, ctypes.c_uint32) for c in cols], n)
        if status != _abi.PSY_OK:
            message = self.lib.psy_last_error().decode()
            for s, _ in work:
                s.diagnostics.append(RenderDiagnostic(message))
            return False
        return True

    def stats(self) -> _abi.BatchStats:
        s = _abi.BatchStats()
        _abi.check(self.lib.psy_batch_get_stats(self.handle, ctypes.byref(s)))
        return s

    def close(self) -> None:
        if self.handle:
            self.lib.psy_batch_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def batch_plan(pixels: list[int], samples: list[int], capacity: int) -> np.ndarray:
    """psy_batch_plan: rows (job, wavefront, path_begin, first sample offset,
    samples, film_begin) of the batch wavefront plan; needs no GPU."""
    lib = _abi.load()
    px = np.ascontiguousarray(pixels, np.uint32)
    sp = np.ascontiguousarray(samples, np.uint32)
    count = ctypes.c_uint32()
    lib.psy_batch_plan(_abi.ptr(px, ctypes.c_uint32), _abi.ptr(sp, ctypes.c_uint32), len(px), capacity, None, 0,
                       ctypes.byref(count))
    out = np.zeros((max(count.value, 1), 6), np.uint32)
    _abi.check(lib.psy_batch_plan(_abi.ptr(px, ctypes.c_uint32), _abi.ptr(sp, ctypes.c_uint32), len(px), capacity,
                                  _abi.ptr(out, ctypes.c_uint32), count.value, ctypes.byref(count)))
    return out[:count.value]


class RenderServer:
    """psy_server_*: a request loop over resident scenes with HBM-budget
    admission and continuous batching of all running jobs."""

    def __init__(self, context: Context, hbm_budget_bytes: int = 0, path_capacity: int = 0, max_running: int = 0,
                 use_graph: bool = True):
        self.context = context
        self.lib = context.lib
        cfg = _abi.ServerConfig(hbm_budget_bytes, path_capacity, max_running, 1 if use_graph else 0, 0)
        h = ctypes.c_void_p()
        _abi.check(self.lib.psy_server_create(context.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        _LIVE["server"].add(self)

    def submit(self, compiled: CompiledScene, settings: _abi.RenderSettings, samples: int, camera=None) -> int:
        from .scenes import camera_desc
        cam = camera_desc(camera) if camera is not None else None
        job = ctypes.c_uint64()
        _abi.check(self.lib.psy_server_submit(self.handle, compiled.handle, ctypes.byref(settings),
                                              ctypes.byref(cam) if cam is not None else None, samples,
                                              ctypes.byref(job)))
        return int(job.value)

    def rebind_parameters(self, compiled: CompiledScene, material: int, scalars, vectors) -> None:
        sc = np.ascontiguousarray(scalars, dtype=np.float32).reshape(-1)
        vc = np.ascontiguousarray(vectors, dtype=np.float32).reshape(-1)
        _abi.check(self.lib.psy_server_rebind_parameters(self.handle, compiled.handle, material, _abi.ptr(sc), sc.size,
                                                         _abi.ptr(vc), vc.size // 3))

    def poll(self, job: int) -> _abi.JobInfo:
        info = _abi.JobInfo()
        _abi.check(self.lib.psy_server_poll(self.handle, job, ctypes.byref(info)))
        return info

    def wait(self, job: int, timeout_ms: int = 60000) -> int:
        """The psy_status of the job's end (PSY_ERROR_TIMEOUT if still running)."""
        return int(self.lib.psy_server_wait(self.handle, job, timeout_ms))

    def read_pass(self, job: int, kind: int, width: int, height: int) -> np.ndarray:
        ch = 1 if kind == _abi.PASS_SAMPLE_COUNT else 4
        out = np.zeros((height, width, ch), dtype=np.float32)
        channels = ctypes.c_uint32()
        _abi.check(self.lib.psy_server_read_pass(self.handle, job, kind, _abi.ptr(out), out.size,
                                                 ctypes.byref(channels)))
        return out

    def release(self, job: int) -> None:
        _abi.check(self.lib.psy_server_release(self.handle, job))

    def cancel(self, job: int) -> None:
        _abi.check(self.lib.psy_server_cancel(self.handle, job))

    def stats(self) -> _abi.ServerStats:
        s = _abi.ServerStats()
        _abi.check(self.lib.psy_server_get_stats(self.handle, ctypes.byref(s)))
        return s

    def close(self) -> None:
        if self.handle:
            self.lib.psy_server_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass
