"""Autotuner for the wavefront launch shape (psy_context_set_tuning).

Searches the knobs of psy_tuning on a short render of the caller's workload:
the path capacity of a wavefront (queue capacity), the grid caps of the
persistent traversal kernels and of the shading kernel (resident blocks of
128 threads per SM; the kernels' register budgets are fixed at compile time,
so occupancy is tuned through blocks per SM rather than block size), the
queue size from which shading queues are sorted by material, and the block
size of the camera-ray and film kernels.  The search is coordinate descent
from the defaults: each knob in turn takes the
candidate with the highest samples/s (device time), the others held.  No
counterpart in the reference.

Results can be cached in a JSON file keyed by device name and workload
signature (`cache`), so a later process reuses them without searching."""

from __future__ import annotations

import ctypes
import dataclasses
import json
import pathlib

from . import _abi
from .backend import CompiledScene, CudaPathTracerBackend, SampleRange

CANDIDATES = {
    "path_capacity": (1 << 20, 1 << 22, 1 << 23, 1 << 24),
    "sort_threshold": (0, 1 << 16, 1 << 20),
    "shadow_sort_threshold": (0, 1 << 16, 1 << 20),
    "ray_sort_threshold": (0, 1 << 16, 1 << 20),
    "traversal_blocks_per_sm": (8, 12, 16),
    "shade_blocks_per_sm": (8, 16, 32),
    "stream_block_size": (128, 256, 512),
}


@dataclasses.dataclass
class TuningResult:
    tuning: dict
    samples_per_s: float
    trials: list


def get_tuning(backend: CudaPathTracerBackend) -> dict:
    t = _abi.Tuning()
    _abi.check(backend.context.lib.psy_context_get_tuning(backend.context.handle, ctypes.byref(t)))
    return {name: int(getattr(t, name)) for name, _ in _abi.Tuning._fields_}


def set_tuning(backend: CudaPathTracerBackend, tuning: dict) -> None:
    t = _abi.Tuning(*[int(tuning.get(name, 0)) for name, _ in _abi.Tuning._fields_])
    _abi.check(backend.context.lib.psy_context_set_tuning(backend.context.handle, ctypes.byref(t)))


def _measure(backend, compiled: CompiledScene, settings, spp: int, repeats: int) -> float:
    best = 0.0
    session = backend.create_session(compiled, settings)
    try:
        for _ in range(repeats + 1):  # the first render allocates the path state
            session.reset(settings)
            if not session.render_samples(SampleRange(0, spp, 0, spp)):
                raise RuntimeError(f"render failed: {session.diagnostics}")
            st = session.stats()
            best = max(best, settings.full_width * settings.full_height * spp / (st.ms_total / 1e3))
    finally:
        session.close()
    return best


def autotune(backend: CudaPathTracerBackend, compiled: CompiledScene, settings, spp: int = 4, repeats: int = 1,
             candidates: dict | None = None, cache: str | pathlib.Path | None = None,
             signature: str = "") -> TuningResult:
    """Finds and applies the fastest tuning for `settings` on `compiled`."""
    key = None
    if cache is not None:
        device = backend.context.device_name if hasattr(backend.context, "device_name") else "cuda"
        key = f"{device}|{signature}|{settings.full_width}x{settings.full_height}|{spp}"
        path = pathlib.Path(cache)
        if path.exists():
            stored = json.loads(path.read_text()).get(key)
            if stored:
                set_tuning(backend, stored["tuning"])
                return TuningResult(stored["tuning"], stored["samples_per_s"], [])
    cands = candidates or CANDIDATES
    current = get_tuning(backend)
    trials = []
    set_tuning(backend, current)
    best_rate = _measure(backend, compiled, settings, spp, repeats)
    trials.append((dict(current), best_rate))
    for knob, values in cands.items():
        for v in values:
            if v == current.get(knob):
                continue
            trial = dict(current, **{knob: v})
            set_tuning(backend, trial)
            rate = _measure(backend, compiled, settings, spp, repeats)
            trials.append((trial, rate))
            if rate > best_rate:
                best_rate = rate
                current = trial
    set_tuning(backend, current)
    if key is not None:
        path = pathlib.Path(cache)
        data = json.loads(path.read_text()) if path.exists() else {}
        data[key] = {"tuning": current, "samples_per_s": best_rate}
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(data, indent=1))
    return TuningResult(current, best_rate, trials)
