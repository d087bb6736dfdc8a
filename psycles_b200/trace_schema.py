"""Per-path traces in the Psycles/Cycles differential trace schema, version 2.

The reference records one RGB triple per slot: 8 global slots, 4 events of
72 slots (48 named slots and 8 closures x 3), and 4 shadow events of 8
slots -- 328 slots in all (include/psycles/luisa/path_trace_schema.h:10-18,
tools/cycles_path_trace_schema.py).  Its comparator
(tools/compare_cycles_path_traces.py:140-280) reads a decoded trace
document -- {"schema", "version", "global": {slot: {"written", component:
value}}, "events": [{"slots": {...}, "closures": [...]}]} -- and gates each
component by a policy: exact, random-exact, float32 within
1e-6 + 2e-6 * max(|a|, |b|), topology (float32, or an equivalent surface
event), or reserved (not compared).

`document(trace)` turns a psy_path_trace (this library's trace record, from
the CUDA path or the oracle) into such a document.  A slot is written only
where the record holds every component it needs; the others stay unwritten
on both sides and the comparator skips them.  `compare(reference, actual)`
applies the same policies; tests check its verdicts against the reference
tool where that tool is present.

Written slots (event k = the path's k-th surface event, k < 4):
  global  header, rng, filter, ray_p, ray_d
  event   isect_coord, isect_id (surface hits), random_scalars, random_light,
          random_bsdf, bsdf_meta, bsdf_wo (a BSDF sample was drawn),
          post_throughput, post_flags, post_visibility (the path continued),
          nee_contribution (a light sample was drawn)
"""

from __future__ import annotations

import math
from dataclasses import dataclass

SCHEMA_NAME = "psycles.cycles-path-trace"
SCHEMA_VERSION = 2
GLOBAL_SLOTS, EVENT_SLOTS, SHADOW_SLOTS = 8, 72, 8
MAX_EVENTS, MAX_CLOSURES = 4, 8
SHADOW_BASE = GLOBAL_SLOTS + EVENT_SLOTS * MAX_EVENTS
SLOT_COUNT = SHADOW_BASE + SHADOW_SLOTS * MAX_EVENTS  # 328

EXACT, RANDOM, F32, TOPOLOGY, RESERVED = "exact", "random_exact", "float32", "topology", "reserved"

XYZ, RGB = ("x", "y", "z"), ("r", "g", "b")

# (name, components, policies) in slot order -- the schema's indexed contract
GLOBAL_LAYOUT = [
    ("header", ("schema_version", "pixel_x", "pixel_y"), (EXACT,) * 3),
    ("rng", ("sample", "rng_pixel_low16", "rng_pixel_high16"), (EXACT,) * 3),
    ("filter", ("filter_x", "filter_y", "reserved"), (RANDOM, RANDOM, RESERVED)),
    ("lens_time", ("time", "lens_u", "lens_v"), (RANDOM,) * 3),
    ("ray_p", XYZ, (F32,) * 3),
    ("ray_d", XYZ, (F32,) * 3),
    ("ray_range", ("tmin", "tmax", "time"), (F32,) * 3),
    ("reserved", XYZ, (RESERVED,) * 3),
]

_E, _R, _F = (EXACT,) * 3, (RANDOM,) * 3, (F32,) * 3
_EER, _EEF = (EXACT, EXACT, RESERVED), (EXACT, EXACT, F32)
EVENT_LAYOUT = [
    ("state_depth", ("event", "rng_offset", "bounce"), _E),
    ("state_lobes", ("transparent_bounce", "diffuse_bounce", "glossy_bounce"), _E),
    ("state_visibility", ("transmission_bounce", "visibility_low16", "visibility_high16"), _E),
    ("state_flags", ("path_flag_low16", "path_flag_high16", "continuation_probability"), _EEF),
    ("throughput", RGB, _F),
    ("ray_p", XYZ, _F),
    ("ray_d", XYZ, _F),
    ("ray_range", ("tmin", "tmax", "time"), _F),
    ("isect_coord", ("distance", "u", "v"), (F32, TOPOLOGY, TOPOLOGY)),
    ("isect_id", ("object", "primitive", "primitive_type"), (EXACT, TOPOLOGY, EXACT)),
    ("surface_meta", ("shader_low16", "shader_high16", "closure_count"), _E),
    ("surface_p", XYZ, _F),
    ("surface_ng", XYZ, _F),
    ("surface_n", XYZ, _F),
    ("random_scalars", ("terminate", "light_terminate", "reserved"), (RANDOM, RANDOM, RESERVED)),
    ("random_light", ("u", "v", "selection"), _R),
    ("random_bsdf", ("u", "v", "selection"), _R),
    ("light_meta", ("type", "emitter", "primitive"), _E),
    ("light_id", ("object", "group", "reserved"), _EER),
    ("light_pdf", ("pdf", "selection_pdf", "eval_factor"), _F),
    ("light_d", XYZ, _F),
    ("light_p", XYZ, _F),
    ("light_ng", XYZ, _F),
    ("light_eval", ("distance", "bsdf_pdf", "mis_weight"), _F),
    ("closure_pick", ("index", "type", "sample_weight"), _EEF),
    ("closure_random", ("u", "v", "selection_rescaled"), _R),
    ("closure_weight", RGB, _F),
    ("closure_n", XYZ, _F),
    ("bsdf_meta", ("pdf", "unguided_pdf", "label"), (F32, F32, EXACT)),
    ("bsdf_wo", XYZ, _F),
    ("bsdf_eval", RGB, _F),
    ("bsdf_roughness_eta", ("roughness_u", "roughness_v", "eta"), _F),
    ("post_depth", ("bounce", "transparent_bounce", "rng_offset"), _E),
    ("post_throughput", RGB, _F),
    ("post_ray_p", XYZ, _F),
    ("post_ray_d", XYZ, _F),
    ("post_flags", ("path_flag_low16", "path_flag_high16", "reserved"), _EER),
    ("post_mis", ("mis_ray_pdf", "min_ray_pdf", "continuation_probability"), _F),
    ("surface_flags", ("runtime_flag_low16", "runtime_flag_high16", "reserved"), _EER),
    ("post_visibility", ("visibility_low16", "visibility_high16", "reserved"), _EER),
    ("light_shader", ("shader_low16", "shader_high16", "reserved"), _EER),
    ("nee_bsdf", RGB, _F),
    ("nee_diffuse", RGB, _F),
    ("nee_glossy", RGB, _F),
    ("nee_weighted_bsdf", RGB, _F),
    ("nee_light_shader", RGB, _F),
    ("nee_unshadowed", RGB, _F),
    ("nee_contribution", RGB, _F),
]
CLOSURE_LAYOUT = [
    ("meta", ("index", "type", "sample_weight"), _EEF),
    ("weight", RGB, _F),
    ("normal", XYZ, _F),
]
SHADOW_LAYOUT = [
    ("shadow_ray_p", XYZ, _F),
    ("shadow_ray_d", XYZ, _F),
    ("shadow_ray_range", ("tmin", "tmax", "cast_shadow"), (F32, F32, EXACT)),
    ("shadow_source", ("object", "primitive", "skip_self"), _E),
    ("shadow_light", ("object", "primitive", "reserved"), _EER),
    ("shadow_hit_id", ("object", "primitive", "kind"), (RESERVED,) * 3),
    ("shadow_hit_coord", ("distance", "u", "v"), (RESERVED,) * 3),
    ("shadow_transmittance", RGB, (RESERVED,) * 3),
]


@dataclass(frozen=True)
class Slot:
    index: int
    scope: str  # "global", "event" (event and shadow slots) or "closure"
    name: str
    components: tuple
    policies: tuple
    event: int | None = None
    closure: int | None = None


def slots() -> list[Slot]:
    """All 328 slots in index order."""
    out = [Slot(i, "global", n, c, p) for i, (n, c, p) in enumerate(GLOBAL_LAYOUT)]
    for e in range(MAX_EVENTS):
        base = GLOBAL_SLOTS + e * EVENT_SLOTS
        out += [Slot(base + i, "event", n, c, p, event=e) for i, (n, c, p) in enumerate(EVENT_LAYOUT)]
        for k in range(MAX_CLOSURES):
            cb = base + len(EVENT_LAYOUT) + 3 * k
            out += [Slot(cb + i, "closure", n, c, p, event=e, closure=k) for i, (n, c, p) in enumerate(CLOSURE_LAYOUT)]
    for e in range(MAX_EVENTS):
        base = SHADOW_BASE + e * SHADOW_SLOTS
        out += [Slot(base + i, "event", n, c, p, event=e) for i, (n, c, p) in enumerate(SHADOW_LAYOUT)]
    assert len(out) == SLOT_COUNT and all(s.index == i for i, s in enumerate(out))
    return out


def _record(components, values=None) -> dict:
    rec = {"written": values is not None}
    for k, c in enumerate(components):
        rec[c] = values[k] if values is not None else 0.0
    return rec


def _split16(v: int) -> tuple[int, int]:
    return int(v) & 0xFFFF, (int(v) >> 16) & 0xFFFF


INVALID = 0xFFFFFFFF


def document(trace, source: str = "") -> dict:
    """The schema-v2 document of a psy_path_trace (psycles_b200._abi.PathTrace)."""
    g = {n: _record(c) for n, c, _ in GLOBAL_LAYOUT}
    lo, hi = _split16(trace.rng_hash)
    g["header"] = _record(GLOBAL_LAYOUT[0][1], [SCHEMA_VERSION, int(trace.pixel_x), int(trace.pixel_y)])
    g["rng"] = _record(GLOBAL_LAYOUT[1][1], [int(trace.sample), lo, hi])
    g["filter"] = _record(GLOBAL_LAYOUT[2][1], [float(trace.filter[0]), float(trace.filter[1]), 0.0])
    g["ray_p"] = _record(XYZ, [float(v) for v in trace.ray_origin])
    g["ray_d"] = _record(XYZ, [float(v) for v in trace.ray_direction])
    events = []
    for e in range(MAX_EVENTS):
        ev_slots = {n: _record(c) for n, c, _ in EVENT_LAYOUT + SHADOW_LAYOUT}
        closures = []
        if e < trace.event_count:
            ev = trace.events[e]
            if ev.hit_object != INVALID:
                ev_slots["isect_coord"] = _record(("distance", "u", "v"),
                                                  [float(ev.hit_t), float(ev.hit_u), float(ev.hit_v)])
                ev_slots["isect_id"] = _record(("object", "primitive", "primitive_type"),
                                               [int(ev.hit_object), int(ev.hit_primitive), 1])
            ev_slots["random_scalars"] = _record(("terminate", "light_terminate", "reserved"),
                                                 [float(ev.random_terminate), float(ev.random_light_terminate), 0.0])
            ev_slots["random_light"] = _record(("u", "v", "selection"), [float(v) for v in ev.random_light])
            ev_slots["random_bsdf"] = _record(("u", "v", "selection"), [float(v) for v in ev.random_bsdf])
            if ev.closure_index != INVALID:
                ev_slots["bsdf_meta"] = _record(("pdf", "unguided_pdf", "label"),
                                                [float(ev.bsdf_pdf), float(ev.bsdf_pdf), int(ev.label)])
                ev_slots["bsdf_wo"] = _record(XYZ, [float(v) for v in ev.wi])
                if ev.flag != 0 or ev.visibility != 0:
                    flo, fhi = _split16(ev.flag)
                    vlo, vhi = _split16(ev.visibility)
                    ev_slots["post_throughput"] = _record(RGB, [float(v) for v in ev.throughput])
                    ev_slots["post_flags"] = _record(("path_flag_low16", "path_flag_high16", "reserved"),
                                                     [flo, fhi, 0])
                    ev_slots["post_visibility"] = _record(("visibility_low16", "visibility_high16", "reserved"),
                                                          [vlo, vhi, 0])
            if ev.light_index != INVALID:
                ev_slots["nee_contribution"] = _record(RGB, [float(v) for v in ev.nee])
        events.append({"slots": ev_slots, "closures": closures})
    return {"schema": SCHEMA_NAME, "version": SCHEMA_VERSION, "source": source, "global": g, "events": events}


def _value(doc: dict, slot: Slot) -> dict:
    if slot.scope == "global":
        return doc["global"][slot.name]
    ev = doc["events"][slot.event]
    if slot.scope == "event":
        return ev["slots"][slot.name]
    found = next((c for c in ev["closures"] if c["index"] == slot.closure), None)
    return found[slot.name] if found is not None else _record(slot.components)


def _within(a: float, b: float, atol: float, rtol: float) -> bool:
    if not math.isfinite(a) or not math.isfinite(b):
        return a == b
    return abs(a - b) <= atol + rtol * max(abs(a), abs(b))


def compare(reference: dict, actual: dict, atol: float = 1.0e-6, rtol: float = 2.0e-6) -> list[str]:
    """Failing field names of `actual` against `reference` under the slot
    policies (an empty list passes).  Topology components fall back to the
    float32 bound; an isect mismatch there is a failure."""
    failures = []
    for slot in slots():
        if all(p == RESERVED for p in slot.policies):
            continue
        ra, aa = _value(reference, slot), _value(actual, slot)
        prefix = f"global.{slot.name}" if slot.scope == "global" else (
            f"events[{slot.event}].closure.{slot.closure}.{slot.name}" if slot.scope == "closure"
            else f"events[{slot.event}].{slot.name}")
        if ra["written"] != aa["written"]:
            failures.append(prefix + ".written")
            continue
        if not ra["written"]:
            continue
        for comp, policy in zip(slot.components, slot.policies):
            if policy == RESERVED:
                continue
            x, y = ra[comp], aa[comp]
            ok = x == y if policy in (EXACT, RANDOM) else _within(float(x), float(y), atol, rtol)
            if not ok:
                failures.append(f"{prefix}.{comp}")
    return failures
