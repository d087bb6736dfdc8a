"""Comparison helpers shared by the GPU parity tests (not a test module).

Bar (the reference comparator policy, docs/cycles-path-trace.md:667-679):
discrete and random per-path fields bit-exact; continuous float32 fields
within 1e-6 + 2e-6 * max(|a|, |b|); final passes within relative RMSE 1e-3
(tools/compare_cycles.py:154-211: rmse / rms(reference))."""

import numpy as np

DISCRETE = ("rng_offset", "bounce", "transparent_bounce", "flag", "visibility", "hit_object", "hit_primitive",
            "closure_index", "label", "light_kind", "light_index", "terminated")
SCALARS = ("hit_t", "hit_u", "hit_v", "random_terminate", "random_light_terminate", "continuation_probability",
           "bsdf_pdf")
VECTORS = ("random_light", "random_bsdf", "wi", "throughput", "emission", "nee")
RANDOM = ("random_terminate", "random_light_terminate", "random_light", "random_bsdf")


def rel_rmse(a, b) -> float:
    ref_rms = float(np.sqrt(np.mean(np.square(b.astype(np.float64)))))
    return float(np.sqrt(np.mean(np.square(a.astype(np.float64) - b.astype(np.float64))))) / max(ref_rms, 1e-12)


def close(x, y) -> bool:
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    return bool(np.all(np.abs(x - y) <= 1e-6 + 2e-6 * np.maximum(np.abs(x), np.abs(y))))


def assert_traces_match(gt, ot, where=None) -> None:
    """CUDA trace `gt` against oracle trace `ot`: header and discrete fields
    bit-exact, Sobol randoms bit-exact, continuous fields within the float bar."""
    assert gt.valid == 1 and ot.valid == 1, where
    assert (gt.pixel_x, gt.pixel_y, gt.sample, gt.rng_hash) == (ot.pixel_x, ot.pixel_y, ot.sample, ot.rng_hash), where
    assert gt.event_count == ot.event_count, (where, gt.event_count, ot.event_count)
    for k in range(gt.event_count):
        a, b = gt.events[k], ot.events[k]
        for f in DISCRETE:
            assert getattr(a, f) == getattr(b, f), (where, k, f, getattr(a, f), getattr(b, f))
        for f in RANDOM:
            x = np.array(getattr(a, f), np.float32).reshape(-1)
            y = np.array(getattr(b, f), np.float32).reshape(-1)
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), (where, k, f, x, y)
        for f in SCALARS + VECTORS:
            assert close(getattr(a, f), getattr(b, f)), (where, k, f, getattr(a, f), getattr(b, f))
    assert close(gt.radiance, ot.radiance), (where, list(gt.radiance), list(ot.radiance))
    # the same pair as schema-v2 documents under the reference comparator's
    # slot policies (psycles_b200.trace_schema)
    from psycles_b200 import trace_schema
    failures = trace_schema.compare(trace_schema.document(ot, "oracle"), trace_schema.document(gt, "cuda"))
    assert failures == [], (where, failures)


def assert_passes_match(session, film, passes, max_bit_mismatch=0.01) -> dict:
    """Every pass of `session` against the oracle film; returns the errors."""
    errors = {}
    for kind in passes:
        got = session.read_pass(kind)
        ref = film.resolve(kind)
        assert got.shape == ref.shape, (kind, got.shape, ref.shape)
        e = rel_rmse(got, ref)
        mismatch = float(np.mean(got.view(np.uint32) != ref.view(np.uint32)))
        errors[kind] = (e, mismatch)
        assert e <= 1e-3, (kind, e)
        assert mismatch <= max_bit_mismatch, (kind, mismatch)
    return errors


def trace_tags(trace, scene) -> set:
    """What a path crosses: transparent surfaces, a multi-closure pick, the
    scene's largest mesh (the deepest BLAS), NEE, a miss."""
    sizes = [len(m.indices) for m in scene.meshes]
    deepest = int(np.argmax(sizes))
    tags = set()
    for k in range(trace.event_count):
        e = trace.events[k]
        if e.label & 32:
            tags.add("transparent")
        if e.closure_index not in (0, 0xFFFFFFFF):
            tags.add("mix")
        if e.hit_object != 0xFFFFFFFF and e.hit_object < len(scene.instances) and \
                scene.instances[e.hit_object].mesh == deepest:
            tags.add("deep")
        if e.light_index != 0xFFFFFFFF and any(v != 0.0 for v in e.nee):
            tags.add("nee")
        if e.hit_object == 0xFFFFFFFF:
            tags.add("miss")
    return tags
