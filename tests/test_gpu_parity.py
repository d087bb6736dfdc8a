"""CUDA kernels against the CPU oracle, through the C ABI (gpu-marked).

Bar: the Sobol lookup, hit identities, closure picks and path-state
transitions are bit-exact; continuous per-path fields within
1e-6 + 2e-6 * max(|a|, |b|) (the reference's float32 comparator policy);
final passes within relative RMSE 1e-3 of the oracle at the same seed and
spp (rmse / rms(reference))."""

import ctypes

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_DENOISING_NORMAL,
          _abi.PASS_DENOISING_ALBEDO, _abi.PASS_SAMPLE_COUNT]


def rel_rmse(a, b):
    ref_rms = float(np.sqrt(np.mean(np.square(b.astype(np.float64)))))
    return float(np.sqrt(np.mean(np.square(a.astype(np.float64) - b.astype(np.float64))))) / max(ref_rms, 1e-12)


def render_both(backend, scene, settings, first, count, total, chunks=None, trace=None):
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    sess = backend.create_session(comp.scene, settings)
    assert sess is not None
    if trace:
        sess.request_trace(*trace)
    for f, c in (chunks or [(first, count)]):
        assert sess.render_samples(SampleRange(f, c, 0, total)), sess.diagnostics
    film = OracleFilm(settings)
    otrace = film.render(scene.to_desc(), first, count, total, threads=0, trace=trace)
    return sess, film, otrace


def test_device_sobol_golden_bits(backend, golden):
    probe = golden["sobol"]["device_probe"]
    x, y = probe["pixel"]
    q = np.array([[x, y, probe["seed"], s, d] for s, d in probe["queries"]], np.uint32)
    out = np.zeros((len(q), 4), np.float32)
    idx = np.zeros(len(q), np.uint32)
    _abi.check(backend.context.lib.psy_debug_sobol_samples(
        backend.context.handle, 256, _abi.ptr(q, ctypes.c_uint32), len(q), _abi.ptr(out), _abi.ptr(idx, ctypes.c_uint32)))
    assert idx.tolist() == probe["shuffled_indices"]
    assert out.view(np.uint32).tolist() == probe["expected_bits"]


def test_cornell_box_passes_match_oracle(backend):
    scene = scenes.cornell_box()
    st = scenes.render_settings(128, 128, max_bounces=4)
    sess, film, _ = render_both(backend, scene, st, 0, 8, 16)
    for kind in PASSES:
        got = sess.read_pass(kind)
        ref = film.resolve(kind)
        assert got.shape == ref.shape
        e = rel_rmse(got, ref)
        assert e <= 1e-3, (kind, e)
        mismatch = np.mean(got.view(np.uint32) != ref.view(np.uint32))
        assert mismatch <= 0.01, (kind, mismatch)


def test_small_scene_all_closures_and_lights(backend):
    scene = scenes.small_test_scene(seed=3)
    st = scenes.render_settings(96, 72, max_bounces=6)
    sess, film, _ = render_both(backend, scene, st, 0, 6, 8)
    for kind in PASSES:
        e = rel_rmse(sess.read_pass(kind), film.resolve(kind))
        assert e <= 1e-3, (kind, e)


def test_per_path_trace_bit_exact(backend):
    scene = scenes.small_test_scene(seed=1)
    st = scenes.render_settings(64, 48, max_bounces=6)
    for px, py, s in [(31, 20, 1), (10, 40, 2), (50, 10, 0)]:
        sess, film, ot = render_both(backend, scene, st, 0, 3, 4, trace=(px, py, s))
        gt = sess.read_trace()
        assert gt.valid == 1 and ot.valid == 1
        assert (gt.pixel_x, gt.pixel_y, gt.sample, gt.rng_hash) == (ot.pixel_x, ot.pixel_y, ot.sample, ot.rng_hash)
        assert gt.event_count == ot.event_count
        for k in range(gt.event_count):
            a, b = gt.events[k], ot.events[k]
            for f in ("rng_offset", "bounce", "transparent_bounce", "flag", "visibility", "hit_object",
                      "hit_primitive", "closure_index", "label", "light_kind", "light_index", "terminated"):
                assert getattr(a, f) == getattr(b, f), (k, f)
            for f in ("hit_t", "hit_u", "hit_v", "random_terminate", "random_light_terminate",
                      "continuation_probability", "bsdf_pdf"):
                x, y = getattr(a, f), getattr(b, f)
                assert abs(x - y) <= 1e-6 + 2e-6 * max(abs(x), abs(y)), (k, f, x, y)
            for f in ("random_light", "random_bsdf", "wi", "throughput", "emission", "nee"):
                x, y = np.array(getattr(a, f)), np.array(getattr(b, f))
                assert np.all(np.abs(x - y) <= 1e-6 + 2e-6 * np.maximum(np.abs(x), np.abs(y))), (k, f, x, y)
        assert np.allclose(np.array(gt.radiance), np.array(ot.radiance), rtol=2e-6, atol=1e-6)


def test_progressive_chunks_equal_one_dispatch(backend):
    scene = scenes.cornell_box()
    st = scenes.render_settings(64, 64, max_bounces=4)
    comp = backend.compile_scene(scene).scene
    a = backend.create_session(comp, st)
    assert a.render_samples(SampleRange(0, 8, 0, 8))
    b = backend.create_session(comp, st)
    for f in (0, 3, 5):
        assert b.render_samples(SampleRange(f, {0: 3, 3: 2, 5: 3}[f], 0, 8))
    assert np.array_equal(a.read_pass(_abi.PASS_COMBINED), b.read_pass(_abi.PASS_COMBINED))
    assert b.rendered_samples() == 8


def test_window_matches_full_frame(backend):
    scene = scenes.cornell_box()
    full = scenes.render_settings(64, 64, max_bounces=4)
    win = scenes.render_settings(64, 64, max_bounces=4, window_x=16, window_y=8, window_width=24, window_height=40)
    comp = backend.compile_scene(scene).scene
    a = backend.create_session(comp, full)
    b = backend.create_session(comp, win)
    assert a.render_samples(SampleRange(0, 4, 0, 4)) and b.render_samples(SampleRange(0, 4, 0, 4))
    assert np.array_equal(a.read_pass(0)[8:48, 16:40], b.read_pass(0))


def test_render_contract_errors(backend):
    scene = scenes.cornell_box()
    comp = backend.compile_scene(scene).scene
    sess = backend.create_session(comp, scenes.render_settings(32, 32))
    assert not sess.render_samples(SampleRange(0, 0, 0, 4))      # empty range
    assert not sess.render_samples(SampleRange(2, 4, 0, 4))      # beyond total
    assert sess.render_samples(SampleRange(0, 2, 0, 4))
    assert not sess.render_samples(SampleRange(2, 2, 0, 8))      # total changed
    sess.cancel()
    assert not sess.render_samples(SampleRange(2, 2, 0, 4))      # cancelled
    bad = scenes.render_settings(32, 32, window_x=30, window_width=8)
    assert backend.create_session(comp, bad) is None


def test_rebind_parameters_equals_recompiled_scene(backend):
    scene = scenes.cornell_box()
    st = scenes.render_settings(48, 48, max_bounces=4)
    comp = backend.compile_scene(scene).scene
    comp.rebind_parameters(1, scene.materials[1].parameters.scalars, np.array([[0.1, 0.6, 0.7]], np.float32))
    s1 = backend.create_session(comp, st)
    assert s1.render_samples(SampleRange(0, 4, 0, 4))
    from psycles_b200.materials import diffuse_material
    db = scenes.SceneDatabase(scene)
    edited = db.apply(material_graphs={1: diffuse_material((0.1, 0.6, 0.7))})
    comp2 = backend.compile_scene(edited).scene
    s2 = backend.create_session(comp2, st)
    assert s2.render_samples(SampleRange(0, 4, 0, 4))
    assert np.array_equal(s1.read_pass(0), s2.read_pass(0))
