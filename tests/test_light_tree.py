"""Many-light tree: oracle self-consistency on CPU, and the device tree
(selection, selection pdf, reverse pdf; tree-mode renders) against the
oracle through the C ABI (gpu-marked).

Bar: selected emitter identities equal; pdfs within
1e-6 + 2e-6 * max(|a|, |b|); rendered passes within relative RMSE 1e-3."""

import ctypes

import numpy as np
import pytest

from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]
INVALID = 0xFFFFFFFF


def tree_scene_small():
    return scenes.small_test_scene(seed=3)


def tree_scene_many():
    return scenes.many_light_scene(seed=1, boxes=40, emitters=1500, emission_materials=64)


def shading_queries(seed: int, count: int, lo, hi, emitters: int):
    rng = np.random.default_rng(seed)
    q = np.zeros((count, 8), np.float32)
    q[:, 0:3] = rng.uniform(lo, hi, (count, 3))
    q[:, 3] = rng.uniform(0.0, 1.0, count)
    n = rng.normal(size=(count, 3))
    q[:, 4:7] = n / np.linalg.norm(n, axis=1, keepdims=True)
    q[:, 7] = (rng.uniform(size=count) < 0.25).astype(np.float32)
    pdf_emitters = rng.integers(0, emitters, count).astype(np.uint32)
    return q, pdf_emitters


def close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= 1e-6 + 2e-6 * np.maximum(np.abs(a), np.abs(b))


# ------------------------------------------------------------------ CPU

def test_oracle_tree_sample_pdf_consistent():
    """For one shading point, the selection frequency over a fine u grid is
    the reverse pdf of each emitter, and the pdf returned with a sample is
    the reverse pdf of the emitter it picked."""
    scene = tree_scene_small()
    osc = OracleScene(scene.to_desc())
    n = 20000
    u = (np.arange(n, dtype=np.float64) + 0.5) / n
    q = np.zeros((n, 8), np.float32)
    q[:, 0:3] = (0.3, 0.8, -0.4)
    q[:, 3] = u.astype(np.float32)
    q[:, 4:7] = (0.0, 1.0, 0.0)
    sel, spdf, _ = osc.light_tree_query(q, np.zeros(n, np.uint32))
    # A descent can end in a cluster whose conservative bound was important
    # while none of its members is (e.g. lights facing away); that mass
    # selects nothing, as in the reference.
    valid = sel != INVALID
    assert valid.mean() > 0.5
    ids, counts = np.unique(sel[valid], return_counts=True)
    qe = np.repeat(q[:1], len(ids), axis=0)
    _, _, rpdf = osc.light_tree_query(qe, ids.astype(np.uint32))
    freq = counts / n
    assert np.all(np.abs(freq - rpdf) <= 2e-3 + 0.02 * rpdf), np.c_[ids, freq, rpdf]
    assert abs(rpdf.sum() - valid.mean()) <= 5e-3
    # the sample's pdf equals the reverse pdf of what it picked
    _, _, back = osc.light_tree_query(q[valid], sel[valid])
    assert np.all(np.abs(spdf[valid] - back) <= 1e-5 * np.maximum(back, 1e-12) + 1e-9)


def test_oracle_tree_render_agrees_with_flat_distribution():
    """Tree and flat light selection are both unbiased estimators of the
    same image: their means agree within Monte-Carlo noise."""
    scene = tree_scene_small()
    means = []
    for tree in (0, 1):
        st = scenes.render_settings(24, 18, max_bounces=3, use_light_tree=tree)
        film = OracleFilm(st)
        film.render(scene.to_desc(), 0, 64, 64, threads=0)
        means.append(float(film.resolve(_abi.PASS_COMBINED)[..., :3].mean()))
    assert abs(means[0] - means[1]) <= 0.05 * max(means), means


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("which", ["small", "many"])
def test_device_tree_queries_match_oracle(backend, which):
    scene = tree_scene_small() if which == "small" else tree_scene_many()
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    osc = OracleScene(scene.to_desc())
    lo, hi = ((-4, 0, -4), (4, 4, 4)) if which == "small" else ((-12, 0, -12), (12, 21, 12))
    q, pe = shading_queries(7, 20000, lo, hi, osc.emitter_count())
    o_sel, o_spdf, o_rpdf = osc.light_tree_query(q, pe)
    n = q.shape[0]
    d_sel = np.zeros(n, np.uint32)
    d_spdf = np.zeros(n, np.float32)
    d_rpdf = np.zeros(n, np.float32)
    _abi.check(backend.context.lib.psy_debug_light_tree(
        comp.scene.handle, _abi.ptr(q), _abi.ptr(pe, ctypes.c_uint32), n, _abi.ptr(d_sel, ctypes.c_uint32),
        _abi.ptr(d_spdf), _abi.ptr(d_rpdf)))
    same = d_sel == o_sel
    assert same.mean() >= 0.999, same.mean()
    assert (o_sel != INVALID).mean() > 0.5
    assert close(d_spdf[same], o_spdf[same]).mean() >= 0.999
    assert close(d_rpdf, o_rpdf).mean() >= 0.999
    assert (o_rpdf > 0).mean() > 0.1


@pytest.mark.gpu
def test_tree_render_small_scene_matches_oracle(backend):
    scene = tree_scene_small()
    st = scenes.render_settings(96, 72, max_bounces=6, use_light_tree=1)
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    sess = backend.create_session(comp.scene, st)
    assert sess.render_samples(SampleRange(0, 6, 0, 8)), sess.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 6, 8, threads=0)
    for kind in PASSES:
        got, ref = sess.read_pass(kind), film.resolve(kind)
        rms = float(np.sqrt(np.mean(np.square(ref.astype(np.float64)))))
        e = float(np.sqrt(np.mean(np.square(got.astype(np.float64) - ref)))) / max(rms, 1e-12)
        assert e <= 1e-3, (kind, e)


@pytest.mark.gpu
def test_tree_render_many_lights_matches_oracle(backend):
    scene = tree_scene_many()
    st = scenes.render_settings(64, 48, max_bounces=4, use_light_tree=1)
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    sess = backend.create_session(comp.scene, st)
    assert sess.render_samples(SampleRange(0, 2, 0, 4)), sess.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 2, 4, threads=0)
    got, ref = sess.read_pass(_abi.PASS_COMBINED), film.resolve(_abi.PASS_COMBINED)
    rms = float(np.sqrt(np.mean(np.square(ref.astype(np.float64)))))
    e = float(np.sqrt(np.mean(np.square(got.astype(np.float64) - ref)))) / max(rms, 1e-12)
    assert e <= 1e-3, e
    assert rms > 0.0


@pytest.mark.gpu
def test_tree_trace_light_picks_bit_exact(backend):
    """Per-path traces with the tree: every event's light pick and the
    radiance along the path agree with the oracle."""
    scene = tree_scene_small()
    st = scenes.render_settings(64, 48, max_bounces=6, use_light_tree=1)
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    for x, y, s in [(10, 20, 0), (33, 17, 1), (50, 40, 2), (5, 5, 3)]:
        sess = backend.create_session(comp.scene, st)
        sess.request_trace(x, y, s)
        assert sess.render_samples(SampleRange(0, 4, 0, 4)), sess.diagnostics
        gt = sess.read_trace()
        film = OracleFilm(st)
        ot = film.render(scene.to_desc(), 0, 4, 4, threads=0, trace=(x, y, s))
        assert gt.valid == 1 and ot.valid == 1
        assert gt.event_count == ot.event_count
        for k in range(gt.event_count):
            g, o = gt.events[k], ot.events[k]
            assert (g.light_kind, g.light_index) == (o.light_kind, o.light_index), (x, y, s, k)
        assert np.allclose(np.array(gt.radiance), np.array(ot.radiance), rtol=2e-6, atol=1e-6)


@pytest.mark.gpu
def test_tree_built_on_first_use_and_rebuilt_after_emission_edit(backend):
    """compile_scene leaves the tree unbuilt; the first session that selects
    lights from it builds it.  A parameter edit of an emissive material
    rebuilds a built tree, and the render afterwards equals a render of the
    scene compiled with the edited parameters, bit for bit."""
    import copy
    scene = tree_scene_small()
    st = scenes.render_settings(64, 48, max_bounces=4, use_light_tree=1)
    comp = backend.compile_scene(scene).scene
    assert comp.build_stats().light_tree_builds == 0
    flat = backend.create_session(comp, scenes.render_settings(64, 48, max_bounces=4))
    assert flat.render_samples(SampleRange(0, 1, 0, 1))
    assert comp.build_stats().light_tree_builds == 0
    before_bytes = comp.device_bytes()
    sess = backend.create_session(comp, st)
    assert comp.build_stats().light_tree_builds == 1 and comp.device_bytes() > before_bytes
    k = next(i for i, m in enumerate(scene.materials) if m.program.has_emission and m.parameters.scalars.size)
    sc = scene.materials[k].parameters.scalars * np.float32(3.0)
    vc = scene.materials[k].parameters.vectors[::-1].copy()
    comp.rebind_parameters(k, sc, vc)
    assert comp.build_stats().light_tree_builds == 2
    sess.reset(st)
    assert sess.render_samples(SampleRange(0, 4, 0, 4)), sess.diagnostics
    edited = copy.deepcopy(scene)
    edited.materials[k].parameters.scalars[:] = sc
    edited.materials[k].parameters.vectors[:] = vc
    comp2 = backend.compile_scene(edited).scene
    ref = backend.create_session(comp2, st)
    assert ref.render_samples(SampleRange(0, 4, 0, 4)), ref.diagnostics
    for kind in PASSES:
        assert np.array_equal(sess.read_pass(kind).view(np.uint32), ref.read_pass(kind).view(np.uint32)), kind
    stats = comp2.build_stats()
    assert stats.total_ms > 0.0 and stats.build_threads >= 1 and stats.light_tree_ms > 0.0
