"""Batched wavefronts (psy_batch_*): many sessions' sample ranges in shared
path state.

CPU: the wavefront plan covers every job's samples once, in order, one item
per job per wavefront, within the path capacity.  GPU: every session of a
batch ends bit-identical to rendering it alone with render_samples (all
passes), with and without CUDA-graph replay, across progressive calls."""

import numpy as np
import pytest

from psycles_b200 import _abi, scenes
from psycles_b200.backend import BatchRenderer, SampleRange, batch_plan


def _check_plan(pixels, samples, capacity):
    plan = batch_plan(pixels, samples, capacity)
    cap = max([capacity] + list(pixels))
    nxt = [0] * len(pixels)
    for wave in np.unique(plan[:, 1]):
        rows = plan[plan[:, 1] == wave]
        jobs = rows[:, 0].tolist()
        assert len(jobs) == len(set(jobs)), "a job appears twice in one wavefront"
        used = 0
        film = 0
        for job, _, begin, first, count, film_begin in rows.tolist():
            assert begin == used and film_begin == film
            assert first == nxt[job], "samples out of order"
            assert count >= 1
            nxt[job] += count
            used += count * pixels[job]
            film += pixels[job]
        assert used <= cap
    assert nxt == list(samples)
    return plan


def test_plan_covers_every_sample_in_order():
    rng = np.random.default_rng(3)
    for _ in range(20):
        n = int(rng.integers(1, 40))
        pixels = [int(rng.choice([128 * 128, 256 * 256, 512 * 512, 1024 * 768, 1920 * 1080, 37])) for _ in range(n)]
        samples = [int(rng.integers(1, 65)) for _ in range(n)]
        _check_plan(pixels, samples, int(rng.choice([1 << 20, 1 << 22, 100000])))


def test_plan_grows_capacity_to_the_largest_window():
    plan = _check_plan([1920 * 1080, 64], [2, 5], 1000)
    assert plan[:, 4].max() >= 1


def test_plan_fills_the_wavefront():
    # 64 small viewports of 1 spp fit one wavefront
    plan = _check_plan([128 * 128] * 64, [1] * 64, 1 << 22)
    assert np.unique(plan[:, 1]).size == 1


# ------------------------------------------------------------------ GPU

def _scenes():
    return [scenes.cornell_box(), scenes.small_test_scene(seed=2), scenes.lamp_scene(seed=1)]


def _jobs():
    # (scene index, width, height, spp, light tree)
    return [(0, 64, 64, 8, 0), (1, 96, 72, 6, 0), (2, 80, 60, 5, 1), (1, 40, 30, 3, 1), (0, 33, 17, 7, 0)]


def _render_alone(backend, compiled, job):
    si, w, h, spp, tree = job
    st = scenes.render_settings(w, h, max_bounces=5, use_light_tree=tree, seed=si)
    sess = backend.create_session(compiled[si], st)
    assert sess.render_samples(SampleRange(0, spp, 0, spp)), sess.diagnostics
    return sess


def _passes(sess):
    return {k: sess.read_pass(k) for k in (_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO,
                                           _abi.PASS_SAMPLE_COUNT)}


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_sessions_alone(backend, use_graph):
    compiled = []
    for sc in _scenes():
        comp = backend.compile_scene(sc)
        assert comp.ok(), comp.diagnostics
        compiled.append(comp.scene)
    alone = [_passes(_render_alone(backend, compiled, j)) for j in _jobs()]
    # a small capacity splits every session over several wavefronts
    batch = BatchRenderer(backend.context, path_capacity=20000, use_graph=use_graph)
    sessions = []
    for si, w, h, spp, tree in _jobs():
        st = scenes.render_settings(w, h, max_bounces=5, use_light_tree=tree, seed=si)
        sessions.append((backend.create_session(compiled[si], st), spp))
    assert batch.render([(s, SampleRange(0, spp, 0, spp)) for s, spp in sessions])
    stats = batch.stats()
    assert stats.wavefronts > 1 and stats.jobs == len(sessions)
    assert stats.samples == sum(w * h * spp for _, w, h, spp, _ in _jobs())
    if use_graph:
        assert stats.graph_launches == stats.wavefronts
    for (s, _), ref in zip(sessions, alone):
        got = _passes(s)
        for k in ref:
            assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
        assert s.rendered_samples() == int(ref[_abi.PASS_SAMPLE_COUNT].max())


@pytest.mark.gpu
def test_batch_progressive_calls_equal_one_call(backend):
    comp = backend.compile_scene(scenes.small_test_scene(seed=4))
    assert comp.ok()
    st = scenes.render_settings(64, 48, max_bounces=4)
    one = backend.create_session(comp.scene, st)
    two = backend.create_session(comp.scene, scenes.render_settings(64, 48, max_bounces=4))
    batch = BatchRenderer(backend.context, path_capacity=5000)
    assert batch.render([(one, SampleRange(0, 8, 0, 8))])
    assert batch.render([(two, SampleRange(0, 3, 0, 8))])
    assert batch.render([(two, SampleRange(3, 5, 0, 8))])
    a, b = one.read_pass(_abi.PASS_COMBINED), two.read_pass(_abi.PASS_COMBINED)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_batch_rejects_bad_calls(backend):
    comp = backend.compile_scene(scenes.cornell_box())
    s = backend.create_session(comp.scene, scenes.render_settings(16, 16))
    batch = BatchRenderer(backend.context)
    assert not batch.render([(s, SampleRange(0, 2, 0, 4)), (s, SampleRange(2, 2, 0, 4))])
    assert "twice" in s.diagnostics[-1].message
    assert not batch.render([(s, SampleRange(0, 5, 0, 4))])
    assert batch.render([(s, SampleRange(0, 2, 0, 4))])
    assert not batch.render([(s, SampleRange(2, 2, 0, 8))])  # total changed within the session
