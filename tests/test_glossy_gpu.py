"""Glossy closures on the device against the oracle (gpu-marked).

The glossy scene (GGX and Beckmann at roughness 0 -- a mirror, sampled as a
singular direction -- through 0.6, on smooth-normal spheres that exercise
the specular-reflection normal correction, one material without the
correction, and random diffuse + glossy, glossy + transparent and
value-linked-roughness mixtures) renders through the CUDA path; passes and
per-path traces must match the oracle (the reference comparator's bar),
with the flat light distribution and with the light tree.  The traces must
cover glossy (reflect | glossy) and singular (reflect | singular) bounces."""

import numpy as np
import pytest

from _parity import assert_passes_match, assert_traces_match
from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


@pytest.mark.parametrize("light_tree", [0, 1])
def test_glossy_scene_matches_oracle(backend, light_tree):
    scene = scenes.glossy_scene(seed=1)
    st = scenes.render_settings(96, 72, max_bounces=6, use_light_tree=light_tree)
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    session = backend.create_session(compiled.scene, st)
    assert session.render_samples(SampleRange(0, 16, 0, 16)), session.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 16, 16)
    assert_passes_match(session, film, PASSES)


def _traced_paths(prepared, seed, want=6, budget=2000):
    """Pixels and samples whose oracle paths take glossy (reflect | glossy)
    and singular (reflect | singular) bounces -- `want` of each -- plus a
    few others, chosen by rendering candidates with the oracle."""
    rng = np.random.default_rng(seed)
    glossy, singular, other = [], [], []
    for _ in range(budget):
        x, y, s = int(rng.integers(0, 96)), int(rng.integers(0, 72)), int(rng.integers(0, 16))
        st = scenes.render_settings(96, 72, max_bounces=6, window_x=x, window_y=y, window_width=1, window_height=1)
        t = OracleFilm(st).render_prepared(prepared, s, 1, 16, trace=(x, y, s))
        labels = {t.events[k].label for k in range(t.event_count)}
        if 2 | 16 in labels and len(singular) < want:
            singular.append((x, y, s))
        elif 2 | 8 in labels and len(glossy) < want:
            glossy.append((x, y, s))
        elif len(other) < 4:
            other.append((x, y, s))
        if len(glossy) >= want and len(singular) >= want and len(other) >= 4:
            break
    return glossy + singular + other, len(glossy), len(singular)


@pytest.mark.parametrize("seed", [1, 2])
def test_glossy_traces_bit_exact(backend, seed):
    scene = scenes.glossy_scene(seed=seed)
    compiled = backend.compile_scene(scene).scene
    prepared = OracleScene(scene.to_desc())
    paths, n_glossy, n_singular = _traced_paths(prepared, seed)
    assert n_glossy >= 6 and n_singular >= 6, (n_glossy, n_singular)
    for x, y, s in paths:
        st = scenes.render_settings(96, 72, max_bounces=6, window_x=x, window_y=y, window_width=1, window_height=1)
        session = backend.create_session(compiled, st)
        session.request_trace(x, y, s)
        assert session.render_samples(SampleRange(s, 1, 0, 16)), session.diagnostics
        ot = OracleFilm(st).render_prepared(prepared, s, 1, 16, trace=(x, y, s))
        assert_traces_match(session.read_trace(), ot, where=(x, y, s))


def test_glossy_batched_equals_alone(backend):
    """Glossy sessions in a shared wavefront end as they do alone, also when
    the wavefront mixes them with a scene without glossy closures (the
    wavefront then shades with the glossy-capable kernel variant)."""
    from psycles_b200.backend import BatchRenderer
    comp = backend.compile_scene(scenes.glossy_scene(seed=3)).scene
    plain = backend.compile_scene(scenes.small_test_scene(seed=4)).scene
    work = [(comp, scenes.render_settings(64, 48, max_bounces=5, seed=k)) for k in range(3)]
    work.append((plain, scenes.render_settings(64, 48, max_bounces=5, seed=9)))
    alone = []
    for sc, st in work:
        s = backend.create_session(sc, st)
        assert s.render_samples(SampleRange(0, 4, 0, 4))
        alone.append(s.read_pass(_abi.PASS_COMBINED))
    batch = BatchRenderer(backend.context, path_capacity=20000)
    sessions = [backend.create_session(sc, st) for sc, st in work]
    assert batch.render([(s, SampleRange(0, 4, 0, 4)) for s in sessions])
    for s, ref in zip(sessions, alone):
        assert np.array_equal(s.read_pass(_abi.PASS_COMBINED).view(np.uint32), ref.view(np.uint32))


def test_malformed_glossy_is_rejected(backend):
    """A distribution outside GGX and Beckmann, or a glossy colour input out
    of the parameter block, fails at compile time."""
    N = _abi.INPUT_NONE
    for closure in [(_abi.CLOSURE_GLOSSY, 7, 0, 0, N, 0), (_abi.CLOSURE_GLOSSY, 0, 0, 5, N, 0),
                    (_abi.CLOSURE_GLOSSY, 0, 0, N, N, 0)]:
        sc = scenes.cornell_box()
        m = sc.materials[0]
        m.program.closures = np.array([closure], np.uint32).reshape(-1, 6)
        m.program.values = np.zeros((0, 8), np.uint32)
        m.program.root = 0
        m.parameters.scalars = np.array([0.3], np.float32)
        m.parameters.vectors = np.array([[0.5, 0.5, 0.5]], np.float32)
        assert not backend.compile_scene(sc).ok(), closure


def test_oversized_closure_trees_are_refused(backend):
    """A material with more BSDF closures than a shading point holds (16)
    is refused at compile instead of rendering with closures dropped; 16
    compile."""
    N = _abi.INPUT_NONE

    def scene_with(leaves):
        closures = [(_abi.CLOSURE_DIFFUSE, 0, 0, 0, N, N)] * leaves
        k = leaves
        prev = 0
        for i in range(1, leaves):
            closures.append((_abi.CLOSURE_ADD, prev, i, N, N, N))
            prev = k
            k += 1
        sc = scenes.cornell_box()
        m = sc.materials[0]
        m.program.closures = np.array(closures, np.uint32).reshape(-1, 6)
        m.program.values = np.zeros((0, 8), np.uint32)
        m.program.root = len(closures) - 1
        m.parameters.scalars = np.array([0.3], np.float32)
        m.parameters.vectors = np.array([[0.5, 0.5, 0.5]], np.float32)
        return sc
    assert backend.compile_scene(scene_with(16)).ok()
    assert not backend.compile_scene(scene_with(17)).ok()
