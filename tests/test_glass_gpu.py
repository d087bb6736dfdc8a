"""Glass and refraction closures on the device against the oracle
(gpu-marked).

The glass scene (smooth and rough GGX glass, Beckmann glass, tinted glass,
smooth and rough refraction, refraction mixed with diffuse, on closed
spheres and boxes that paths enter and leave) renders through the CUDA
path; passes and per-path traces must match the oracle with the flat light
distribution and with the light tree, the traces covering transmitted and
reflected glossy and singular bounces.  A glass closure mixed with another
BSDF closure is refused at compile; a batched wavefront equals the sessions
alone."""

import numpy as np
import pytest

from _parity import assert_passes_match, assert_traces_match
from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange
from psycles_b200.materials import ShaderGraph

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


@pytest.mark.parametrize("light_tree", [0, 1])
def test_glass_scene_matches_oracle(backend, light_tree):
    scene = scenes.glass_scene(seed=1)
    st = scenes.render_settings(96, 72, max_bounces=8, use_light_tree=light_tree)
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    session = backend.create_session(compiled.scene, st)
    assert session.render_samples(SampleRange(0, 16, 0, 16)), session.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 16, 16)
    assert_passes_match(session, film, PASSES)


def _traced_paths(prepared, seed, want=5, budget=3000):
    """Oracle-chosen pixels whose paths take each of the four dielectric
    events (transmit / reflect x glossy / singular), `want` of each."""
    rng = np.random.default_rng(seed)
    picked = {1 | 8: [], 1 | 16: [], 2 | 8: [], 2 | 16: []}
    for _ in range(budget):
        x, y, s = int(rng.integers(0, 96)), int(rng.integers(0, 72)), int(rng.integers(0, 16))
        st = scenes.render_settings(96, 72, max_bounces=8, window_x=x, window_y=y, window_width=1, window_height=1)
        t = OracleFilm(st).render_prepared(prepared, s, 1, 16, trace=(x, y, s))
        labels = {t.events[k].label for k in range(t.event_count)}
        for lab, lst in picked.items():
            if lab in labels and len(lst) < want:
                lst.append((x, y, s))
                break
        if all(len(v) >= want for v in picked.values()):
            break
    return picked


@pytest.mark.parametrize("seed", [1, 2])
def test_glass_traces_bit_exact(backend, seed):
    scene = scenes.glass_scene(seed=seed)
    compiled = backend.compile_scene(scene).scene
    prepared = OracleScene(scene.to_desc())
    picked = _traced_paths(prepared, seed)
    assert all(len(v) >= 3 for v in picked.values()), {k: len(v) for k, v in picked.items()}
    for paths in picked.values():
        for x, y, s in paths:
            st = scenes.render_settings(96, 72, max_bounces=8, window_x=x, window_y=y, window_width=1,
                                        window_height=1)
            session = backend.create_session(compiled, st)
            session.request_trace(x, y, s)
            assert session.render_samples(SampleRange(s, 1, 0, 16)), session.diagnostics
            ot = OracleFilm(st).render_prepared(prepared, s, 1, 16, trace=(x, y, s))
            assert_traces_match(session.read_trace(), ot, where=(x, y, s))


def test_glass_mixed_with_another_bsdf_is_refused(backend):
    """A glass closure beside another BSDF closure in one material fails at
    compile; refraction beside diffuse compiles (the scene's last
    material)."""
    scene = scenes.glass_scene(seed=1)
    assert backend.compile_scene(scene).ok()
    g = ShaderGraph()
    g.set_output(g.mix_shader(0.5, g.glass_bsdf(), g.diffuse_bsdf((0.5, 0.5, 0.5))))
    scene.materials[2] = scenes._materials([g])[0]
    assert not backend.compile_scene(scene).ok()


def test_glass_batched_equals_alone(backend):
    from psycles_b200.backend import BatchRenderer
    comp = backend.compile_scene(scenes.glass_scene(seed=3)).scene
    plain = backend.compile_scene(scenes.small_test_scene(seed=4)).scene
    work = [(comp, scenes.render_settings(64, 48, max_bounces=8, seed=k)) for k in range(2)]
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
