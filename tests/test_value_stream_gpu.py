"""SurfaceProgram value streams on the device against the oracle (gpu-marked).

Materials whose closure inputs are linked to value nodes (RGB and Value
nodes through colour blends, float math, conversions, separate / combine
RGB into rough diffuse colours, mix factors and emission strengths) render
through the device interpreter of the value stream; passes and per-path
traces must match the oracle, with the flat distribution and with the light
tree (whose emission estimates read only unlinked literals).  Malformed
streams are rejected at compile time."""

import ctypes

import numpy as np
import pytest

from _parity import assert_passes_match, assert_traces_match, trace_tags
from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


@pytest.mark.parametrize("light_tree", [0, 1])
def test_value_graph_scene_matches_oracle(backend, light_tree):
    scene = scenes.value_graph_scene(seed=1)
    st = scenes.render_settings(96, 72, max_bounces=6, use_light_tree=light_tree)
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    session = backend.create_session(compiled.scene, st)
    assert session.render_samples(SampleRange(0, 8, 0, 8)), session.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 8, 8)
    assert_passes_match(session, film, PASSES)


def test_value_graph_traces_bit_exact(backend):
    scene = scenes.value_graph_scene(seed=1)
    compiled = backend.compile_scene(scene).scene
    prepared = OracleScene(scene.to_desc())
    for x, y, s in [(40, 30, 1), (20, 50, 3), (70, 20, 0), (55, 40, 5)]:
        st = scenes.render_settings(96, 72, max_bounces=6, window_x=x, window_y=y, window_width=1, window_height=1)
        session = backend.create_session(compiled, st)
        session.request_trace(x, y, s)
        assert session.render_samples(SampleRange(s, 1, 0, 8)), session.diagnostics
        ot = OracleFilm(st).render_prepared(prepared, s, 1, 8, trace=(x, y, s))
        assert_traces_match(session.read_trace(), ot, where=(x, y, s))


def _scene_with_program(closures, values, scalars=(0.5,), vectors=((0.5, 0.5, 0.5),)):
    sc = scenes.cornell_box()
    m = sc.materials[0]
    prog = m.program
    prog.closures = np.array(closures, np.uint32).reshape(-1, 6)
    prog.values = np.array(values, np.uint32).reshape(-1, 8)
    prog.root = len(closures) - 1
    m.parameters.scalars = np.array(scalars, np.float32)
    m.parameters.vectors = np.array(vectors, np.float32).reshape(-1, 3)
    return sc


def test_malformed_value_streams_are_rejected(backend):
    V, N = _abi.INPUT_VALUE, _abi.INPUT_NONE
    diffuse = lambda color, rough=N: [(_abi.CLOSURE_DIFFUSE, 0, 0, color, N, rough)]
    cases = {
        # an operand that names a later instruction
        "forward": (diffuse(V | 0), [(_abi.VALUE_SCALAR_TO_COLOR, 1, 0, 1, 0, 0, 0, 0),
                                     (_abi.VALUE_PARAMETER, 0, 0, 0, 0, 0, 0, 0)]),
        # a vector operand where a scalar is required
        "type": (diffuse(V | 1), [(_abi.VALUE_PARAMETER, 1, 0, 0, 0, 0, 0, 0),
                                  (_abi.VALUE_SCALAR_TO_COLOR, 1, 0, 0, 0, 0, 0, 0)]),
        # a parameter slot outside the block
        "slot": (diffuse(V | 0), [(_abi.VALUE_PARAMETER, 1, 7, 0, 0, 0, 0, 0)]),
        # an operation outside the supported set (texture lookup)
        "op": (diffuse(V | 0), [(71, 1, 0, 0, 0, 0, 0, 0)]),
        # a colour input fed by a scalar value
        "input": (diffuse(V | 0), [(_abi.VALUE_PARAMETER, 0, 0, 0, 0, 0, 0, 0)]),
        # a blend mode outside the supported set (hue)
        "blend": (diffuse(V | 2), [(_abi.VALUE_PARAMETER, 1, 0, 0, 0, 0, 0, 0),
                                   (_abi.VALUE_PARAMETER, 0, 0, 0, 0, 0, 0, 0),
                                   (_abi.VALUE_MIX, 1, 0, 0, 0, 1, 15, 1)]),
    }
    for name, (closures, values) in cases.items():
        comp = backend.compile_scene(_scene_with_program(closures, values))
        assert not comp.ok(), name
    # a well-formed stream of the same shape compiles
    ok = _scene_with_program(diffuse(V | 1, V | 2), [(_abi.VALUE_PARAMETER, 0, 0, 0, 0, 0, 0, 0),
                                                       (_abi.VALUE_SCALAR_TO_COLOR, 1, 0, 0, 0, 0, 0, 0),
                                                       (_abi.VALUE_CLAMP01, 0, 0, 0, 0, 0, 0, 0)])
    assert backend.compile_scene(ok).ok()


def test_rebind_of_a_linked_value_equals_recompile(backend):
    scene = scenes.value_graph_scene(seed=2)
    st = scenes.render_settings(48, 36, max_bounces=4)
    k = 2
    comp = backend.compile_scene(scene).scene
    sc = scene.materials[k].parameters.scalars.copy()
    vc = scene.materials[k].parameters.vectors[::-1].copy()
    comp.rebind_parameters(k, sc * np.float32(0.5), vc)
    a = backend.create_session(comp, st)
    assert a.render_samples(SampleRange(0, 4, 0, 4))
    scene.materials[k].parameters.scalars[:] = sc * np.float32(0.5)
    scene.materials[k].parameters.vectors[:] = vc
    b = backend.create_session(backend.compile_scene(scene).scene, st)
    assert b.render_samples(SampleRange(0, 4, 0, 4))
    assert np.array_equal(a.read_pass(_abi.PASS_COMBINED), b.read_pass(_abi.PASS_COMBINED))
