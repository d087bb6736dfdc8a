"""Glossy closures on the host and in the oracle (not gpu-marked).

The Glossy BSDF node (src/compiler/core_nodes.cpp:980-990) lowers to a
closure instruction with the distribution in `a`, its colour and roughness
as inputs; the Distribution property is structural (a parameter-only edit
cannot switch it).  The oracle renders the glossy scene with glossy
(reflect | glossy) and singular (reflect | singular) bounces, and its
visible-normal samplers are pinned in tests/test_oracle_golden.py."""

import numpy as np
import pytest

from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.materials import MaterialLibrary, MaterialUpdateKind, ShaderGraph, ShaderGraphError, \
    compile_surface_program, glossy_material


def test_glossy_lowering():
    g = ShaderGraph()
    r = g.math("multiply", g.value(0.4), 0.5)
    g.set_output(g.glossy_bsdf((0.9, 0.8, 0.7), r, "BECKMANN"))
    prog, block = compile_surface_program(g)
    c = prog.closures[prog.root]
    assert c[0] == _abi.CLOSURE_GLOSSY and c[1] == _abi.GLOSSY_BECKMANN
    assert not c[3] & _abi.INPUT_VALUE and c[5] & _abi.INPUT_VALUE  # unlinked colour, linked roughness
    assert np.allclose(block.vectors[c[3]], (0.9, 0.8, 0.7))
    prog2, _ = compile_surface_program(glossy_material((0.5, 0.5, 0.5)))
    c2 = prog2.closures[prog2.root]
    assert c2[1] == _abi.GLOSSY_GGX and not c2[5] & _abi.INPUT_VALUE
    with pytest.raises(ShaderGraphError):
        ShaderGraph().glossy_bsdf((1, 1, 1), 0.2, "ASHIKHMIN_SHIRLEY")


def test_distribution_is_structural():
    lib = MaterialLibrary()
    lib.update({"m": glossy_material((0.5, 0.5, 0.5), 0.2, "GGX")})
    assert lib.update({"m": glossy_material((0.9, 0.5, 0.5), 0.4, "GGX")})["m"] == MaterialUpdateKind.PARAMETERS_REBOUND
    assert lib.update({"m": glossy_material((0.9, 0.5, 0.5), 0.4, "BECKMANN")})["m"] == \
        MaterialUpdateKind.PROGRAM_RECOMPILED


def test_oracle_renders_glossy_and_singular_bounces():
    scene = scenes.glossy_scene(seed=1)
    prepared = OracleScene(scene.to_desc())
    labels = set()
    rng = np.random.default_rng(0)
    for _ in range(40):
        x, y, s = int(rng.integers(0, 96)), int(rng.integers(0, 72)), int(rng.integers(0, 16))
        st = scenes.render_settings(96, 72, max_bounces=6, window_x=x, window_y=y, window_width=1, window_height=1)
        t = OracleFilm(st).render_prepared(prepared, s, 1, 16, trace=(x, y, s))
        labels |= {t.events[k].label for k in range(t.event_count)}
    assert 2 | 8 in labels and 2 | 16 in labels, labels
    st = scenes.render_settings(48, 36, max_bounces=6)
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 4, 4)
    img = film.resolve(_abi.PASS_COMBINED)
    assert np.isfinite(img).all() and img[..., :3].mean() > 0.0
