"""Glass and refraction closures on the host and in the oracle (not
gpu-marked).

The Glass and Refraction BSDF nodes (src/compiler/core_nodes.cpp:992-1019)
lower to closure instructions with the distribution in `a` and colour,
roughness and IOR inputs.  The oracle's dielectric closure
(src/luisa/microfacet_glass_component.cpp) passes a white-furnace check: a
closed sphere of clear glass under a uniform white background renders white
-- exactly for smooth glass and smooth refraction (delta lobes, Fresnel
split by probability) and for Beckmann at roughness 0.3 (its rational
Lambda is zero at these slopes, so every sample carries weight one), and
slightly darker for rough GGX glass (single-scattering microfacets lose
energy) -- and its traces reach transmitted glossy and singular bounces."""

import math

import numpy as np

from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.materials import ShaderGraph, compile_surface_program, glass_material
from psycles_b200.scenes import Camera, Instance, Scene, _materials, geodesic_sphere, look_at


def test_glass_lowering():
    prog, block = compile_surface_program(glass_material((0.9, 0.95, 1.0), 0.1, 1.45, "BECKMANN"))
    c = prog.closures[prog.root]
    assert c[0] == _abi.CLOSURE_GLASS and c[1] == _abi.GLOSSY_BECKMANN
    assert np.isclose(block.scalars[c[4]], 1.45) and np.isclose(block.scalars[c[5]], 0.1)
    g = ShaderGraph()
    g.set_output(g.refraction_bsdf((1.0, 1.0, 1.0), 0.0, 1.33))
    prog, block = compile_surface_program(g)
    c = prog.closures[prog.root]
    assert c[0] == _abi.CLOSURE_REFRACTION and c[1] == _abi.GLOSSY_GGX and np.isclose(block.scalars[c[4]], 1.33)


def _furnace(graph, bounces=48, spp=64):
    sc = Scene([geodesic_sphere(8)], [Instance(0, 0)], _materials([graph]), [],
               Camera(look_at((0, 0, 4.0), (0, 0, 0)), math.radians(30), math.radians(30), 0),
               background=(1.0, 1.0, 1.0))
    st = scenes.render_settings(48, 48, max_bounces=bounces, transparent_max_bounces=bounces,
                                transmission_bounces=bounces, glossy_bounces=bounces, min_bounces=bounces)
    film = OracleFilm(st)
    film.render(sc.to_desc(), 0, spp, spp)
    return film.resolve(_abi.PASS_COMBINED)[16:32, 16:32, :3]


def test_white_furnace():
    assert np.all(_furnace(glass_material((1, 1, 1), 0.0, 1.5)) == 1.0)
    assert np.all(_furnace(glass_material((1, 1, 1), 0.3, 1.5, "BECKMANN")) == 1.0)
    g = ShaderGraph()
    g.set_output(g.refraction_bsdf((1, 1, 1), 0.0, 1.5))
    assert np.all(_furnace(g) == 1.0)
    rough = _furnace(glass_material((1, 1, 1), 0.3, 1.5))
    assert 0.95 < rough.mean() < 1.0


def test_oracle_reaches_transmission():
    scene = scenes.glass_scene(seed=1)
    prepared = OracleScene(scene.to_desc())
    labels = set()
    rng = np.random.default_rng(0)
    for _ in range(200):
        x, y, s = int(rng.integers(0, 96)), int(rng.integers(0, 72)), int(rng.integers(0, 8))
        st = scenes.render_settings(96, 72, max_bounces=8, window_x=x, window_y=y, window_width=1, window_height=1)
        t = OracleFilm(st).render_prepared(prepared, s, 1, 8, trace=(x, y, s))
        labels |= {t.events[k].label for k in range(t.event_count)}
    assert {1 | 8, 1 | 16, 2 | 8, 2 | 16} <= labels, labels
