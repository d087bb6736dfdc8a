"""SurfaceProgram value streams and rough diffuse on the CPU (not gpu-marked).

- Oren-Nayar diffuse_intensity (src/luisa/graph_surface_scattering.cpp:
  463-506) in the oracle: Lambert below roughness 1e-5, reciprocal in its two
  directions, and energy-preserving for a white albedo (Cycles' multiple-
  scattering term keeps the directional albedo at one for every roughness).
- The host lowering of graphs with value nodes: literal edits keep the
  structure signature (parameters_rebound), link edits change it.
- The oracle's value-stream interpreter against exact identities: an RGB
  node linked to a diffuse colour, a colour mix at factor 0 and a product
  with one render exactly what the literal colour renders.
"""

import ctypes

import numpy as np

from oracle import oracle
from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from psycles_b200.materials import (MaterialLibrary, MaterialUpdateKind, ShaderGraph, compile_surface_program,
                                    diffuse_material, value_graph_material)


def intensity(normal, color, roughness, incoming, outgoing):
    lib = oracle.load()
    out = np.zeros(3, np.float32)
    args = [np.ascontiguousarray(v, np.float32) for v in (normal, color, incoming, outgoing)]
    lib.oracle_diffuse_intensity(args[0].ctypes.data, args[1].ctypes.data, ctypes.c_float(roughness),
                                 args[2].ctypes.data, args[3].ctypes.data, out.ctypes.data)
    return out


def hemisphere(n_theta=48, n_phi=96):
    """Midpoint cosine-weighted quadrature of the upper hemisphere: unit
    directions and weights w with sum(w * g / cos) = integral of g."""
    u = (np.arange(n_theta) + 0.5) / n_theta
    v = (np.arange(n_phi) + 0.5) / n_phi
    uu, vv = np.meshgrid(u, v, indexing="ij")
    ct = np.sqrt(uu).reshape(-1)
    st = np.sqrt(1.0 - ct * ct)
    ph = 2.0 * np.pi * vv.reshape(-1)
    dirs = np.stack([st * np.cos(ph), st * np.sin(ph), ct], 1)
    return dirs, ct / np.pi


def test_rough_diffuse_is_lambert_below_cutoff():
    n, c = (0.0, 0.0, 1.0), (0.5, 0.6, 0.7)
    wi = np.array([0.3, 0.1, 0.95]) / np.linalg.norm([0.3, 0.1, 0.95])
    wo = np.array([-0.5, 0.2, 0.8]) / np.linalg.norm([-0.5, 0.2, 0.8])
    lam = intensity(n, c, 0.0, wi, wo)
    assert np.allclose(lam, wo[2] / np.pi, rtol=1e-6)
    assert np.array_equal(intensity(n, c, 0.9e-5, wi, wo), lam)
    assert not np.array_equal(intensity(n, c, 0.5, wi, wo), lam)


def test_rough_diffuse_is_reciprocal():
    rng = np.random.default_rng(4)
    for _ in range(50):
        a, b = rng.normal(size=3), rng.normal(size=3)
        a[2], b[2] = abs(a[2]) + 0.05, abs(b[2]) + 0.05
        a, b = a / np.linalg.norm(a), b / np.linalg.norm(b)
        c = rng.uniform(0.0, 1.0, 3)
        r = float(rng.uniform(0.0, 1.0))
        # f = intensity / cos(outgoing); reciprocity of the BRDF
        fab = intensity((0, 0, 1), c, r, a, b) / np.float32(b[2])
        fba = intensity((0, 0, 1), c, r, b, a) / np.float32(a[2])
        assert np.allclose(fab, fba, rtol=2e-5, atol=1e-7), (r, fab, fba)


def test_rough_diffuse_preserves_white_energy():
    dirs, pdf = hemisphere()
    for r in (0.2, 0.5, 1.0):
        for mu in (0.15, 0.5, 0.95):
            wi = np.array([np.sqrt(1.0 - mu * mu), 0.0, mu])
            e = sum(intensity((0, 0, 1), (1, 1, 1), r, wi, d)[0] / p for d, p in zip(dirs, pdf)) / len(dirs)
            assert 0.985 <= e <= 1.01, (r, mu, e)


def test_literal_edits_rebind_and_link_edits_recompile():
    rng = np.random.default_rng(2)
    g1 = value_graph_material(np.random.default_rng(7))
    g2 = value_graph_material(np.random.default_rng(7))
    # change one literal of a value node: same structure
    node = next(i for i, n in enumerate(g2.nodes) if n.type.value == "psycles.constant.color")
    g2.nodes[node].sockets["Color"] = tuple(float(v) for v in rng.uniform(0, 1, 3))
    assert g1.structure_signature() == g2.structure_signature()
    assert g1.parameter_signature() != g2.parameter_signature()
    lib = MaterialLibrary()
    assert lib.update({"m": g1})["m"] == MaterialUpdateKind.ADDED
    assert lib.update({"m": g2})["m"] == MaterialUpdateKind.PARAMETERS_REBOUND
    p1, _ = compile_surface_program(g1)
    p2, b2 = compile_surface_program(g2)
    assert np.array_equal(p1.values, p2.values) and np.array_equal(p1.closures, p2.closures)
    assert lib.materials["m"].parameters.vectors.tolist() == b2.vectors.tolist()
    # a link instead of a literal: a new structure
    g3 = value_graph_material(np.random.default_rng(7))
    d = next(i for i, n in enumerate(g3.nodes) if n.type.value == "psycles.closure.diffuse")
    g3.nodes[d].sockets["Roughness"] = g3.value(0.25)
    assert g3.structure_signature() != g1.structure_signature()
    assert lib.update({"m": g3})["m"] == MaterialUpdateKind.PROGRAM_RECOMPILED


def test_value_program_encoding():
    g = ShaderGraph()
    c = g.mix_color(0.25, g.rgb((0.2, 0.4, 0.6)), g.rgb((0.9, 0.1, 0.3)), blend="MULTIPLY")
    g.set_output(g.diffuse_bsdf(c, 0.3))
    prog, block = compile_surface_program(g)
    root = [int(v) for v in prog.closures[prog.root]]
    assert root[0] == _abi.CLOSURE_DIFFUSE
    assert root[3] & _abi.INPUT_VALUE and not root[5] & _abi.INPUT_VALUE  # linked colour, literal roughness
    color_id = root[3] & 0x7FFFFFFF
    mix = [int(v) for v in prog.values[color_id]]
    assert mix[0] == _abi.VALUE_MIX and mix[1] == _abi.VALUE_TYPE_VECTOR and mix[6] == _abi.BLEND_MULTIPLY
    for operand in mix[3:6]:
        assert operand < color_id  # topological order
    assert block.scalars[root[5]] == np.float32(0.3)


def _wall_scene(graph) -> scenes.Scene:
    sc = scenes.cornell_box()
    sc.materials = scenes._materials([graph] + [m.graph for m in sc.materials[1:]])
    return sc


def _render(scene):
    st = scenes.render_settings(32, 32, max_bounces=4)
    f = OracleFilm(st)
    f.render(scene.to_desc(), 0, 4, 4)
    return f.combined


def test_oracle_value_stream_identities():
    color = (0.73, 0.41, 0.29)
    literal = _render(_wall_scene(diffuse_material(color, 0.4)))
    g = ShaderGraph()
    g.set_output(g.diffuse_bsdf(g.rgb(color), g.value(0.4)))
    assert np.array_equal(_render(_wall_scene(g)), literal)
    g = ShaderGraph()
    g.set_output(g.diffuse_bsdf(g.mix_color(0.0, g.rgb(color), g.rgb((0.1, 0.9, 0.5))),
                                g.math("multiply", 0.4, 1.0)))
    assert np.array_equal(_render(_wall_scene(g)), literal)
    g = ShaderGraph()
    r, gg, b = g.separate_color(g.rgb(color))
    g.set_output(g.diffuse_bsdf(g.combine_color(r, gg, b), 0.4))
    assert np.array_equal(_render(_wall_scene(g)), literal)
    # and the roughness matters
    assert not np.array_equal(_render(_wall_scene(diffuse_material(color, 0.0))), literal)


def test_value_graph_scene_renders_finite():
    sc = scenes.value_graph_scene(seed=1)
    assert any(m.program.values.shape[0] > 4 for m in sc.materials)
    st = scenes.render_settings(40, 30, max_bounces=5)
    f = OracleFilm(st)
    f.render(sc.to_desc(), 0, 4, 4)
    img = f.resolve(_abi.PASS_COMBINED)
    assert np.all(np.isfinite(img)) and img[..., :3].mean() > 0.0
