"""MULTI_GGX glossy closures: GGX with Cycles' tabulated multiple-scattering
energy preservation (src/luisa/graph_surface_scattering.cpp:170-198,
src/luisa/graph_surface_physical_closures.cpp:360-392).  The weight takes
the darkening (1 + Fms (1 - E) / E) E and every evaluation (the singular
mirror's too) the scale 1 / E, with E and its average read from Cycles' GGX
albedo tables, which the scene carries: the tests take the reference's own
tables from oracle/_ref (src/luisa/cycles_shader_tables_4_5_10.inl).

Not gpu-marked: energy preservation brightens a rough glossy scene in the
oracle and leaves a mirror's weight as it is.  gpu-marked: the CUDA passes
match the oracle's, and a scene without the tables is refused."""

import ctypes
import pathlib

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from psycles_b200.materials import emission_material, glossy_material

ROOT = pathlib.Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref" / "libpsycles_ref.so"

pytestmark = pytest.mark.skipif(not REF.exists(), reason="reference shim not built (make -C oracle ref)")

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


def ggx_tables():
    lib = ctypes.CDLL(str(REF))
    e = np.zeros(1024, np.float32)
    eavg = np.zeros(32, np.float32)
    lib.ref_ggx_tables(e.ctypes.data_as(ctypes.c_void_p), eavg.ctypes.data_as(ctypes.c_void_p))
    return e, eavg


def multi_ggx_scene(distribution="MULTI_GGX", seed=1):
    """The glossy test scene with its glossy materials at roughness 0 (a
    mirror), 0.3 and 0.6 in the given distribution."""
    scene = scenes.glossy_scene(seed=seed)
    graphs = [glossy_material((0.8, 0.8, 0.8), 0.6, distribution), emission_material((1.0, 0.9, 0.8), 6.0),
              glossy_material((0.9, 0.8, 0.6), 0.0, distribution), glossy_material((0.6, 0.8, 0.9), 0.3, distribution),
              glossy_material((0.9, 0.9, 0.9), 0.6, distribution), glossy_material((0.7, 0.9, 0.7), 0.45, distribution),
              glossy_material((0.5, 0.5, 0.9), 0.2, distribution), glossy_material((0.9, 0.5, 0.5), 0.8, distribution)]
    scene.materials = scenes._materials(graphs)
    scene.ggx_tables = ggx_tables()
    return scene


def test_reference_tables_are_albedos():
    e, eavg = ggx_tables()
    assert np.all((e > 0.0) & (e <= 1.0)) and np.all((eavg > 0.0) & (eavg <= 1.0))
    # a smooth GGX surface loses no energy; a rough one loses some
    assert e.reshape(32, 32)[:, 0].min() > 0.97 and eavg[-1] < eavg[0]


def test_energy_preservation_brightens_rough_glossy():
    st = scenes.render_settings(64, 48, max_bounces=4)
    means = {}
    for dist in ("GGX", "MULTI_GGX"):
        film = OracleFilm(st)
        film.render(multi_ggx_scene(dist).to_desc(), 0, 8, 8)
        img = film.resolve(_abi.PASS_COMBINED)
        assert np.all(np.isfinite(img))
        means[dist] = float(img[..., :3].mean())
    assert means["MULTI_GGX"] > means["GGX"] * 1.005, means


@pytest.mark.gpu
def test_multi_ggx_matches_oracle(backend):
    from _parity import assert_passes_match
    from psycles_b200.backend import SampleRange
    scene = multi_ggx_scene()
    st = scenes.render_settings(96, 72, max_bounces=6)
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    session = backend.create_session(compiled.scene, st)
    assert session.render_samples(SampleRange(0, 16, 0, 16)), session.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 16, 16)
    assert_passes_match(session, film, PASSES)


@pytest.mark.gpu
def test_multi_ggx_without_tables_is_refused(backend):
    scene = multi_ggx_scene()
    scene.ggx_tables = None
    compiled = backend.compile_scene(scene)
    assert not compiled.ok()
    assert any("GGX albedo tables" in str(d) for d in compiled.diagnostics), compiled.diagnostics
