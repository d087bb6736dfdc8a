"""CUDA kernels against the CPU oracle on the benchmark workloads at their own
sizes, through the C ABI (gpu-marked).

- Closed box: 256x256, 16 spp, 4 bounces, the whole frame.
- Procedural scene (997,920 instanced triangles, 64 instances of 8 meshes of
  2k-38.7k triangles, 32 random closure graphs, 24 lamps): the 1920x1080
  frame's centre band of 16 full rows at all 64 spp, 8 bounces; plus
  per-path traces of ten (pixel, sample) pairs whose paths cross
  transparent and mixed materials, hit instances of the largest mesh (the
  deepest BLAS) and take NEE samples.
- Many-light scene (10,000 emissive triangles, light tree): the 1280x720
  frame's centre band of 16 rows at all 32 spp, 6 bounces; plus traces.

Bar: passes within relative RMSE 1e-3 of the oracle with at most 1 % of
pixels differing in any bit; traces bit-exact on discrete and random
fields and within 1e-6 + 2e-6 * max(|a|, |b|) on continuous ones."""

import pytest

from _parity import assert_passes_match, assert_traces_match, trace_tags
from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_DENOISING_NORMAL,
          _abi.PASS_DENOISING_ALBEDO, _abi.PASS_SAMPLE_COUNT]

# (x, y, sample) of the procedural frame: paths of 5-8 events over
# transparent and mix materials and instances of the 38,720-triangle mesh
PROCEDURAL_TRACES = [(1208, 476, 32), (1271, 575, 8), (1844, 615, 17), (1206, 524, 50), (1397, 462, 5),
                     (1395, 548, 39), (116, 406, 62), (1576, 141, 51), (105, 27, 46), (1231, 630, 36)]
# (x, y, sample) of the many-light frame: NEE through the light tree
MANY_LIGHT_TRACES = [(821, 420, 18), (1026, 533, 28), (963, 535, 25), (396, 516, 4), (42, 710, 16),
                     (1209, 450, 21)]


def band_settings(width, height, bounces, rows, light_tree=0):
    return scenes.render_settings(width, height, max_bounces=bounces, window_y=(height - rows) // 2,
                                  window_height=rows, use_light_tree=light_tree)


def compare_band(backend, scene, settings, spp):
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    session = backend.create_session(compiled.scene, settings)
    assert session.render_samples(SampleRange(0, spp, 0, spp)), session.diagnostics
    prepared = OracleScene(scene.to_desc())
    film = OracleFilm(settings)
    film.render_prepared(prepared, 0, spp, spp)
    errors = assert_passes_match(session, film, PASSES)
    return compiled.scene, prepared, errors


def compare_traces(backend, compiled, prepared, scene, width, height, bounces, spp, pixels, light_tree=0):
    tags = set()
    for x, y, s in pixels:
        st = scenes.render_settings(width, height, max_bounces=bounces, window_x=x, window_y=y, window_width=1,
                                    window_height=1, use_light_tree=light_tree)
        session = backend.create_session(compiled, st)
        session.request_trace(x, y, s)
        assert session.render_samples(SampleRange(s, 1, 0, spp)), session.diagnostics
        gt = session.read_trace()
        ot = OracleFilm(st).render_prepared(prepared, s, 1, spp, trace=(x, y, s))
        assert_traces_match(gt, ot, where=(x, y, s))
        tags |= trace_tags(ot, scene)
        session.close()
    return tags


def test_closed_box_full_frame(backend):
    scene = scenes.cornell_box()
    st = scenes.render_settings(256, 256, max_bounces=4)
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    session = backend.create_session(compiled.scene, st)
    assert session.render_samples(SampleRange(0, 16, 0, 16)), session.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 16, 16)
    assert_passes_match(session, film, PASSES)


def test_procedural_band_and_traces(backend):
    scene = scenes.procedural_scene(seed=0)
    assert scene.instanced_triangles == 997920
    st = band_settings(1920, 1080, 8, 16)
    compiled, prepared, _ = compare_band(backend, scene, st, 64)
    stats = compiled.build_stats()
    assert 0 < stats.stack_need <= stats.stack_capacity
    tags = compare_traces(backend, compiled, prepared, scene, 1920, 1080, 8, 64, PROCEDURAL_TRACES)
    assert {"transparent", "mix", "deep", "nee"} <= tags, tags


def test_many_light_band_and_traces(backend):
    scene = scenes.many_light_scene(seed=0)
    st = band_settings(1280, 720, 6, 16, light_tree=1)
    compiled, prepared, _ = compare_band(backend, scene, st, 32)
    tags = compare_traces(backend, compiled, prepared, scene, 1280, 720, 6, 32, MANY_LIGHT_TRACES, light_tree=1)
    assert "nee" in tags, tags
