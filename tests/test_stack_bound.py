"""Traversal-stack bound on degenerate geometry (gpu-marked).

A binned-SAH build of a geometric chain of 4000 triangles (each one 0.4 %
further out and larger than the last, from 1 to about 1e7) peels a few
triangles off per level, and its 4-wide tree would need 57 stack entries
below the instance, over the device's 48.
Scene compile must detect that, rebuild the mesh with median splits and
report a bound within the stack; the render must then equal the oracle's
brute-force closest hits.  Thousands of coincident triangles, nested
triangles and coincident instances ride along (ties at equal distance
resolve to the greatest identity on both sides)."""

import math

import numpy as np
import pytest

from _parity import assert_passes_match
from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange
from psycles_b200.materials import diffuse_material

pytestmark = pytest.mark.gpu

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


def chain_mesh(n=4000, ratio=1.00404):
    pos = []
    x = 1.0
    for _ in range(n):
        s = 0.2 * x
        pos += [(x, 0.0, 0.0), (x + s, 0.0, 0.0), (x, s, s)]
        x *= ratio
    return scenes.Mesh(np.array(pos, np.float32), np.arange(3 * n, dtype=np.uint32).reshape(-1, 3))


def coincident_mesh(n=1000):
    tri = np.array([(-0.5, 0.0, 0.0), (0.5, 0.0, 0.0), (0.0, 0.8, 0.0)], np.float32)
    return scenes.Mesh(np.tile(tri, (n, 1)), np.arange(3 * n, dtype=np.uint32).reshape(-1, 3))


def nested_mesh(n=1000):
    pos = []
    for k in range(n):
        s = 0.2 + 0.001 * k
        pos += [(-s, -s, 0.001 * k), (s, -s, 0.001 * k), (0.0, s, 0.001 * k)]
    return scenes.Mesh(np.array(pos, np.float32), np.arange(3 * n, dtype=np.uint32).reshape(-1, 3))


def degenerate_scene():
    mats = scenes._materials([diffuse_material((0.7, 0.7, 0.7)), diffuse_material((0.8, 0.3, 0.2)),
                              diffuse_material((0.2, 0.5, 0.8))])
    meshes = [scenes.quad((-20, 0, -20), (-20, 0, 20), (20, 0, 20), (20, 0, -20)), chain_mesh(), coincident_mesh(),
              nested_mesh()]
    instances = [scenes.Instance(0, 0), scenes.Instance(1, 1, scenes.translate(-3.0, 0.2, -2.0)),
                 scenes.Instance(3, 2, scenes.translate(1.5, 1.0, 0.0))]
    # coincident instances of the coincident mesh: equal boxes in the TLAS
    for _ in range(12):
        instances.append(scenes.Instance(2, 2, scenes.translate(-1.0, 0.5, 1.0)))
    cam = scenes.Camera(scenes.look_at((0.0, 2.0, 7.0), (0.0, 0.8, 0.0)), math.radians(50.0), math.radians(50.0), 0)
    return scenes.Scene(meshes, instances, mats, [], cam, background=(0.8, 0.8, 0.8))


def test_degenerate_trees_fit_the_stack_and_match_brute_force(backend):
    scene = degenerate_scene()
    compiled = backend.compile_scene(scene)
    assert compiled.ok(), compiled.diagnostics
    stats = compiled.scene.build_stats()
    assert stats.stack_capacity == 48
    assert stats.median_rebuilds >= 1, "the chain's SAH tree should have needed a rebuild"
    assert 0 < stats.stack_need <= stats.stack_capacity, stats.stack_need
    st = scenes.render_settings(48, 32, max_bounces=3)
    session = backend.create_session(compiled.scene, st)
    assert session.render_samples(SampleRange(0, 2, 0, 2)), session.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 2, 2, brute_force=True)
    assert_passes_match(session, film, PASSES)


def test_regular_scene_needs_no_rebuild(backend):
    compiled = backend.compile_scene(scenes.procedural_scene(seed=0))
    assert compiled.ok(), compiled.diagnostics
    stats = compiled.scene.build_stats()
    assert stats.median_rebuilds == 0
    assert 0 < stats.stack_need <= stats.stack_capacity
    # BVH nodes, triangle records, vertices and indices of the 124,740 triangles of the eight meshes
    assert stats.upload_bytes > 20_000_000
