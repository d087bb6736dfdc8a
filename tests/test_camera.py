"""Camera projections of construct_camera_ray (src/luisa/path_tracer_camera.cpp:
51-246): perspective, orthographic and equirectangular panorama, with thin-lens
depth of field (round and bladed apertures, anamorphic ratio) for perspective
cameras.

CPU: geometric properties of the oracle's camera rays (orthographic rays are
parallel to the view axis; the panorama's centre ray is the view axis; rays of
one pixel through a thin lens meet near the focal plane).  GPU: the CUDA camera
rays and passes equal the oracle's (per-path trace bit for bit, passes within
relative RMSE 1e-3)."""

import dataclasses
import math

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange

PASSES = [_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT]


def camera_scene(**camera):
    scene = scenes.small_test_scene(seed=4)
    cam = dataclasses.replace(scene.camera, **camera)
    return dataclasses.replace(scene, camera=cam)


def oracle_ray(scene, settings, x, y, sample, total=4):
    film = OracleFilm(settings)
    t = film.render(scene.to_desc(), 0, total, total, threads=1, trace=(x, y, sample))
    assert t.valid == 1
    return np.array(t.ray_origin, np.float64), np.array(t.ray_direction, np.float64)


def view_axis(scene):
    m = np.asarray(scene.camera.transform, np.float64)
    fwd = -m[:3, 2]
    return fwd / np.linalg.norm(fwd)


CASES = {
    "orthographic": dict(projection=_abi.CAMERA_ORTHOGRAPHIC, orthographic_scale=6.0),
    "panorama": dict(projection=_abi.CAMERA_PANORAMA),
    "dof_round": dict(aperture_radius=0.15, focal_distance=6.0),
    "dof_blades": dict(aperture_radius=0.2, focal_distance=5.0, aperture_blades=6,
                       aperture_rotation=math.radians(20.0), aperture_ratio=0.7),
}


def test_orthographic_rays_are_parallel():
    scene = camera_scene(**CASES["orthographic"])
    st = scenes.render_settings(40, 30, max_bounces=2)
    axis = view_axis(scene)
    origins = []
    for x, y in [(0, 0), (39, 0), (20, 15), (5, 29)]:
        o, d = oracle_ray(scene, st, x, y, 1)
        assert np.allclose(d, axis, atol=1e-6)
        origins.append(o)
    # distinct pixels start at distinct points of the view plane
    assert len({tuple(np.round(o, 5)) for o in origins}) == 4


def test_panorama_centre_ray_is_the_view_axis():
    scene = camera_scene(**CASES["panorama"])
    st = scenes.render_settings(64, 32, max_bounces=2)
    # sample 0 uses the pixel centre; the film's centre lies between the four
    # central pixels
    dirs = [oracle_ray(scene, st, x, y, 0)[1] for x, y in [(31, 15), (32, 15), (31, 16), (32, 16)]]
    mean = np.mean(dirs, axis=0)
    assert np.allclose(mean / np.linalg.norm(mean), view_axis(scene), atol=2e-3)
    # the left edge looks backwards
    _, d = oracle_ray(scene, st, 0, 16, 0)
    assert float(np.dot(d, view_axis(scene))) < -0.99


def test_thin_lens_rays_meet_on_the_focal_plane():
    scene = camera_scene(**CASES["dof_blades"])
    st = scenes.render_settings(48, 36, max_bounces=2)
    axis = view_axis(scene)
    eye = np.asarray(scene.camera.transform, np.float64)[:3, 3]
    points, origins = [], []
    for s in range(1, 4):
        o, d = oracle_ray(scene, st, 20, 17, s, total=8)
        # intersect with the plane at focal_distance along the view axis
        t = float(np.dot(eye + axis * 5.0 - o, axis)) / float(np.dot(d, axis))
        points.append(o + d * t)
        origins.append(o)
    # the filter jitter differs per sample, so the focus points differ by at
    # most a pixel footprint; the lens origins differ by up to the aperture
    spread_focus = np.max(np.linalg.norm(np.array(points) - points[0], axis=1))
    spread_lens = np.max(np.linalg.norm(np.array(origins) - origins[0], axis=1))
    assert spread_lens > 1e-3
    assert spread_focus < 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_camera_rays_and_passes_match_oracle(backend, case):
    scene = camera_scene(**CASES[case])
    st = scenes.render_settings(64, 48, max_bounces=4)
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    for px, py, s in [(5, 7, 0), (40, 30, 2), (63, 47, 3)]:
        sess = backend.create_session(comp.scene, st)
        sess.request_trace(px, py, s)
        assert sess.render_samples(SampleRange(0, 4, 0, 4)), sess.diagnostics
        gt = sess.read_trace()
        film = OracleFilm(st)
        ot = film.render(scene.to_desc(), 0, 4, 4, threads=0, trace=(px, py, s))
        assert gt.valid == 1 and ot.valid == 1
        for f in ("ray_origin", "ray_direction"):
            a, b = np.array(getattr(gt, f), np.float32), np.array(getattr(ot, f), np.float32)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (case, f, a, b)
        assert gt.event_count == ot.event_count
    for kind in PASSES:
        got, ref = sess.read_pass(kind), film.resolve(kind)
        rms = float(np.sqrt(np.mean(np.square(ref.astype(np.float64)))))
        e = float(np.sqrt(np.mean(np.square(got.astype(np.float64) - ref)))) / max(rms, 1e-12)
        assert e <= 1e-3, (case, kind, e)


@pytest.mark.gpu
def test_unknown_camera_projection_is_rejected(backend):
    scene = camera_scene(projection=7)
    comp = backend.compile_scene(scene)
    assert comp.ok()
    assert backend.create_session(comp.scene, scenes.render_settings(16, 16)) is None
