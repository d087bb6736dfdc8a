"""Forward lamp events: camera and BSDF rays that reach an area lamp or a
finite-radius point / spot disk before the mesh event add its emission with
the forward MIS weight, count a transparent bounce and continue
(src/luisa/path_kernel_closest_event.cpp:56-230,
src/luisa/path_kernel_forward_light.cpp:14-118); NEE of those lamps takes the
complementary weight (src/luisa/path_kernel_nee_analytic.cpp:286-292).

CPU: the oracle's MIS and NEE-only estimators agree (both unbiased), and a
camera ray that meets a lamp records exactly its radiance.  GPU: the CUDA
path against the oracle on a lamp-heavy scene (passes and per-path traces)."""

import math

import numpy as np
import pytest

from oracle.oracle import OracleFilm
from psycles_b200 import _abi, scenes
from psycles_b200.backend import SampleRange


def _mean(scene, mode, spp, size=(40, 30), **kw):
    st = scenes.render_settings(size[0], size[1], max_bounces=3, direct_light_sampling=mode, **kw)
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, spp, spp, threads=0)
    return film.resolve(_abi.PASS_COMBINED)[..., :3]


def test_mis_and_nee_estimators_agree():
    scene = scenes.lamp_scene()
    mis = _mean(scene, _abi.DIRECT_MIS, 192)
    nee = _mean(scene, _abi.DIRECT_NEE, 192)
    assert abs(mis.mean() - nee.mean()) <= 0.015 * nee.mean(), (mis.mean(), nee.mean())


def test_forward_lamp_hits_change_the_mis_image():
    """Without the forward events the MIS estimator would lose the BSDF share
    of every finite lamp; with them it matches NEE (above).  Here the lamps
    are all excluded from MIS, so NEE carries them with weight one and the
    two modes give the same image sample for sample."""
    scene = scenes.lamp_scene()
    for light in scene.lights:
        light.use_mis = False
    mis = _mean(scene, _abi.DIRECT_MIS, 16, size=(24, 18))
    nee = _mean(scene, _abi.DIRECT_NEE, 16, size=(24, 18))
    # camera-visible lamps still appear; indirect lamp light is NEE-only in both
    assert abs(mis.mean() - nee.mean()) <= 0.02 * nee.mean()


def test_camera_ray_records_lamp_radiance_exactly():
    """A primary ray through a rectangle lamp adds color * power / (pi area)
    (normalised power, MIS weight one at depth zero) at its first event."""
    scene = scenes.lamp_scene()
    scene.background = (0.0, 0.0, 0.0)
    lamp = scene.lights[0]  # rectangle facing the camera, nothing in front
    expected = np.array(lamp.color, np.float32) * np.float32(
        np.float32(lamp.power) * np.float32(np.float32(1.0 / math.pi) * np.float32(1.0 / (lamp.size_u * lamp.size_v))))
    width, height = 64, 48
    found = 0
    for y in range(14, 26, 2):
        for x in range(10, 28, 2):
            st = scenes.render_settings(width, height, max_bounces=3, window_x=x, window_y=y, window_width=1,
                                        window_height=1)
            film = OracleFilm(st)
            t = film.render(scene.to_desc(), 0, 1, 1, threads=1, trace=(x, y, 0))
            if t.valid and t.event_count > 0:
                e = np.array(t.events[0].emission[:], np.float32)
                if np.allclose(e, expected, rtol=1e-6, atol=0):
                    found += 1
    assert found >= 3, found


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
def test_lamp_scene_passes_match_oracle(backend):
    scene = scenes.lamp_scene()
    st = scenes.render_settings(96, 72, max_bounces=5)
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    sess = backend.create_session(comp.scene, st)
    assert sess.render_samples(SampleRange(0, 8, 0, 8)), sess.diagnostics
    film = OracleFilm(st)
    film.render(scene.to_desc(), 0, 8, 8, threads=0)
    for kind in (_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT):
        got, ref = sess.read_pass(kind).astype(np.float64), film.resolve(kind).astype(np.float64)
        rms = float(np.sqrt(np.mean(np.square(ref))))
        e = float(np.sqrt(np.mean(np.square(got - ref)))) / max(rms, 1e-12)
        assert e <= 1e-3, (kind, e)


@pytest.mark.gpu
@pytest.mark.parametrize("tree", [0, 1])
def test_lamp_scene_traces_bit_exact(backend, tree):
    scene = scenes.lamp_scene()
    st = scenes.render_settings(64, 48, max_bounces=5, use_light_tree=tree, transparent_max_bounces=3)
    comp = backend.compile_scene(scene)
    assert comp.ok(), comp.diagnostics
    for x, y, s in [(40, 20, 0), (18, 14, 1), (33, 30, 2), (50, 12, 3), (10, 40, 0)]:
        sess = backend.create_session(comp.scene, st)
        sess.request_trace(x, y, s)
        assert sess.render_samples(SampleRange(0, 4, 0, 4)), sess.diagnostics
        gt = sess.read_trace()
        ot = OracleFilm(st).render(scene.to_desc(), 0, 4, 4, threads=0, trace=(x, y, s))
        assert gt.valid == 1 and ot.valid == 1
        assert gt.event_count == ot.event_count
        for k in range(gt.event_count):
            a, b = gt.events[k], ot.events[k]
            for f in ("transparent_bounce", "flag", "light_kind", "light_index", "terminated", "hit_object"):
                assert getattr(a, f) == getattr(b, f), (x, y, s, k, f)
            for f in ("emission", "nee", "throughput"):
                u, v = np.array(getattr(a, f)), np.array(getattr(b, f))
                assert np.all(np.abs(u - v) <= 1e-6 + 2e-6 * np.maximum(np.abs(u), np.abs(v))), (x, y, s, k, f, u, v)
        assert np.allclose(np.array(gt.radiance), np.array(ot.radiance), rtol=2e-6, atol=1e-6)
