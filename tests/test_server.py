"""Render server (psy_server_*): request loop, HBM-budget admission,
continuous batching, ordered parameter edits, cancellation and latency
statistics.  Every job's passes must equal a session rendering the same
settings and samples alone, bit for bit, whatever else shared its
wavefronts (gpu-marked)."""

import math
import time

import numpy as np
import pytest

from psycles_b200 import _abi, scenes
from psycles_b200.backend import RenderServer, SampleRange

pytestmark = pytest.mark.gpu

PASSES = (_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT)


def _alone(backend, compiled, settings, spp, camera=None):
    s = backend.create_session(compiled, settings)
    if camera is not None:
        s.set_camera(camera)
    assert s.render_samples(SampleRange(0, spp, 0, spp)), s.diagnostics
    return {k: s.read_pass(k) for k in PASSES}


def _from_server(server, job, w, h):
    assert server.wait(job, 120000) == _abi.PSY_OK
    return {k: server.read_pass(job, k, w, h) for k in PASSES}


def _same(a, b):
    return all(np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)) for k in PASSES)


def _cam(rng):
    eye = (float(rng.uniform(-3, 3)), float(rng.uniform(1.5, 4)), float(rng.uniform(6, 9)))
    return scenes.Camera(scenes.look_at(eye, (0.0, 1.0, 0.0)), math.radians(40), math.radians(40), 0)


def test_jobs_equal_sessions_alone_in_a_mix(backend):
    rng = np.random.default_rng(5)
    scs = [backend.compile_scene(scenes.small_test_scene(seed=1)).scene,
           backend.compile_scene(scenes.lamp_scene(seed=2)).scene]
    jobs = []
    for k in range(8):
        w, h = [(48, 32), (64, 64), (96, 72), (20, 16)][k % 4]
        spp = int(rng.integers(1, 9))
        cam = _cam(rng) if k % 3 == 0 else None
        jobs.append((k % 2, scenes.render_settings(w, h, max_bounces=4, seed=k, use_light_tree=k % 2), spp, cam, w, h))
    server = RenderServer(backend.context, path_capacity=30000)
    ids = []
    for i, (si, st, spp, cam, w, h) in enumerate(jobs):
        ids.append(server.submit(scs[si], st, spp, camera=cam))
        if i == 3:
            time.sleep(0.05)  # later jobs arrive while the first ones run
    got = [_from_server(server, j, w, h) for j, (_, _, _, _, w, h) in zip(ids, jobs)]
    for (si, st, spp, cam, w, h), g in zip(jobs, got):
        ref = _alone(backend, scs[si], scenes.render_settings(w, h, max_bounces=4, seed=st.seed,
                                                               use_light_tree=st.use_light_tree), spp, cam)
        assert _same(g, ref)
    stats = server.stats()
    assert stats.jobs_done == len(jobs) and stats.jobs_failed == 0
    assert stats.latency_jobs == len(jobs) and 0.0 < stats.latency_p50_ms <= stats.latency_p99_ms
    assert stats.wavefronts >= 2
    assert 0.0 < stats.device_ms <= stats.busy_ms + 1.0
    for j in ids:
        server.release(j)
    server.close()


def test_admission_respects_the_budget(backend):
    comp = backend.compile_scene(scenes.cornell_box()).scene
    scene_bytes = backend.context.lib.psy_scene_device_bytes(comp.handle)
    capacity = 20000
    server_probe = RenderServer(backend.context, path_capacity=capacity)
    fixed = server_probe.stats().bytes_in_use
    server_probe.close()
    job_bytes = 64 * 64 * 52 + 256 * 256 * 16 + 4096
    budget = fixed + scene_bytes + int(2.5 * job_bytes)  # two jobs at a time
    server = RenderServer(backend.context, hbm_budget_bytes=budget, path_capacity=capacity)
    st = scenes.render_settings(64, 64, max_bounces=3)
    ids = [server.submit(comp, st, 4) for _ in range(6)]
    for j in ids:
        assert server.wait(j, 120000) == _abi.PSY_OK
        server.release(j)
    s = server.stats()
    assert s.jobs_done == 6 and s.bytes_peak <= budget
    big = server.submit(comp, scenes.render_settings(512, 512), 4)
    assert server.wait(big, 60000) == _abi.PSY_ERROR_OUT_OF_MEMORY
    assert server.poll(big).state == _abi.JOB_FAILED
    server.close()


def test_parameter_edits_are_ordered_with_jobs(backend):
    scene = scenes.cornell_box()
    comp = backend.compile_scene(scene).scene
    st = scenes.render_settings(48, 48, max_bounces=3)
    mat = scene.materials[0]
    before_sc = mat.parameters.scalars.copy()
    after_vc = np.array([[0.2, 0.6, 0.9]], np.float32)
    server = RenderServer(backend.context, path_capacity=20000)
    a = server.submit(comp, st, 6)
    server.rebind_parameters(comp, 0, before_sc, after_vc)
    b = server.submit(comp, st, 6)
    ra, rb = _from_server(server, a, 48, 48), _from_server(server, b, 48, 48)
    server.close()
    # references: the same scene compiled with each parameter state
    ref_before = _alone(backend, backend.compile_scene(scene).scene, st, 6)
    comp2 = backend.compile_scene(scene).scene
    comp2.rebind_parameters(0, before_sc, after_vc)
    ref_after = _alone(backend, comp2, st, 6)
    assert _same(ra, ref_before)
    assert _same(rb, ref_after)
    assert not _same(ra, rb)


def test_cancel_and_errors(backend):
    comp = backend.compile_scene(scenes.cornell_box()).scene
    server = RenderServer(backend.context, path_capacity=20000, max_running=1)
    long_job = server.submit(comp, scenes.render_settings(128, 128, max_bounces=4), 64)
    queued = server.submit(comp, scenes.render_settings(32, 32), 2)
    server.cancel(queued)
    assert server.wait(queued, 60000) == _abi.PSY_ERROR_CANCELLED
    assert server.wait(long_job, 120000) == _abi.PSY_OK
    with pytest.raises(_abi.PsyError):
        server.release(12345)
    assert server.wait(long_job, 1) == _abi.PSY_OK
    server.close()


def test_emissive_edit_while_a_tree_job_runs(backend):
    """An edit of an emissive material reaches the server while a job that
    samples the light tree is running: that job keeps the tree and the
    parameter block it was admitted with, the next job sees the edited
    ones, each equal to a session alone on a scene compiled with the same
    parameters."""
    import copy
    scene = scenes.small_test_scene(seed=3)
    k = next(i for i, m in enumerate(scene.materials) if m.program.has_emission and m.parameters.scalars.size)
    sc = scene.materials[k].parameters.scalars * np.float32(2.5)
    vc = scene.materials[k].parameters.vectors[::-1].copy()
    comp = backend.compile_scene(scene).scene
    st_a = scenes.render_settings(160, 120, max_bounces=5, use_light_tree=1)
    st_b = scenes.render_settings(48, 40, max_bounces=5, use_light_tree=1)
    server = RenderServer(backend.context, path_capacity=40000)
    a = server.submit(comp, st_a, 32)
    server.rebind_parameters(comp, k, sc, vc)
    b = server.submit(comp, st_b, 4)
    ra, rb = _from_server(server, a, 160, 120), _from_server(server, b, 48, 40)
    server.close()
    ref_a = _alone(backend, backend.compile_scene(scene).scene, st_a, 32)
    edited = copy.deepcopy(scene)
    edited.materials[k].parameters.scalars[:] = sc
    edited.materials[k].parameters.vectors[:] = vc
    ref_b = _alone(backend, backend.compile_scene(edited).scene, st_b, 4)
    assert _same(ra, ref_a)
    assert _same(rb, ref_b)
