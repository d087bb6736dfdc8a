"""Launch tuning (psy_context_set_tuning): material-sorted shading queues,
grid caps and path capacity change only the schedule, never a result; the
autotuner applies the fastest candidate it measured (gpu-marked)."""

import numpy as np
import pytest

from psycles_b200 import _abi, autotune, scenes
from psycles_b200.backend import BatchRenderer, SampleRange

pytestmark = pytest.mark.gpu

PASSES = (_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT)


def _render(backend, compiled, st, spp):
    s = backend.create_session(compiled, st)
    assert s.render_samples(SampleRange(0, spp, 0, spp)), s.diagnostics
    out = {k: s.read_pass(k) for k in PASSES}
    s.close()
    return out


@pytest.mark.parametrize("tuning", [
    {"sort_threshold": 1, "shadow_sort_threshold": 1, "ray_sort_threshold": 1},
    {"sort_threshold": 1, "shadow_sort_threshold": 0, "path_capacity": 3000, "traversal_blocks_per_sm": 2,
     "shade_blocks_per_sm": 1},
    {"stream_blocks_per_sm": 1, "traversal_blocks_per_sm": 64, "shade_blocks_per_sm": 64},
    {"stream_block_size": 128, "stream_blocks_per_sm": 1},
    {"stream_block_size": 512},
])
def test_tuning_never_changes_results(backend, tuning):
    default = autotune.get_tuning(backend)
    comp = backend.compile_scene(scenes.small_test_scene(seed=6)).scene
    st = scenes.render_settings(80, 60, max_bounces=5)
    ref = _render(backend, comp, st, 6)
    try:
        autotune.set_tuning(backend, dict(default, **tuning))
        got = _render(backend, comp, st, 6)
        batch = BatchRenderer(backend.context, path_capacity=9000)
        s = backend.create_session(comp, st)
        assert batch.render([(s, SampleRange(0, 6, 0, 6))])
        got_batch = {k: s.read_pass(k) for k in PASSES}
    finally:
        autotune.set_tuning(backend, default)
    for k in PASSES:
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
        assert np.array_equal(got_batch[k].view(np.uint32), ref[k].view(np.uint32)), k


def test_autotune_applies_its_best_trial(backend):
    default = autotune.get_tuning(backend)
    comp = backend.compile_scene(scenes.cornell_box()).scene
    st = scenes.render_settings(64, 64, max_bounces=3)
    try:
        res = autotune.autotune(backend, comp, st, spp=2, candidates={"sort_threshold": (0, 1),
                                                                     "shade_blocks_per_sm": (8, 16)})
        assert res.samples_per_s == max(r for _, r in res.trials)
        assert autotune.get_tuning(backend) == res.tuning
    finally:
        autotune.set_tuning(backend, default)


def test_tuning_rejects_out_of_range(backend):
    with pytest.raises(_abi.PsyError):
        autotune.set_tuning(backend, {"shade_blocks_per_sm": 1000})
    with pytest.raises(_abi.PsyError):
        autotune.set_tuning(backend, {"stream_block_size": 96})
