"""Per-path traces in the reference's schema v2 (not gpu-marked).

psycles_b200.trace_schema restates the 328-slot layout of
include/psycles/luisa/path_trace_schema.h / tools/cycles_path_trace_schema.py
and the comparator policy of tools/compare_cycles_path_traces.py:140-280.
Where the reference tree is present (this container) its own schema module
and comparator are imported from tools/ and must agree with ours: the same
slots, components and policies, and the same verdicts on oracle trace
documents -- identical, a changed random sample, float differences inside
and outside the 1e-6 + 2e-6 * max bound, a slot written on one side only.
The GPU tests compare CUDA traces with the oracle's through `compare`."""

import copy
import os
import pathlib
import sys

import pytest

from oracle.oracle import OracleFilm, OracleScene
from psycles_b200 import scenes, trace_schema

REFERENCE_TOOLS = pathlib.Path(os.environ.get("PSYCLES_REFERENCE", "/root/reference")) / "tools"


def reference_tools():
    if not (REFERENCE_TOOLS / "compare_cycles_path_traces.py").exists():
        pytest.skip("the reference's tools/ directory is not present")
    if str(REFERENCE_TOOLS) not in sys.path:
        sys.path.insert(0, str(REFERENCE_TOOLS))
    import compare_cycles_path_traces
    import cycles_path_trace_schema
    return cycles_path_trace_schema, compare_cycles_path_traces


def oracle_documents():
    scene = scenes.small_test_scene(seed=1)
    prepared = OracleScene(scene.to_desc())
    docs = []
    for x, y, s in [(31, 20, 1), (10, 40, 2), (50, 10, 0), (20, 25, 3)]:
        st = scenes.render_settings(64, 48, max_bounces=6, window_x=x, window_y=y, window_width=1, window_height=1)
        t = OracleFilm(st).render_prepared(prepared, s, 1, 4, trace=(x, y, s))
        docs.append(trace_schema.document(t, source=f"oracle {x},{y},{s}"))
    return docs


def test_slot_layout_matches_the_reference_schema():
    schema, _ = reference_tools()
    ours = trace_schema.slots()
    assert len(ours) == schema.AOV_COUNT == trace_schema.SLOT_COUNT == 328
    assert (schema.SCHEMA_NAME, schema.SCHEMA_VERSION) == (trace_schema.SCHEMA_NAME, trace_schema.SCHEMA_VERSION)
    for a, b in zip(ours, schema.SLOTS):
        assert (a.index, a.scope, a.name, tuple(a.components), a.event, a.closure) == \
            (b.index, b.scope, b.name, tuple(b.components), b.event, b.closure)
        assert tuple(a.policies) == tuple(schema.comparison_policies(b)), a.name


def test_documents_written_where_recorded():
    docs = oracle_documents()
    for d in docs:
        assert d["global"]["header"]["written"] and d["global"]["header"]["schema_version"] == 2
    written = {name for d in docs for e in d["events"] for name, rec in e["slots"].items() if rec["written"]}
    assert {"random_bsdf", "isect_id", "bsdf_wo", "post_flags", "nee_contribution"} <= written, written


def test_comparator_verdicts_equal_the_reference_comparator():
    _, compare_tool = reference_tools()
    docs = oracle_documents()
    for doc in docs:
        same = copy.deepcopy(doc)
        assert compare_tool.compare_traces(doc, same)["passed"]
        assert trace_schema.compare(doc, same) == []
        cases = []
        # a random sample differs by one bit: exact gate
        r = copy.deepcopy(doc)
        r["events"][0]["slots"]["random_bsdf"]["u"] = float(r["events"][0]["slots"]["random_bsdf"]["u"]) * (1 + 2 ** -23)
        cases.append(r)
        # a float inside and one outside the bound
        for scale in (1 + 1e-7, 1 + 1e-4):
            f = copy.deepcopy(doc)
            f["global"]["ray_d"]["x"] = float(f["global"]["ray_d"]["x"]) * scale + 1e-9
            cases.append(f)
        # a slot written on one side only
        w = copy.deepcopy(doc)
        w["events"][0]["slots"]["bsdf_wo"]["written"] = not w["events"][0]["slots"]["bsdf_wo"]["written"]
        cases.append(w)
        # an exact discrete field
        x = copy.deepcopy(doc)
        x["global"]["rng"]["sample"] += 1
        cases.append(x)
        for case in cases:
            ref = compare_tool.compare_traces(doc, case)
            ours = trace_schema.compare(doc, case)
            assert ref["passed"] == (ours == []), (case["global"]["ray_d"], ref["failures"], ours)
            assert sorted(f["field"] for f in ref["failures"]) == sorted(ours)
