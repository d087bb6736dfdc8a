"""The CPU oracle pinned to the reference's golden vectors: the tabulated
Sobol LUT fingerprint and rows (tests/test_tabulated_sobol.cpp), the device
Sobol probe bits and shuffled indices (tests/test_luisa_sobol_fallback.cpp),
the cosine-hemisphere and GGX / Beckmann visible-normal cases
(tests/test_luisa_cycles_sample_mapping.cpp),
the path-state transitions (tests/test_luisa_cycles_path_state.cpp), and the
tables the reference's own sampling code produces (oracle/_ref)."""

import ctypes

import numpy as np
import pytest

from oracle import oracle


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_sobol_table_fingerprint(oracle_lib, golden):
    assert oracle_lib.oracle_sobol_fingerprint(256) == golden["sobol"]["table256_fnv1a"]
    t = np.zeros(256 * 256 * 4, np.float32)
    oracle_lib.oracle_sobol_table(256, _p(t))
    bits = t.view(np.uint32).reshape(-1, 4)
    assert bits[0].tolist() == golden["sobol"]["table256_row0_bits"]
    assert bits[1].tolist() == golden["sobol"]["table256_row1_bits"]


@pytest.mark.parametrize("samples,size", [(1, 256), (16, 256), (64, 256), (256, 256), (257, 512),
                                          (4096, 4096), (5000, 8192), (100000, 8192)])
def test_sequence_size_for_samples(oracle_lib, samples, size):
    assert oracle_lib.oracle_sobol_sequence_size(samples) == size


def test_device_sobol_probe(oracle_lib, golden):
    probe = golden["sobol"]["device_probe"]
    t = np.zeros(256 * 256 * 4, np.float32)
    oracle_lib.oracle_sobol_table(256, _p(t))
    rows = t.view(np.uint32).reshape(-1, 4)
    x, y = probe["pixel"]
    h = oracle_lib.oracle_pixel_hash(x, y, probe["seed"]) & 0xFFFFFFFF
    assert h == probe["rng_hash"]
    for (sample, dim), bits, index in zip(probe["queries"], probe["expected_bits"], probe["shuffled_indices"]):
        i = oracle_lib.oracle_shuffled_sample_index(sample, dim, h, 256)
        assert i == index
        assert rows[i].tolist() == bits


def test_cosine_hemisphere_cases(oracle_lib, golden):
    cases = golden["sample_mapping"]["cosine_hemisphere"]
    tol = golden["sample_mapping"]["tolerance"]
    assert len(cases) >= 4
    for c in cases:
        n = np.array(c["normal"], np.float32)
        r = np.array(c["random"], np.float32)
        d = np.zeros(3, np.float32)
        pdf = np.zeros(1, np.float32)
        oracle_lib.oracle_sample_cosine_hemisphere(_p(n), _p(r), _p(d), _p(pdf))
        exp = np.array(c["direction"], np.float32)
        assert np.all(np.abs(d - exp) <= tol * np.maximum(1.0, np.maximum(np.abs(d), np.abs(exp)))), (d, exp)
        assert abs(pdf[0] - c["pdf"]) <= tol * max(1.0, abs(c["pdf"]))


def test_path_state_transitions(oracle_lib, golden):
    ps = golden["path_state"]
    names = ["flag", "visibility", "bounce", "diffuse_bounce", "glossy_bounce", "transmission_bounce",
             "transparent_bounce", "rng_offset"]
    results = {}
    for c in ps["cases"]:
        state = np.array(c["state"], np.uint32)
        limits = np.array(c["limits"], np.uint32)
        out = np.zeros(8, np.uint32)
        oracle_lib.oracle_next_surface(_p(state), c["label"], c["runtime"], _p(limits), _p(out))
        got = dict(zip(names, out.tolist()))
        results[c["name"]] = out
        for k, v in c["expect"].items():
            if k == "contract_visibility":
                assert oracle_lib.oracle_contract_visibility(got["visibility"]) == v
            else:
                assert got[k] == v, (c["name"], k, got[k], v)
    # two transparent transitions consume two 16-dimension blocks
    once = results["transparent"]
    limits = np.array([8, 8, 8, 8, 8], np.uint32)
    out = np.zeros(8, np.uint32)
    oracle_lib.oracle_next_surface(_p(once), 32, 8 | 1024, _p(limits), _p(out))
    tw = ps["transparent_twice"]
    assert out[7] == tw["rng_offset"] and out[7] + 1 == tw["light_dimension"]
    assert out[2] == tw["bounce"] and out[6] == tw["transparent_bounce"]
    assert oracle_lib.oracle_contract_visibility(2 | 4 | 8) == ps["contract_visibility_transmit_diffuse_glossy"]


def test_pixel_filter_tables_match_reference(oracle_lib, golden):
    ref = golden["reference_tables"]["pixel_filter_bits_every37"]
    for key, bits in ref.items():
        f, w = key.split(":")
        t = np.zeros(1024, np.float32)
        oracle_lib.oracle_pixel_filter_table(int(f), ctypes.c_float(float(w)), _p(t))
        assert t.view(np.uint32)[::37].tolist() == bits, key


def test_reference_library_tables_when_built():
    """Cross-checks against the reference's own sampling code compiled into
    oracle/_ref (present where the reference tree was available)."""
    if not oracle.REF_LIB.exists():
        pytest.skip("oracle/_ref not built")
    ref = ctypes.CDLL(str(oracle.REF_LIB))
    lib = oracle.load()
    for size in (256, 512):
        a = np.zeros(size * 256 * 4, np.float32)
        b = np.zeros_like(a)
        lib.oracle_sobol_table(size, _p(a))
        assert ref.ref_sobol_generate_table(size, _p(b)) == 0
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_light_tree_build_matches_reference_fixtures(oracle_lib, golden):
    """The oracle's build_cycles_light_tree restatement reproduces every
    output word (nodes, measures, emitter order, mappings) the reference
    builder produced for seeded populations (src/sampling/light_tree.cpp)."""
    cases = golden["reference_tables"]["light_tree"]
    assert len(cases) >= 6
    for case in cases:
        tree = oracle.build_light_tree(oracle_lib, "oracle_build_light_tree",
                                       oracle.light_tree_emitter_records(case["seed"], case["count"]))
        assert len(tree["node_topology"]) == case["nodes"], case
        assert tree["root"] == case["root"], case
        assert oracle.light_tree_fingerprint(tree) == case["fingerprint"], case


def test_light_tree_structure_invariants(oracle_lib):
    """Parent / child links, leaf ranges and the two identity mappings are
    consistent; distant emitters sit in the root's right branch."""
    rec = oracle.light_tree_emitter_records(11, 300)
    t = oracle.build_light_tree(oracle_lib, "oracle_build_light_tree", rec)
    topo = t["node_topology"]
    root = t["root"]
    assert topo[root][0] == 0xFFFFFFFF and topo[root][5] == 0
    distant_node = topo[root][2]
    assert topo[distant_node][5] == 2
    n = rec.shape[0]
    by_id = rec[np.argsort(rec[:, 18])]
    seen = np.zeros(n, bool)
    for idx, (parent, left, right, first, count, kind) in enumerate(topo):
        if kind == 0:
            assert topo[left][0] == idx and topo[right][0] == idx
        else:
            for slot in range(first, first + count):
                eid = t["emitter_ids"][slot]
                assert not seen[eid]
                seen[eid] = True
                assert t["to_tree"][eid] == slot and t["to_leaf"][eid] == idx
                assert (by_id[eid, 17] != 0.0) == (idx == distant_node)
    assert seen.all()


def test_light_tree_against_reference_library_when_built(oracle_lib):
    """Fresh populations (not in the fixtures) against oracle/_ref."""
    if not oracle.REF_LIB.exists():
        pytest.skip("oracle/_ref not built")
    ref = ctypes.CDLL(str(oracle.REF_LIB))
    for seed, count in [(21, 2), (22, 17), (23, 640), (24, 2500)]:
        rec = oracle.light_tree_emitter_records(seed, count)
        for max_leaf in (1, 8):
            a = oracle.build_light_tree(oracle_lib, "oracle_build_light_tree", rec, max_leaf)
            b = oracle.build_light_tree(ref, "ref_build_light_tree", rec, max_leaf)
            assert oracle.light_tree_fingerprint(a) == oracle.light_tree_fingerprint(b), (seed, count, max_leaf)


def _reflect(half, incoming):
    d = np.float32(2.0) * np.float32(np.dot(incoming, half)) * half - incoming
    return d.astype(np.float32)


def test_visible_normal_cases(oracle_lib, golden):
    """The glossy closures' visible-normal samplers against the GGX sample
    Cycles recorded and the two Beckmann cases of
    tests/test_luisa_cycles_sample_mapping.cpp (reflected directions)."""
    vn = golden["sample_mapping"]["visible_normal"]
    g = vn["ggx"]
    n, i = np.array(g["normal"], np.float32), np.array(g["incoming"], np.float32)
    r = np.array(g["random"], np.float32)
    h = np.zeros(3, np.float32)
    oracle_lib.oracle_sample_visible_normal(0, _p(n), _p(i), ctypes.c_float(g["alpha"]), _p(r), _p(h))
    d, exp = _reflect(h, i), np.array(g["direction"], np.float32)
    tol = g["tolerance"]
    assert np.all(np.abs(d - exp) <= tol * np.maximum(1.0, np.maximum(np.abs(d), np.abs(exp)))), (d, exp)
    for c in vn["beckmann"]:
        n = np.array(c["normal"], np.float32)
        i = np.array(c["incoming_unnormalised"], np.float32)
        i = (i / np.float32(np.sqrt(np.float32(np.dot(i, i))))).astype(np.float32)
        r = np.array(c["random"], np.float32)
        oracle_lib.oracle_sample_visible_normal(1, _p(n), _p(i), ctypes.c_float(c["alpha"]), _p(r), _p(h))
        d, exp = _reflect(h, i), np.array(c["direction"], np.float32)
        tol = vn["beckmann_tolerance"]
        assert np.all(np.abs(d - exp) <= tol * np.maximum(1.0, np.maximum(np.abs(d), np.abs(exp)))), (d, exp)
