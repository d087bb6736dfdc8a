"""Generate tests/golden/reference_vectors.json from the Psycles reference.

Reads the reference's own C++ tests as text (their expected constants are
golden vectors of the path) and, when oracle/_ref/libpsycles_ref.so was
built from the reference sources (``make -C oracle ref``), records tables
produced by the reference's host code.  Run it where the reference tree is
mounted:

    python tests/golden/make_golden.py /path/to/Psycles

The output is committed; the tests read only the JSON.
"""

from __future__ import annotations

import ctypes
import json
import os
import pathlib
import re
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from oracle import oracle  # noqa: E402  (seeded emitter records, tree outputs)

# (seed, emitter count) of the light-tree build fixtures
LIGHT_TREE_CASES = [(1, 12), (2, 100), (3, 1000), (4, 1), (5, 3), (6, 7), (7, 9), (8, 4000)]


def _hex_list(text: str) -> list[int]:
    return [int(v, 16) for v in re.findall(r"0x([0-9a-fA-F]+)u", text)]


def sobol_fixtures(ref: pathlib.Path) -> dict:
    table_test = (ref / "tests/test_tabulated_sobol.cpp").read_text()
    fingerprint = int(re.search(r"expected_fingerprint\s*=\s*std::uint64_t\{(\d+)ull\}", table_test).group(1))
    rows = _hex_list(table_test[table_test.index("expect_bits(\n        table[0]"):])[:8]
    fallback = (ref / "tests/test_luisa_sobol_fallback.cpp").read_text()
    bits_block = fallback[fallback.index("constexpr std::array expected_bits"):]
    bits_block = bits_block[: bits_block.index("for (auto i")]
    bits = _hex_list(bits_block)
    meta_block = fallback[fallback.index("expected_metadata{"):]
    meta_block = meta_block[: meta_block.index("};")]
    meta = [int(v, 16) if v.startswith("0x") else int(v)
            for v in re.findall(r"(0x[0-9a-fA-F]+|\d+)u", meta_block)]
    # Kernel arguments of the fixture: pixel (17, 29), seed 0, camera
    # sample 0, path sample 63, dims: camera filter 0, first light 17,
    # first bsdf 19, next light 33 (test_luisa_sobol_fallback.cpp:215-227).
    return {
        "table256_fnv1a": fingerprint,
        "table256_row0_bits": rows[:4],
        "table256_row1_bits": rows[4:8],
        "device_probe": {
            "pixel": [17, 29],
            "seed": 0,
            "queries": [[0, 0], [63, 17], [63, 19], [63, 33]],
            "expected_bits": [bits[i:i + 4] for i in range(0, 16, 4)],
            "rng_hash": meta[0],
            "shuffled_indices": meta[7:11],
        },
    }


def sample_mapping_fixtures(ref: pathlib.Path) -> dict:
    text = (ref / "tests/test_luisa_cycles_sample_mapping.cpp").read_text()
    block = text[text.index("constexpr std::array sample_cases"):]
    block = block[: block.index("[[nodiscard]] bool approximately_equal")]
    consts = {
        "inverse_sqrt_three": 0.57735026918962576451,
        "sample_mapping::inverse_pi": 0.31830988618379067154,
    }
    cases = []
    for m in re.finditer(r"SampleCase\{(.*?)\}(?=,\s*(?://.*\n\s*)*SampleCase|\};)", block, re.S):
        body = m.group(1)
        for k, v in consts.items():
            body = body.replace(k, repr(v))
        nums = [float(x) for x in re.findall(r"-?\d+\.\d+(?:e-?\d+)?|-?\d+(?=\.?f)", body.replace("f", " "))]
        cases.append(nums)
    out = []
    for c in cases:
        if len(c) >= 9:
            out.append({"normal": c[0:3], "random": c[3:5], "direction": c[5:8], "pdf": c[8]})
    return {"cosine_hemisphere": out, "tolerance": 2.5e-6, "visible_normal": visible_normal_fixtures(text)}


def _floats(text: str) -> list[float]:
    return [float(x) for x in re.findall(r"-?\d+\.\d+(?:e-?\d+)?", text)]


def visible_normal_fixtures(text: str) -> dict:
    """The GGX and Beckmann visible-normal cases of
    test_luisa_cycles_sample_mapping.cpp: the GGX reflection recorded from
    Cycles (normal, incoming, alpha, random -> reflected direction) and the
    two Beckmann cases (oblique and normal incidence, alpha 0.64, random
    (0.37, 0.73) -> reflected direction)."""
    ggx_call = text[text.index("sample_ggx_visible_normal_reflection("):]
    ggx_call = ggx_call[: ggx_call.index("ggx.write")]
    g = _floats(ggx_call)
    ggx_expected = text[text.index("expected_ggx_direction"):]
    ggx_expected = _floats(ggx_expected[: ggx_expected.index("};")])
    beck = text[text.index("const auto normal = make_float3(0.0f, 0.0f, 1.0f);"):]
    beck = beck[: beck.index("beckmann.write(1u")]
    oblique = _floats(beck[beck.index("oblique_incoming ="): beck.index("const auto sample_random")])
    random = _floats(beck[beck.index("sample_random ="): beck.index("const auto oblique_half")])
    alpha = _floats(beck[beck.index("normal, oblique_incoming,"): beck.index("sample_random);")])
    expected = text[text.index("expected_beckmann_directions{"):]
    expected = _floats(expected[: expected.index("}};")])
    return {
        "ggx": {"normal": g[0:3], "incoming": g[3:6], "alpha": g[6], "random": g[7:9],
                "direction": ggx_expected[0:3], "tolerance": 2.5e-6},
        "beckmann": [
            {"normal": [0.0, 0.0, 1.0], "incoming_unnormalised": oblique, "alpha": alpha[0], "random": random,
             "direction": expected[0:3]},
            {"normal": [0.0, 0.0, 1.0], "incoming_unnormalised": [0.0, 0.0, 1.0], "alpha": alpha[0],
             "random": random, "direction": expected[3:6]},
        ],
        "beckmann_tolerance": 1.0e-5,
    }


def path_state_fixtures(ref: pathlib.Path) -> dict:
    header = (ref / "include/psycles/luisa/cycles_path_state.h").read_text()
    flags = {n: 1 << int(b) for n, b in re.findall(r"constexpr std::uint32_t (flag_\w+) = 1u << (\d+)u;", header)}
    text = (ref / "tests/test_luisa_cycles_path_state.cpp").read_text()
    diffuse_flag = flags["flag_reflect"] | flags["flag_diffuse_ancestor"] | \
        flags["flag_terminate_after_transparent"] | flags["flag_surface_pass"]
    singular_flag = flags["flag_reflect"] | flags["flag_singular"] | flags["flag_mis_skip"] | \
        flags["flag_terminate_after_transparent"] | flags["flag_surface_pass"]
    assert "expected_diffuse_flag" in text and "1668.0f" in text and "48.0f, 49.0f" in text
    # Transitions exercised by test_luisa_cycles_path_state.cpp:38-175 with
    # the records it expects at :341-358.
    initial = [flags["flag_mis_skip"] | flags["flag_transparent_background"], 1, 0, 0, 0, 0, 0, 16]
    return {
        "initial": initial,
        "cases": [
            {"name": "diffuse", "state": initial, "label": 2 | 4, "runtime": 8 | 16,
             "limits": [1, 4, 4, 4, 8],
             "expect": {"flag": diffuse_flag, "visibility": 4, "bounce": 1, "rng_offset": 32,
                        "diffuse_bounce": 1, "glossy_bounce": 0, "transmission_bounce": 0,
                        "transparent_bounce": 0, "contract_visibility": 2}},
            {"name": "transparent", "state": initial, "label": 32, "runtime": 8 | 1024,
             "limits": [8, 8, 8, 8, 1],
             "expect": {"flag": 1668, "visibility": 1, "bounce": 0, "transparent_bounce": 1,
                        "rng_offset": 32, "contract_visibility": 1}},
            {"name": "singular", "state": initial, "label": 2 | 16, "runtime": 8,
             "limits": [8, 8, 1, 8, 8],
             "expect": {"flag": singular_flag, "visibility": 8, "glossy_bounce": 1, "rng_offset": 32}},
        ],
        "transparent_twice": {"rng_offset": 48, "light_dimension": 49, "bounce": 0, "transparent_bounce": 2},
        "contract_visibility_transmit_diffuse_glossy": 8,
    }


def reference_tables() -> dict:
    lib_path = REPO / "oracle/_ref/libpsycles_ref.so"
    if not lib_path.exists():
        return {}
    lib = ctypes.CDLL(str(lib_path))
    out = {}
    filt = {}
    for f in (0, 1, 2):
        for w in (1.0, 1.5, 2.0):
            t = np.zeros(1024, np.float32)
            lib.ref_pixel_filter_table(f, ctypes.c_float(w), t.ctypes.data_as(ctypes.c_void_p))
            filt[f"{f}:{w}"] = t.view(np.uint32)[::37].tolist()
    out["pixel_filter_bits_every37"] = filt
    areas = np.array([0.5, 0.25, 0.0, 2.0, 1e-3], np.float32)
    entries = np.zeros((len(areas) + 3 + 1) * 4, np.float32)
    pdfs = np.zeros(2, np.float32)
    lib.ref_light_distribution.restype = ctypes.c_uint
    n = lib.ref_light_distribution(areas.ctypes.data_as(ctypes.c_void_p), len(areas), 3, 0,
                                   entries.ctypes.data_as(ctypes.c_void_p), pdfs.ctypes.data_as(ctypes.c_void_p))
    out["light_distribution"] = {
        "areas": areas.tolist(), "analytic": 3,
        "entries_bits": entries[: (n + 1) * 4].view(np.uint32).tolist(),
        "triangle_area_pdf_bits": int(pdfs.view(np.uint32)[0]),
        "light_selection_pdf_bits": int(pdfs.view(np.uint32)[1]),
    }
    # build_cycles_light_tree over seeded emitter populations: a fingerprint
    # of every output word, and the node count.
    cases = []
    for seed, count in LIGHT_TREE_CASES:
        tree = oracle.build_light_tree(lib, "ref_build_light_tree", oracle.light_tree_emitter_records(seed, count))
        cases.append({"seed": seed, "count": count, "nodes": int(len(tree["node_topology"])),
                      "root": int(tree["root"]), "fingerprint": oracle.light_tree_fingerprint(tree)})
    out["light_tree"] = cases
    return out


def main() -> None:
    ref = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PSYCLES_REFERENCE", "/root/reference"))
    data = {
        "source": "Psycles reference tests read as text; tables from its sampling sources",
        "sobol": sobol_fixtures(ref),
        "sample_mapping": sample_mapping_fixtures(ref),
        "path_state": path_state_fixtures(ref),
        "reference_tables": reference_tables(),
    }
    (HERE / "reference_vectors.json").write_text(json.dumps(data, indent=1) + "\n")
    print("wrote", HERE / "reference_vectors.json")


if __name__ == "__main__":
    main()
