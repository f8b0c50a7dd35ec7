"""Golden files written by the reference's own CUDA engine (core_pipeline, built from its sources;
tests/golden/make_reference_engine_json.py made them on a B200 for the small test system):
the output format and energy vector of this build's JSON writer checked against them on the CPU.

* every number the reference printed follows the rule the writer restates (rapidjson's Double
  with 3 decimal places: truncated, trailing zeros dropped keeping one): a float32 value that
  truncates to the printed text is printed identically by ``_fmt`` and ``_fmt_array``;
* the file layout: ligand -> list of poses, each {"energy", "coords", "dihedrals"} in that order,
  7 energies, 3N coordinates, T dihedrals (src/format/json.cpp:88-191);
* the energy vector relations the writer computes (src/task/DockTask.cpp:224-282): total =
  intra + inter + penalty, affinity = (total - rank-1 intra) / (1 + 0.05846 T), conf_indep =
  affinity - (total - rank-1 intra), each within the 3-decimal truncation of the printed values.
"""
import glob
import json
import os
import re

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_engine_small_*.json")))
SIZES = {"l0": (8, 0), "l1": (14, 2), "l2": (20, 4), "l3": (30, 6), "l4": (41, 9)}
NUM = re.compile(r"(?<=[\[,:])-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?")


@pytest.fixture(scope="module")
def golden():
    assert FILES, "tests/golden/ref_engine_small_*.json missing"
    return [open(fp).read() for fp in FILES]


def _float32_printed_as(tok: str) -> np.float32:
    """A float32 value the reference could have printed as tok: the smallest in magnitude at or
    beyond the printed (truncated) value."""
    t = abs(float(tok))
    v = np.float32(t)
    if float(v) < t:
        v = np.nextafter(v, np.float32(np.inf))
    return -v if tok.startswith("-") else v


def test_number_format_matches_reference_writer(golden):
    from unidock_engine.api.python.pipeline import _fmt, _fmt_array
    toks = [m.group(0) for text in golden for m in NUM.finditer(text)]
    assert len(toks) > 1000
    vals = [_float32_printed_as(t) for t in toks]
    bad = [(t, _fmt(v)) for t, v in zip(toks, vals) if _fmt(v) != t]
    assert not bad, bad[:10]
    assert _fmt_array(np.array(vals, np.float32)) == toks
    # the reference drops trailing zeros: some printed values have fewer than 3 decimals
    assert any(re.fullmatch(r"-?\d+\.\d{1,2}", t) and not t.endswith(".0") for t in toks)


def test_layout_and_energy_vector(golden):
    seen = {}
    for text in golden:
        d = json.loads(text)
        # key order of every pose object as printed
        assert all(m.group(1) == "energy" for m in re.finditer(r'\{"(\w+)":', text) if m.group(1) not in SIZES)
        for name, poses in d.items():
            seen[name] = poses
            n, t = SIZES[name]
            assert 1 <= len(poses) <= 4
            intra_r1 = poses[0]["energy"][2]
            for p in poses:
                assert list(p.keys()) == ["energy", "coords", "dihedrals"]
                e = p["energy"]
                assert len(e) == 7 and len(p["coords"]) == 3 * n and len(p["dihedrals"]) == t
                # each printed value is truncated to 3 decimals: a relation among k printed
                # values holds within k * 1e-3
                total = e[2] + e[3] + e[4]
                assert abs(e[1] - total) <= 4e-3, (name, e)
                aff = (e[1] - intra_r1) / (1.0 + 0.05846 * t)
                assert abs(e[0] - aff) <= 3e-3, (name, e)
                assert abs(e[5] - (e[0] - (e[1] - intra_r1))) <= 4e-3, (name, e)
                assert e[6] == 0.0
                assert all(-180.0 <= a <= 180.0 for a in p["dihedrals"])
    assert set(seen) == set(SIZES)
