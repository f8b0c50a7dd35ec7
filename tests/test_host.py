"""Host-side logic and the C ABI's presence (no GPU needed)."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "udock_b200.h")).read()
    return sorted(set(re.findall(r"\b(ud_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "uni-dock2_b200"))
    import build as b
    b.build()
    return C.CDLL(b.OUT)


def test_abi_exports_every_declared_symbol(lib):
    syms = _header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s


def test_abi_error_path_without_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib.ud_create.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]
    lib.ud_last_error.restype = C.c_char_p
    box = np.array([-5, 5, -5, 5, -5, 5], np.float32)
    h = C.c_void_p()
    rc = lib.ud_create(0, box.ctypes.data, C.byref(h))
    assert rc < 0
    assert lib.ud_last_error().decode()
    lib.ud_version.restype = C.c_int
    assert lib.ud_version() >= 100


def test_pack_ligands_roundtrip(small_system):
    from ud2b200.engine import pack_ligands
    ligs = small_system["ligs"]
    p = pack_ligands(ligs)
    assert p["atom_off"][-1] == sum(l.natom for l in ligs)
    assert p["tors_off"][-1] == sum(l.ntors for l in ligs)
    a0 = p["atom_off"][3]
    l3 = ligs[3]
    assert np.array_equal(p["types"][a0:a0 + l3.natom], l3.types)
    assert np.array_equal(p["pairs"][p["pair_off"][a0]:p["pair_off"][a0 + l3.natom]], l3.pairs)


def test_parser_exclusions(small_system):
    """Intra pairs exclude 1-2/1-3, 1-4 and same-rigid-fragment pairs and are symmetric."""
    from ud2b200.model import split_torsions_into_frags
    for name, obj in small_system["ligd"].items():
        lig = [l for l in small_system["ligs"] if l.name == name][0]
        n = lig.natom
        adj = [set(lig.pairs[lig.pair_off[i]:lig.pair_off[i + 1]].tolist()) for i in range(n)]
        for i in range(n):
            for j in adj[i]:
                assert i in adj[j]
        for i, a in enumerate(obj["atoms"]):
            for j in a[6] + a[7]:
                assert j not in adj[i]
        frags = split_torsions_into_frags(set(obj["root_atoms"]), lig.axis, lig.rotated)
        for f in frags:
            for i in f:
                for j in f:
                    assert j not in adj[i]


def test_dihedral_conversion_matches_reference_precision():
    from ud2b200.model import DEG2RAD_F, parse_ligand
    obj = {"atoms": [[0, 0, 0, 2, 0, 0, [1, 2], [3]], [1.5, 0, 0, 2, 0, 0, [0, 2, 3], []],
                     [2, 1.4, 0, 2, 0, 0, [0, 1, 3], []], [3.4, 1.6, 0.5, 2, 0, 0, [1, 2], [0]]],
           "torsions": [[[0, 1, 2, 3], 177.0, [[-180, 180]], [2, 3], []]], "root_atoms": [0, 1]}
    lig = parse_ligand("x", obj)
    assert lig.dihedrals[0] == np.float32(np.float32(177.0) * DEG2RAD_F)
    assert lig.axis.tolist() == [[1, 2]]
    assert np.allclose(lig.ranges[0], [[-3.1415927, 3.1415927]])


def test_tor_lib_ranges_split_across_pi():
    from ud2b200.model import parse_ligand
    obj = {"atoms": [[0, 0, 0, 2, 0, 0, [], []], [1.5, 0, 0, 2, 0, 0, [], []], [2, 1.4, 0, 2, 0, 0, [], []],
                     [3.4, 1.6, 0.5, 2, 0, 0, [], []]],
           "torsions": [[[0, 1, 2, 3], 10.0, [[-180, -160], [-20, 20], [160, -170]], [2, 3], []]], "root_atoms": [0, 1]}
    lig = parse_ligand("x", obj, use_tor_lib=True)
    r = lig.ranges[0]
    assert r.shape == (4, 2)      # the 160..-170 range crossing 180 is split (rapidjson_parser.cpp:152-169)
    assert np.isclose(r[2, 1], 3.1415927) and np.isclose(r[3, 0], -3.1415927)


def test_receptor_filter_box_margin():
    from ud2b200.model import Box, parse_receptor
    box = Box.from_center_size([0, 0, 0], [10, 10, 10])
    rows = [[0, 0, 0, 2, 0, 0.0], [12.9, 0, 0, 3, 0, 0.0], [13.1, 0, 0, 3, 0, 0.0], [1, 1, 1, 0, 0, 0.0]]
    rec = parse_receptor(rows, box)
    assert rec.natom == 2 and rec.types.tolist() == [2, 3]


def test_synth_deterministic():
    from ud2b200 import synth
    a = synth.make_ligand(20, 4, 5, [0, 0, 0])
    b = synth.make_ligand(20, 4, 5, [0, 0, 0])
    assert json.dumps(a) == json.dumps(b)
    assert len(a["torsions"]) == 4 and len(a["atoms"]) == 20


def test_pipeline_presets_and_kwargs():
    import inspect
    from unidock_engine.api.python import pipeline
    sig = inspect.signature(pipeline.DockingPipeline.__init__)
    ref_kw = ["output_dir", "center_x", "center_y", "center_z", "size_x", "size_y", "size_z", "task", "search_mode",
              "exhaustiveness", "randomize", "mc_steps", "opt_steps", "refine_steps", "num_pose", "rmsd_limit",
              "energy_range", "seed", "bias", "bias_k", "constraint_docking", "use_tor_lib", "energy_decomp",
              "gpu_device_id", "name_json", "max_gpu_mem"]
    for k in ref_kw:
        assert k in sig.parameters and sig.parameters[k].kind == inspect.Parameter.KEYWORD_ONLY
    d = {k: v.default for k, v in sig.parameters.items()}
    assert d["exhaustiveness"] == 512 and d["mc_steps"] == 20 and d["opt_steps"] == -1 and d["refine_steps"] == 5
    assert d["num_pose"] == 10 and d["seed"] == 12345 and d["search_mode"] == "balance" and d["task"] == "screen"
    assert d["name_json"] == "from_python_obj" and d["output_dir"] == "./res_ud2"
    mk = lambda **kw: pipeline.DockingPipeline(center_x=0, center_y=0, center_z=0, size_x=1, size_y=1, size_z=1, **kw)
    assert mk(search_mode="fast")._params()["exhaustiveness"] == 128
    assert mk(search_mode="detail")._params()["mc_steps"] == 40
    p = mk(search_mode="free", task="score")._params()
    assert p["mc_steps"] == 0 and p["num_pose"] == 1 and p["exhaustiveness"] == 1
    p = mk(search_mode="free", task="randomize", exhaustiveness=7)._params()
    assert p["num_pose"] == 7 and p["rmsd_limit"] == 0.0
    assert mk(constraint_docking=True)._params()["randomize"] is False
    with pytest.raises(ValueError):
        mk(search_mode="bogus")._params()
    with pytest.raises(ValueError):
        mk(bias="bogus")._params()


def test_pipeline_run_fails_loudly_without_gpu(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from unidock_engine.api.python import pipeline
    from ud2b200 import synth
    rows, c = synth.make_receptor(50, 16.0, seed=1)
    p = pipeline.DockingPipeline(output_dir=str(tmp_path), center_x=c[0], center_y=c[1], center_z=c[2],
                                 size_x=8, size_y=8, size_z=8, search_mode="free", exhaustiveness=2, mc_steps=1)
    p.set_receptor(rows)
    p.add_ligands({"a": synth.make_ligand(6, 1, 1, c)})
    with pytest.raises(RuntimeError, match="Core pipeline failed"):
        p.run()


def test_json_number_format():
    from unidock_engine.api.python.pipeline import _fmt
    assert _fmt(-7.23456) == "-7.234"
    assert _fmt(12.0) == "12.0"
    assert _fmt(float("nan")) == "1000000.0"
    assert _fmt(3e7) == "1000000.0"
