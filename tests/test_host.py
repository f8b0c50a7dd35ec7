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
    """rapidjson's Double with 3 decimal places (include/rapidjson/internal/dtoa.h, Prettify):
    truncation of the shortest digits, trailing zeros dropped keeping one, the sign kept on
    values that truncate to zero; non-finite values and |v| > 1e6 clamped (json.cpp:78-85)."""
    from unidock_engine.api.python.pipeline import _fmt
    cases = [(-7.23456, "-7.234"), (12.0, "12.0"), (float("nan"), "1000000.0"), (3e7, "1000000.0"),
             (-3e7, "-1000000.0"), (float("-inf"), "1000000.0"), (0.1, "0.1"), (12.3004, "12.3"),
             (1.102, "1.101"), (1.25, "1.25"), (-0.0004, "-0.0"), (1e-7, "0.0"), (0.0, "0.0"), (-0.0, "-0.0"),
             (0.30000001, "0.3"), (999999.9, "999999.875"), (0.001, "0.001")]
    for v, want in cases:
        assert _fmt(v) == want, (v, _fmt(v), want)


def test_json_number_format_vectorised_matches_scalar():
    from unidock_engine.api.python.pipeline import _fmt, _fmt_array
    rng = np.random.default_rng(4)
    parts = [rng.normal(0, s, 20000) for s in (1e-3, 0.1, 1.0, 30.0, 1e3, 1e5, 3e6)]
    parts.append(np.round(rng.normal(0, 10, 20000), 3))             # values near multiples of 1/1000
    parts.append(rng.integers(-2000, 2000, 5000) / 8.0)             # exact multiples
    parts.append(np.array([0.0, -0.0, np.nan, np.inf, -np.inf, 1e-40, -1e-40, 1e6, -1e6]))
    v = np.concatenate(parts).astype(np.float32)
    got = _fmt_array(v)
    want = [_fmt(float(x)) for x in v]
    bad = [(float(x), a, b) for x, a, b in zip(v, got, want) if a != b]
    assert not bad, bad[:10]


def test_json_writer_layout(tmp_path, small_system):
    """The batch file: per ligand its poses with the 7-value energy vector (affinity from the
    rank-1 intra, float32 arithmetic), 3N coordinates, T dihedrals in degrees and the
    per-atom decomposition, each value printed by the scalar rule."""
    import json
    from ud2b200.engine import DockResult, record_len
    from ud2b200.model import RAD2DEG_F
    from unidock_engine.api.python.pipeline import DockingPipeline, W_CONF, _fmt
    rng = np.random.default_rng(5)
    ligs = small_system["ligs"]
    res = []
    for i, lig in enumerate(ligs):
        k = i % 3                                                       # 0 poses for the first ligand
        recs = [rng.normal(0, 5, record_len(lig)).astype(np.float32) for _ in range(k)]
        res.append(DockResult(recs, rng.normal(0, 3, (k, 4)).astype(np.float32),
                              rng.normal(0, 1, (k, lig.natom, 5)).astype(np.float32)))
    c = small_system["center"]
    p = DockingPipeline(output_dir=str(tmp_path), center_x=c[0], center_y=c[1], center_z=c[2], size_x=20,
                        size_y=20, size_z=20, energy_decomp=True)
    fp = str(tmp_path / "b.json")
    p._dump(fp, ligs, res)
    text = open(fp).read()
    got = json.loads(text)
    assert list(got) == [l.name for l in ligs]
    F = np.float32
    for lig, r in zip(ligs, res):
        poses = got[lig.name]
        assert len(poses) == len(r.records)
        for j, (rec, pose) in enumerate(zip(r.records, poses)):
            intra, inter, pen, bias = (F(x) for x in r.terms[j])
            total = F(F(intra + inter) + pen)
            e_inter = F(total - F(r.terms[0, 0]))
            aff = F(e_inter / F(F(1) + W_CONF * F(lig.ntors)))
            want = [aff, total, intra, inter, pen, F(aff - e_inter), bias]
            n3 = 3 * lig.natom
            exp = ('{"energy":[' + ",".join(_fmt(x) for x in want) + '],"coords":[' +
                   ",".join(_fmt(x) for x in rec[8:8 + n3]) + '],"dihedrals":[' +
                   ",".join(_fmt(F(x * RAD2DEG_F)) for x in rec[8 + n3:8 + n3 + lig.ntors]) +
                   '],"decomp":[' + ",".join("[" + ",".join(_fmt(x) for x in a) + "]" for a in r.decomp[j]) + "]}")
            assert exp in text, (lig.name, j)


def test_bench_contract_helpers():
    """bench.py's metric is the headline metric of the benchmark definition, and the per-launch
    DRAM traffic it reports comes from the committed ncu summaries of both dominant kernels."""
    import bench
    with open(os.path.join(ROOT, "BASELINE.json")) as f:
        assert bench.METRIC == json.load(f)["metric"]
    assert bench.load_traffic("k_search_screen.md") == 12984320.0
    assert bench.load_traffic("k_learn_step_screen.md") == 27495936.0
    peak, kind = bench.load_peaks()
    assert peak > 1000.0 and kind in ("measured", "fallback")


def test_learned_block_sizes(lib):
    """Steps per launch of the learned search: floor(1 / p) in 1..8, 8 at p = 0, 1 while
    recording or for an invalid p (no device needed)."""
    lib.ud_learned_block.argtypes = [C.c_float, C.c_int]
    lib.ud_learned_block.restype = C.c_int
    want = {0.0: 8, 0.05: 8, 0.125: 8, 0.2: 5, 0.25: 4, 0.3: 3, 0.5: 2, 0.6: 1, 1.0: 1, -0.1: 1, 1.5: 1}
    for p, k in want.items():
        assert lib.ud_learned_block(p, 0) == k, p
        assert lib.ud_learned_block(p, 1) == 1
    from ud2b200.engine import learned_block
    assert learned_block(0.25) == 4 and learned_block(0.25, recording=True) == 1


def test_reference_arm_line_contract():
    """bench.py --impl reference prints one JSON line with the arm's contract keys (a tiny
    sample: 4 ligands, 2 MC steps, 1 s)."""
    import subprocess
    import sys
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--ligands", "4", "--mc-steps", "2", "--ref-sample-s", "1"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench_metric() and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["config"]["mc_steps"] == 2 and d["higher_is_better"] is True


def bench_metric():
    with open(os.path.join(ROOT, "BASELINE.json")) as f:
        return json.load(f)["metric"]


def test_size_groups_batches_and_opt_steps_rule():
    """Size groups at their limits (screening.h:19-30: a ligand goes to the first group whose
    atom and torsion limits it meets), batches of at most 1000 in input order, and the
    opt_steps = -1 rule from the first batch (screening.cpp:206-208)."""
    from ud2b200.batching import batches, heuristic_opt_steps, size_groups
    na = [40, 41, 40, 80, 81, 160, 161, 10]
    nt = [8, 8, 9, 16, 1, 32, 0, 33]
    g = size_groups(na, nt)
    assert g == [[0], [1, 2, 3], [4], [5], [6, 7]]
    big = [20] * 2500 + [60] * 10
    b = batches(big, [2] * len(big))
    assert [len(x) for x in b] == [1000, 1000, 500, 10]
    assert b[0][0] == 0 and b[2][-1] == 2499 and b[3][0] == 2500
    assert heuristic_opt_steps(big, [2] * len(big)) == (25 + 20) // 3
    assert heuristic_opt_steps([], []) == 0
    # the first batch is the first non-empty group's: medium ligands only
    assert heuristic_opt_steps([70, 50], [10, 9]) == (25 + 70) // 3
