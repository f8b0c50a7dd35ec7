"""The reference's own acceptance cases on real molecules, through the drop-in DockingPipeline
(hydrogens kept in the coordinates and rotated-atom lists, skipped in scoring; torsion
trees of real ligands), with the settings of each case's ud2.yaml:

* 5S8I crystal redock (test/feature/bin/run_test.sh, validate.py:55-90): the best of the
  output poses lies within 2.0 A all-atom RMSD of the crystal ligand;
* bias_hbond (test/feature/bias_hbond/validate.py:9-30): with a positional bias on atom 6,
  atom 6 of each of the top 5 poses lies within 0.2 A, per axis, of the bias site;
* 1W1P pipeline test (api/python/test/test_pipeline.py:59-157): one pose of the 21-atom
  ligand written to the output directory, and the same run by the reference's own CUDA
  engine (oracle/_ref/udref_dock, when built) reaching a top score this engine matches.

Inputs are the compact fixtures made by tests/golden/make_reference_fixtures.py.
"""
import glob
import json
import math
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
EXE = os.path.join(ROOT, "oracle", "_ref", "udref_dock")


def _case(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def _run(case, out_dir, **over):
    from unidock_engine.api.python import pipeline
    s = dict(case["settings"], **over)
    c, z = s["center"], s["size"]
    dp = pipeline.DockingPipeline(
        output_dir=str(out_dir), center_x=c[0], center_y=c[1], center_z=c[2], size_x=z[0], size_y=z[1], size_z=z[2],
        task=s["task"], search_mode=s["search_mode"], exhaustiveness=s["exhaustiveness"], randomize=s["randomize"],
        mc_steps=s["mc_steps"], opt_steps=s["opt_steps"], refine_steps=s["refine_steps"], num_pose=s["num_pose"],
        rmsd_limit=s["rmsd_limit"], energy_range=s["energy_range"], seed=s["seed"], bias=s["bias"],
        bias_k=s["bias_k"], use_tor_lib=s["use_tor_lib"], constraint_docking=s["constraint_docking"])
    dp.set_receptor(case["receptor"])
    dp.add_ligands(case["ligands"])
    dp.run()
    out = {}
    for fp in sorted(glob.glob(os.path.join(str(out_dir), "*.json"))):
        with open(fp) as f:
            out.update(json.load(f))
    return out


def _rmsd(a, b):
    a = np.asarray(a, np.float64).reshape(-1, 3)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    assert a.shape == b.shape
    return math.sqrt(float(np.sum((a - b) ** 2)) / len(a))


def test_5s8i_redock_finds_the_crystal_pose(tmp_path):
    case = _case("ref_5s8i.json")
    out = _run(case, tmp_path)
    (name,) = case["ligands"]
    poses = out[name]
    assert 1 <= len(poses) <= case["settings"]["num_pose"]
    r = [_rmsd(p["coords"], case["crystal"]) for p in poses]
    print(f"5S8I: top-1 RMSD {r[0]:.3f} A, best {min(r):.3f} A over {len(poses)} poses; "
          f"top-1 energy {poses[0]['energy']}")
    assert min(r) <= case["acceptance"]["best_rmsd_all_atoms_max"]
    es = [p["energy"][0] for p in poses]
    assert es == sorted(es)


def test_bias_hbond_places_the_biased_atom(tmp_path):
    case = _case("ref_bias_hbond.json")
    acc = case["acceptance"]
    out = _run(case, tmp_path)
    (name,) = case["ligands"]
    poses = out[name]
    assert len(poses) >= acc["top_poses"]
    a = acc["atom"]
    for k, p in enumerate(poses[:acc["top_poses"]]):
        xyz = p["coords"][3 * a:3 * a + 3]
        d = [abs(x - y) for x, y in zip(xyz, acc["site"])]
        print(f"bias_hbond pose {k}: atom {a} at {xyz}, |d| per axis {np.round(d, 3).tolist()}, energy {p['energy'][:2]}")
        assert max(d) <= acc["per_axis_max"], (k, xyz)


def test_1w1p_pipeline_and_reference_engine(tmp_path):
    case = _case("ref_1w1p.json")
    out = _run(case, tmp_path / "ours")
    (name,) = case["ligands"]
    natom = len(case["ligands"][name]["atoms"])
    assert len(out[name]) == 1
    pose = out[name][0]
    assert len(pose["coords"]) == 3 * natom and len(pose["dihedrals"]) == 0
    assert all(math.isfinite(v) for v in pose["energy"]) and pose["energy"][1] < 0.0
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/udref_dock not built")
    s = case["settings"]
    inp = tmp_path / "input.json"
    inp.write_text(json.dumps(dict(receptor=case["receptor"], **case["ligands"])))
    rdir = tmp_path / "ref"
    rdir.mkdir()
    opt = (25 + natom) // 3
    cmd = [EXE, str(inp), str(rdir), *map(str, s["center"]), *map(str, s["size"]), str(s["exhaustiveness"]),
           str(s["mc_steps"]), str(opt), str(s["refine_steps"]), str(s["num_pose"]), str(s["rmsd_limit"]),
           str(s["energy_range"]), str(s["seed"]), "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    ref = {}
    for fp in glob.glob(str(rdir / "udref_*.json")):
        ref.update(json.load(open(fp)))
    rp = ref[name][0]
    gap = pose["energy"][1] - rp["energy"][1]
    d = _rmsd(pose["coords"], rp["coords"])
    print(f"1W1P top pose: total {pose['energy'][1]:.3f} here, {rp['energy'][1]:.3f} in the reference engine "
          f"(gap {gap:+.3f} kcal/mol), RMSD between them {d:.3f} A")
    assert gap <= 0.3
