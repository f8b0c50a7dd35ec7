"""Compact copies of the reference's own acceptance-test inputs, for tests that run where
the reference tree is absent.

Sources (read from the reference tree, paths within the project):
  unidock/unidock_engine/test/data/dev1/simple.json          (parser test, test_json.cpp)
  unidock/unidock_engine/test/data/5S8I/5S8I_unidock2.json   (crystal redock, test/feature/bin)
  unidock/unidock_engine/test/data/5S8I/5S8I_ligand.sdf
  unidock/unidock_engine/test/feature/bin/ud2.yaml
  unidock/unidock_engine/test/data/bias_hbond/input.json     (bias placement, test/feature/bias_hbond)
  unidock/unidock_engine/test/feature/bias_hbond/ud2.yaml
  unidock/unidock_engine/api/python/test/data/1W1P/1W1P_unidock2.json  (pipeline test)
  unidock/unidock_engine/api/python/test/data/1W1P/ud2.yaml

What is kept: simple.json unchanged; for the three docking cases the run settings of the
case's ud2.yaml, the ligands unchanged, and the receptor rows that the engine keeps
(non-hydrogen atoms inside the box grown by 8 A) with a 1 A margin -- every row the engine
drops is dropped here too, so docking results are the same -- with coordinates and charges
written as the shortest decimal of their float32 value (the engine reads float32).  For
5S8I the crystal ligand's coordinates (all atoms, SDF order) are added.

    python tests/golden/make_reference_fixtures.py [reference_root]
"""
import json
import os
import sys

import numpy as np
import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
ENGINE = "unidock/unidock_engine"


def f32(x):
    """The shortest decimal that reads back as the same float32."""
    return float(str(np.float32(x)))


def cut_receptor(rows, center, size, margin=9.0):
    out = []
    c = np.asarray(center, np.float64)
    h = np.asarray(size, np.float64) / 2.0 + margin
    for r in rows:
        if int(r[3]) == 0:
            continue
        if np.all(np.abs(np.asarray(r[:3], np.float64) - c) <= h):
            out.append([f32(r[0]), f32(r[1]), f32(r[2]), int(r[3]), int(r[4]), f32(r[5])])
    return out


def sdf_coords(path):
    with open(path) as f:
        lines = f.readlines()
    n = int(lines[3].split()[0])
    return [[float(v) for v in lines[4 + i].split()[:3]] for i in range(n)]


def case(root, json_rel, yaml_rel, name, extra=None):
    with open(os.path.join(root, json_rel)) as f:
        data = json.load(f)
    with open(os.path.join(root, yaml_rel)) as f:
        cfg = yaml.safe_load(f)
    st, adv = cfg.get("Settings", {}), cfg.get("Advanced", {})
    center = [st["center_x"], st["center_y"], st["center_z"]]
    size = [st["size_x"], st["size_y"], st["size_z"]]
    ligs = {k: v for k, v in data.items() if k not in ("receptor", "score")}
    out = dict(source=dict(json=json_rel, yaml=yaml_rel, receptor_rows_in_source=len(data["receptor"])),
               settings=dict(center=center, size=size, task=st.get("task", "screen"),
                             search_mode=st.get("search_mode", "free"),
                             constraint_docking=bool(st.get("constraint_docking", False)),
                             exhaustiveness=adv["exhaustiveness"], randomize=bool(adv["randomize"]),
                             mc_steps=adv["mc_steps"], opt_steps=adv["opt_steps"], refine_steps=adv["refine_steps"],
                             rmsd_limit=adv["rmsd_limit"], num_pose=adv["num_pose"],
                             energy_range=adv["energy_range"], seed=adv["seed"],
                             use_tor_lib=bool(adv.get("tor_lib", False)),
                             bias=adv.get("bias", st.get("bias", "no")),
                             bias_k=adv.get("bias_k", st.get("bias_k", 0.1))),
               receptor=cut_receptor(data["receptor"], center, size), ligands=ligs)
    if extra:
        out.update(extra)
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(name, len(out["receptor"]), "receptor rows of", len(data["receptor"]), os.path.getsize(os.path.join(HERE, name)))


def main(root):
    with open(os.path.join(root, ENGINE, "test/data/dev1/simple.json")) as f:
        simple = json.load(f)
    with open(os.path.join(HERE, "ref_simple.json"), "w") as f:
        json.dump(simple, f)
    case(root, f"{ENGINE}/test/data/5S8I/5S8I_unidock2.json", f"{ENGINE}/test/feature/bin/ud2.yaml", "ref_5s8i.json",
         extra=dict(crystal=sdf_coords(os.path.join(root, ENGINE, "test/data/5S8I/5S8I_ligand.sdf")),
                    acceptance=dict(best_rmsd_all_atoms_max=2.0)))
    case(root, f"{ENGINE}/test/data/bias_hbond/input.json", f"{ENGINE}/test/feature/bias_hbond/ud2.yaml",
         "ref_bias_hbond.json",
         extra=dict(acceptance=dict(atom=6, site=[1.782, 66.634, 6.337], per_axis_max=0.2, top_poses=5)))
    case(root, f"{ENGINE}/api/python/test/data/1W1P/1W1P_unidock2.json", f"{ENGINE}/api/python/test/data/1W1P/ud2.yaml",
         "ref_1w1p.json")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
