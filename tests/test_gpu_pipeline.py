"""The drop-in boundary on the GPU: DockingPipeline (the reference's keyword arguments)
docks a small system and writes the reference's JSON files
(<output_dir>/<name_json>_<batch>.json: per ligand a list of poses with a 7-value energy
vector, 3N coordinates and T dihedrals in degrees), as the reference's pose writer reads them
(unidock_processing/unidocktools/unidock_ligand_pose_writer.py:61-91: the coordinate count
must match the ligand's atoms)."""
import glob
import json
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(tmp_path, small_system, **kw):
    from unidock_engine.api.python import pipeline
    c = small_system["center"]
    args = dict(output_dir=str(tmp_path), center_x=c[0], center_y=c[1], center_z=c[2], size_x=20, size_y=20,
                size_z=20, search_mode="free", exhaustiveness=16, mc_steps=8, opt_steps=-1, refine_steps=2,
                num_pose=4, seed=7)
    args.update(kw)
    p = pipeline.DockingPipeline(**args)
    p.set_receptor(small_system["rows"])
    p.add_ligands(small_system["ligd"])
    p.run()
    out = {}
    for fp in sorted(glob.glob(os.path.join(str(tmp_path), "from_python_obj_*.json"))):
        out.update(json.load(open(fp)))
    return p, out


def _check(out, small_system):
    assert set(out) == set(small_system["ligd"])
    for name, poses in out.items():
        lig = small_system["ligd"][name]
        n, t = len(lig["atoms"]), len(lig["torsions"])
        assert 1 <= len(poses) <= 4
        for pose in poses:
            assert len(pose["energy"]) == 7 and all(math.isfinite(v) for v in pose["energy"])
            assert len(pose["coords"]) == 3 * n and len(pose["dihedrals"]) == t


def test_pipeline_writes_reference_json(tmp_path, small_system):
    p, out = _run(tmp_path, small_system)
    _check(out, small_system)
    assert p.last_stats["ligands"] == len(small_system["ligd"])


def test_pipeline_with_learned_proposal_and_kept_poses(tmp_path, small_system):
    from ud2b200 import Engine
    eng = Engine(small_system["box"])
    try:
        eng.mlp_init(3)
        params = eng.mlp_get_params()
    finally:
        eng.close()
    path = str(tmp_path / "proposal.npy")
    np.save(path, params)
    _, out = _run(tmp_path, small_system, proposal_params=path, p_learned=0.5, poses_per_chain=2, autotune=True)
    _check(out, small_system)


def test_pipeline_launches_follow_the_memory_budget(tmp_path, small_system):
    """With the default budget the ligands dock in one launch per size group (the small
    system's 41-atom ligand is in the second group); with max_gpu_mem just above the
    largest ligand's predicted bytes (4096 chains) they dock in the launches the plan gives
    for that budget.  The output files and their layout are the same either way."""
    from ud2b200.batching import plan_launches, predict_dock_bytes, reference_batches, size_groups
    from ud2b200.ligset import parse_ligands_bulk
    kw = dict(exhaustiveness=4096, mc_steps=2)
    ls = parse_ligands_bulk(small_system["ligd"])
    p1, out1 = _run(tmp_path / "one", small_system, **kw)
    assert p1.last_stats["launches"] == sum(1 for g in size_groups(ls.natoms, ls.ntors) if g) == 2
    a = ls.a
    per = predict_dock_bytes(ls.natoms, ls.ntors, np.diff(a["pair_off"][a["atom_off"]]),
                             np.diff(a["rot_off"][a["tors_off"]]), np.diff(a["range_off"][a["tors_off"]]),
                             np.diff(a["bias_off"][a["atom_off"]]), nchain=4096, num_pose=4)
    mb = (int(per.max()) >> 20) + 1
    want = len(plan_launches(reference_batches(ls.natoms, ls.ntors), per, mb << 20))
    assert want > 1
    p2, out2 = _run(tmp_path / "many", small_system, max_gpu_mem=mb, **kw)
    assert p2.last_stats["launches"] == want
    _check(out2, small_system)
    names = lambda d: [f.split("/")[-1] for f in sorted(glob.glob(str(d / "*.json")))]
    assert names(tmp_path / "one") == names(tmp_path / "many") != []
