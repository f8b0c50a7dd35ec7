"""The drop-in boundary on the GPU: DockingPipeline (the reference's keyword arguments)
docks a small system and writes the reference's JSON files
(<output_dir>/<name_json>_<batch>.json: per ligand a list of poses with a 7-value energy
vector, 3N coordinates and T dihedrals in degrees), as the reference's pose writer reads them
(unidock_processing/unidocktools/unidock_ligand_pose_writer.py:61-91: the coordinate count
must match the ligand's atoms)."""
import glob
import json
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(tmp_path, small_system, **kw):
    from unidock_engine.api.python import pipeline
    c = small_system["center"]
    p = pipeline.DockingPipeline(output_dir=str(tmp_path), center_x=c[0], center_y=c[1], center_z=c[2],
                                 size_x=20, size_y=20, size_z=20, search_mode="free", exhaustiveness=16,
                                 mc_steps=8, opt_steps=-1, refine_steps=2, num_pose=4, seed=7, **kw)
    p.set_receptor(small_system["rows"])
    p.add_ligands(small_system["ligd"])
    p.run()
    out = {}
    for fp in sorted(glob.glob(str(tmp_path / "from_python_obj_*.json"))):
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
