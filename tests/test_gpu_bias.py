"""The bias term (positional and z-align, src/cuda/bfgs.cuh:356-388, src/score/vina.h:277-324)
on the GPU against the FP64 oracle: energies and generalised gradients of random poses of
ligands carrying bias records ([x, y, z, V, r2] per atom in the input schema), and the bias
component of the final-score terms."""
import copy

import numpy as np
import pytest

from gpu_helpers import map_types_for, oracle_grid, perturbed_poses, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def bias_sys(small_system, oracle64):
    from ud2b200.model import parse_ligands
    rng = np.random.default_rng(17)
    ligd = copy.deepcopy(small_system["ligd"])
    for name, lig in ligd.items():
        for k, atom in enumerate(lig["atoms"]):
            if k % 3 == 0:                      # bias records on every third atom, some with two
                recs = [[atom[0] + rng.uniform(-1, 1), atom[1] + rng.uniform(-1, 1), atom[2] + rng.uniform(-1, 1),
                         float(rng.uniform(-2, 2)), float(rng.uniform(0.5, 3.0))]]
                if k % 6 == 0:
                    recs.append([atom[0], atom[1] + 0.5, atom[2], -1.0, 1.5])
                atom[:] = list(atom[:8]) + [recs]
    ligs = parse_ligands(ligd)
    assert all(l.bias_atoms.size > 0 for l in ligs)
    return dict(small_system, ligs=ligs, ligd=ligd)


@pytest.mark.parametrize("bias_type,bias_k", [(1, 0.5), (2, 0.1)])
def test_bias_energy_and_gradient_match_oracle(bias_sys, oracle64, bias_type, bias_k):
    from ud2b200 import Engine, MODE_GRID
    box = bias_sys["box"]
    eng = Engine(box)
    try:
        eng.set_flags(False, bias_type, bias_k)
        rows = np.asarray([r[:4] for r in bias_sys["rows"]], np.float64)
        eng.set_receptor(rows[:, :3].astype(np.float32), rows[:, 3].astype(np.int32))
        eng.build_grid(0.375, map_types_for(bias_sys["ligs"]), 0)
        eng.add_ligands(bias_sys["ligs"])
        ogrid, _ = oracle_grid(oracle64, bias_sys, eng)
        env = oracle64.make_env(bias_sys["rec"], box, grid=ogrid, mode="grid", bias_type=bias_type, bias_k=bias_k)
        rng = np.random.default_rng(23)
        pl, xs, cs, rs, we, wg = [], [], [], [], [], []
        for li, lig in enumerate(bias_sys["ligs"]):
            olig = oracle64.ligand(lig)
            for p in perturbed_poses(oracle64, olig, env, lig, rng, 12, box):
                e, g, _ = oracle64.e_grad(olig, env, p["coords"].astype(np.float64), p["center"].astype(np.float64),
                                          p["rot_vec"].astype(np.float64), vcap=10.0)
                pl.append(li); xs.append(p["coords"]); cs.append(p["center"]); rs.append(p["rot_vec"])
                we.append(e); wg.append(g)
        e, gs = eng.score_batch(pl, xs, np.array(cs), np.array(rs), mode=MODE_GRID, vcap=10.0, slope=1e6)
        for k in range(len(pl)):
            assert abs(e[k] - we[k]) <= TOL * max(1.0, abs(we[k])), (k, e[k], we[k])
            assert rel_err(gs[k], wg[k]) <= TOL, (k, gs[k], wg[k])
        # the bias column of the final-score terms
        terms, _ = eng.score_terms(pl, xs)
        env_d = oracle64.make_env(bias_sys["rec"], box, mode="direct", bias_type=bias_type, bias_k=bias_k)
        for k in range(0, len(pl), 7):
            want = oracle64.score_terms(oracle64.ligand(bias_sys["ligs"][pl[k]]), env_d, xs[k].astype(np.float64))
            assert abs(terms[k, 3] - want[3]) <= TOL * max(1.0, abs(want[3])), (k, terms[k], want)
    finally:
        eng.close()
