"""GPU parity of every intra-pair evaluation path against the FP64 oracle.

Ligand sizes from 12 to 80 atoms, through the pair list with the per-warp pair buffer
(every ligand whose list fits it).  Energies and generalised
gradients within 1e-4 relative, grid and direct scoring, curl caps 10 and off.
"""
import numpy as np
import pytest

from gpu_helpers import map_types_for, oracle_grid, perturbed_poses, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-4
SIZES = [(12, 2), (31, 5), (32, 6), (33, 6), (47, 9), (64, 12), (65, 12), (80, 16)]


@pytest.fixture(scope="module")
def path_sys(small_system, oracle64):
    from ud2b200 import Engine, synth
    from ud2b200.model import parse_ligands
    ligd = {f"p{i}": synth.make_ligand(n, t, seed=500 + i, center=small_system["center"])
            for i, (n, t) in enumerate(SIZES)}
    ligs = parse_ligands(ligd)
    sysd = dict(small_system, ligs=ligs)
    eng = Engine(sysd["box"])
    rows = np.asarray([r[:4] for r in sysd["rows"]], np.float64)
    eng.set_receptor(rows[:, :3].astype(np.float32), rows[:, 3].astype(np.int32))
    eng.build_grid(0.375, map_types_for(ligs), 0)
    eng.add_ligands(ligs)
    ogrid, _ = oracle_grid(oracle64, sysd, eng)
    yield dict(sysd, eng=eng, ogrid=ogrid)
    eng.close()


@pytest.mark.parametrize("mode", ["grid", "direct"])
@pytest.mark.parametrize("vcap", [1e30, 10.0])
def test_intra_paths_match_oracle(path_sys, oracle64, mode, vcap):
    from ud2b200 import MODE_DIRECT, MODE_GRID
    eng, box = path_sys["eng"], path_sys["box"]
    env = oracle64.make_env(path_sys["rec"], box, grid=path_sys["ogrid"], mode=mode)
    rng = np.random.default_rng(11)
    pl, xs, cs, rs, want_e, want_g = [], [], [], [], [], []
    for li, lig in enumerate(path_sys["ligs"]):
        assert lig.natom == SIZES[li][0]
        olig = oracle64.ligand(lig)
        for p in perturbed_poses(oracle64, olig, env, lig, rng, 6, box):
            e, g, _ = oracle64.e_grad(olig, env, p["coords"].astype(np.float64), p["center"].astype(np.float64),
                                      p["rot_vec"].astype(np.float64), vcap=vcap)
            pl.append(li); xs.append(p["coords"]); cs.append(p["center"]); rs.append(p["rot_vec"])
            want_e.append(e); want_g.append(g)
    e, gs = eng.score_batch(pl, xs, np.array(cs), np.array(rs), mode=MODE_GRID if mode == "grid" else MODE_DIRECT,
                            vcap=vcap, slope=1e6)
    for k in range(len(pl)):
        n = SIZES[pl[k]][0]
        assert abs(e[k] - want_e[k]) <= TOL * max(1.0, abs(want_e[k])), (n, k, e[k], want_e[k])
        assert rel_err(gs[k], want_g[k]) <= TOL, (n, k, gs[k], want_g[k])


def test_intra_paths_bfgs_lowers_energy(path_sys):
    """A few BFGS steps from the input pose on every path: the energy never rises and the
    records stay finite (the search loop's use of each path)."""
    from ud2b200 import MODE_GRID, make_record
    eng = path_sys["eng"]
    pl = list(range(len(path_sys["ligs"])))
    recs = [make_record(l) for l in path_sys["ligs"]]
    e0, _ = eng.score_batch(pl, [l.coords for l in path_sys["ligs"]], np.array([l.center for l in path_sys["ligs"]]),
                            np.zeros((len(pl), 3), np.float32), mode=MODE_GRID, vcap=10.0, slope=1e6)
    out, ne = eng.bfgs_batch(pl, recs, max_steps=8, vcap=10.0, slope0=1e6, mode=MODE_GRID)
    for k, r in enumerate(out):
        assert np.all(np.isfinite(r))
        assert r[0] <= e0[k] + 1e-3 * max(1.0, abs(e0[k])), (SIZES[k], r[0], e0[k])
        assert ne[k] >= 1
