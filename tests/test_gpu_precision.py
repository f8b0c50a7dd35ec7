"""Map precision on the uneven workload: energies and gradients of 10,000 random poses of
ligands with 8-80 heavy atoms and 0-20 torsions, scored on FP32 and on FP16 grid maps
(FP32 interpolation), against the FP64 oracle on FP64 maps.  The error statistics are
printed; the bars: FP32 maps 1e-4 relative (the accuracy contract), FP16 maps 2e-2
relative to max(1, |E|) for energies and to max(1, |g|) for gradients."""
import numpy as np
import pytest

from gpu_helpers import map_types_for, oracle_grid, perturbed_poses, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uneven_sys(small_system, oracle64):
    from ud2b200 import Engine, synth
    from ud2b200.model import parse_ligands
    sizes = synth.ligand_sizes("uneven", 25, seed=77)
    ligd = {f"u{i}": synth.make_ligand(n, t, seed=9000 + i, center=small_system["center"]) for i, (n, t) in enumerate(sizes)}
    ligs = parse_ligands(ligd)
    sysd = dict(small_system, ligs=ligs)
    eng = Engine(sysd["box"])
    rows = np.asarray([r[:4] for r in sysd["rows"]], np.float64)
    eng.set_receptor(rows[:, :3].astype(np.float32), rows[:, 3].astype(np.int32))
    eng.build_grid(0.375, map_types_for(ligs), 1)          # FP32 master and FP16 copy
    eng.add_ligands(ligs)
    ogrid, _ = oracle_grid(oracle64, sysd, eng)
    yield dict(sysd, eng=eng, ogrid=ogrid)
    eng.close()


def test_fp16_and_fp32_maps_vs_fp64_on_10000_poses(uneven_sys, oracle64):
    from ud2b200 import GRID_F16, GRID_F32, MODE_GRID
    eng, box, ligs = uneven_sys["eng"], uneven_sys["box"], uneven_sys["ligs"]
    env = oracle64.make_env(uneven_sys["rec"], box, grid=uneven_sys["ogrid"], mode="grid")
    rng = np.random.default_rng(123)
    pl, xs, cs, rs, we, wg = [], [], [], [], [], []
    for li, lig in enumerate(ligs):
        olig = oracle64.ligand(lig)
        for p in perturbed_poses(oracle64, olig, env, lig, rng, 400, box):
            e, g, _ = oracle64.e_grad(olig, env, p["coords"].astype(np.float64), p["center"].astype(np.float64),
                                      p["rot_vec"].astype(np.float64), vcap=10.0)
            pl.append(li); xs.append(p["coords"]); cs.append(p["center"]); rs.append(p["rot_vec"])
            we.append(e); wg.append(g)
    assert len(pl) == 10000
    cs, rs, we = np.array(cs), np.array(rs), np.array(we)
    stats = {}
    for name, prec in (("fp32", GRID_F32), ("fp16", GRID_F16)):
        eng.set_grid_precision(prec)
        e, gs = eng.score_batch(pl, xs, cs, rs, mode=MODE_GRID, vcap=10.0, slope=1e6)
        de = np.abs(e - we) / np.maximum(1.0, np.abs(we))
        dg = np.array([rel_err(g, w) for g, w in zip(gs, wg)])
        stats[name] = (de, dg)
        print(f"{name} maps vs FP64: energy rel err max {de.max():.2e} p99 {np.quantile(de, 0.99):.2e} "
              f"mean {de.mean():.2e}; gradient rel err max {dg.max():.2e} p99 {np.quantile(dg, 0.99):.2e}")
    eng.set_grid_precision(GRID_F32)
    assert stats["fp32"][0].max() <= 1e-4 and stats["fp32"][1].max() <= 1e-4
    assert stats["fp16"][0].max() <= 2e-2 and stats["fp16"][1].max() <= 2e-2
