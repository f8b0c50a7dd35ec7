"""GPU parity for the optimiser, the MC search, clustering and the full docking path."""
import numpy as np
import pytest

from gpu_helpers import engine_for, oracle_grid, perturbed_poses

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_sys(small_system, oracle64):
    eng, mt = engine_for(small_system)
    ogrid, _ = oracle_grid(oracle64, small_system, eng)
    return dict(eng=eng, mt=mt, ogrid=ogrid, **small_system)


def _starts(gpu_sys, oracle, rng, per_lig):
    from ud2b200 import make_record
    env = oracle.make_env(gpu_sys["rec"], gpu_sys["box"], grid=gpu_sys["ogrid"], mode="grid")
    pl, recs, poses = [], [], []
    for li, lig in enumerate(gpu_sys["ligs"]):
        olig = oracle.ligand(lig)
        for p in perturbed_poses(oracle, olig, env, lig, rng, per_lig, gpu_sys["box"]):
            pl.append(li)
            poses.append(p)
            recs.append(make_record(lig, p["coords"], p["center"], p["rot_vec"], p["dihedrals"]))
    return env, pl, recs, poses


def _oracle_bfgs(oracle, lig, env, p, steps, vcap):
    d = dict(coords=p["coords"].astype(np.float64), center=p["center"].astype(np.float64),
             rot_vec=p["rot_vec"].astype(np.float64), dihedrals=p["dihedrals"].astype(np.float64))
    return oracle.bfgs(oracle.ligand(lig), env, d, steps, vcap, 1e6)[0]["energy"]


@pytest.mark.parametrize("steps", [20, 400])
def test_bfgs_minimum_vs_fp64_oracle(gpu_sys, oracle64, oracle32, steps):
    """BFGS from identical starts vs the FP64 oracle.

    The reference algorithm (accepting the last trial after 10 failed Armijo halvings,
    bfgs.cuh:653-667; EPSILON-gated updates) is chaotic in FP32: the oracle's own FP32
    build reaches the FP64 oracle's minimum (|dE| <= 1e-3) only for a fraction of starts.
    The engine is held to that same bar: its agreement rate with the FP64 oracle is not
    worse than the FP32 restatement's (minus sampling noise), its energies carry no bias,
    and every energy it reports is the energy of the pose it returns."""
    from ud2b200 import MODE_GRID, split_record
    eng = gpu_sys["eng"]
    rng = np.random.default_rng(21)
    env, pl, recs, poses = _starts(gpu_sys, oracle64, rng, 8)
    env32 = oracle32.make_env(gpu_sys["rec"], gpu_sys["box"], grid=gpu_sys["ogrid"], mode="grid")
    out, ne = eng.bfgs_batch(pl, recs, max_steps=steps, rounds=1, vcap=10.0, slope0=1e6, mode=MODE_GRID)
    gpu_ok = f32_ok = 0
    d_gpu, d_f32 = [], []
    for k, li in enumerate(pl):
        lig = gpu_sys["ligs"][li]
        got = split_record(lig, out[k])
        e64 = _oracle_bfgs(oracle64, lig, env, poses[k], steps, 10.0)
        e32 = _oracle_bfgs(oracle32, lig, env32, poses[k], steps, 10.0)
        gpu_ok += abs(got["energy"] - e64) <= 1e-3
        f32_ok += abs(e32 - e64) <= 1e-3
        d_gpu.append(got["energy"] - e64)
        d_f32.append(e32 - e64)
        e_chk, _, _ = oracle64.e_grad(oracle64.ligand(lig), env, got["coords"].astype(np.float64),
                                      got["center"].astype(np.float64), got["rot_vec"].astype(np.float64), vcap=10.0)
        assert abs(e_chk - got["energy"]) <= 1e-4 * max(1.0, abs(e_chk))
    n = len(pl)
    print(f"steps={steps}: same minimum as FP64 oracle: engine {gpu_ok}/{n}, FP32 oracle {f32_ok}/{n}; "
          f"median dE engine {np.median(d_gpu):+.4f} FP32 oracle {np.median(d_f32):+.4f}")
    assert gpu_ok >= f32_ok - 0.15 * n
    assert abs(np.median(d_gpu)) <= max(0.05, 2 * abs(np.median(d_f32)))


@pytest.mark.parametrize("steps", [2, 5])
def test_bfgs_short_same_minimum(gpu_sys, oracle64, oracle32, steps):
    """At the refinement unit (2 steps) BFGS from identical starts reaches the FP32
    restatement's energy within 1e-3 kcal/mol for >= 85 % of starts; at 5 steps, where
    FP32 rounding already separates trajectories, it matches the FP64 oracle as often as
    the FP32 restatement does (within 10 % of the starts)."""
    from ud2b200 import MODE_GRID, split_record
    eng = gpu_sys["eng"]
    rng = np.random.default_rng(22)
    env, pl, recs, poses = _starts(gpu_sys, oracle64, rng, 8)
    env32 = oracle32.make_env(gpu_sys["rec"], gpu_sys["box"], grid=gpu_sys["ogrid"], mode="grid")
    out, _ = eng.bfgs_batch(pl, recs, max_steps=steps, rounds=1, vcap=1000.0, slope0=1e6, mode=MODE_GRID)
    ok32 = ok64 = ref_ok = 0
    for k, li in enumerate(pl):
        lig = gpu_sys["ligs"][li]
        got = split_record(lig, out[k])["energy"]
        e32 = _oracle_bfgs(oracle32, lig, env32, poses[k], steps, 1000.0)
        e64 = _oracle_bfgs(oracle64, lig, env, poses[k], steps, 1000.0)
        ok32 += abs(got - e32) <= 1e-3
        ok64 += abs(got - e64) <= 1e-3
        ref_ok += abs(e32 - e64) <= 1e-3
    n = len(pl)
    print(f"steps={steps}: engine vs FP32 oracle {ok32}/{n}, vs FP64 oracle {ok64}/{n}; FP32 vs FP64 oracle {ref_ok}/{n}")
    if steps <= 2:
        assert ok32 >= 0.85 * n
    assert ok64 >= ref_ok - 0.1 * n


def test_search_deterministic(gpu_sys):
    eng = gpu_sys["eng"]
    eng.search(seed=42, nchain=16, mc_steps=20, opt_steps=6, randomize=True)
    a = [eng.chain_poses(l).copy() for l in range(len(gpu_sys["ligs"]))]
    eng.search(seed=42, nchain=16, mc_steps=20, opt_steps=6, randomize=True)
    b = [eng.chain_poses(l).copy() for l in range(len(gpu_sys["ligs"]))]
    for x, y in zip(a, b):
        assert np.array_equal(x, y, equal_nan=True)


def test_search_matches_oracle_chains(gpu_sys, oracle32):
    """Short MC chains (same counter-based RNG stream) against the FP32 oracle: the best
    energy of most chains agrees; all GPU best energies are real energies of their poses."""
    from ud2b200 import split_record
    from oracle import initial_pose
    eng = gpu_sys["eng"]
    nchain, steps, opt = 8, 3, 4
    eng.search(seed=7, nchain=nchain, mc_steps=steps, opt_steps=opt, randomize=True)
    env = oracle32.make_env(gpu_sys["rec"], gpu_sys["box"], grid=gpu_sys["ogrid"], mode="grid")
    agree = total = 0
    for li, lig in enumerate(gpu_sys["ligs"]):
        recs = eng.chain_poses(li)
        olig = oracle32.ligand(lig)
        for c in range(nchain):
            got = split_record(lig, recs[c])
            want, _ = oracle32.mc_chain(olig, env, initial_pose(lig), seed=7, lig_uid=li, chain=c, nchain=nchain,
                                        mc_steps=steps, opt_steps=opt, randomize=True)
            total += 1
            agree += abs(got["energy"] - want["energy"]) <= 1e-3 * max(1.0, abs(want["energy"]))
    print(f"MC chains agreeing with the FP32 oracle: {agree}/{total}")
    assert agree >= 0.6 * total


def test_randomize_matches_oracle(gpu_sys, oracle64):
    """mc_steps=0: the chain's pose is the randomised start, scored with curl 10."""
    from ud2b200 import split_record
    from oracle import initial_pose
    eng = gpu_sys["eng"]
    eng.search(seed=99, nchain=8, mc_steps=0, opt_steps=0, randomize=True)
    env = oracle64.make_env(gpu_sys["rec"], gpu_sys["box"], grid=gpu_sys["ogrid"], mode="grid")
    for li, lig in enumerate(gpu_sys["ligs"]):
        recs = eng.chain_poses(li)
        for c in range(8):
            got = split_record(lig, recs[c])
            want = oracle64.randomize(oracle64.ligand(lig), env, initial_pose(lig), 99, li, c, 8)
            assert np.allclose(got["coords"], want["coords"], atol=2e-3), (li, c)


def test_cluster_bit_exact(gpu_sys, oracle64):
    eng = gpu_sys["eng"]
    eng.search(seed=5, nchain=64, mc_steps=10, opt_steps=4, randomize=True)
    for limit in (0.5, 1.0, 2.0):
        lead, cnt = eng.cluster(limit)
        for li, lig in enumerate(gpu_sys["ligs"]):
            recs = eng.chain_poses(li)
            n = lig.natom
            coords = np.ascontiguousarray(recs[:, 8:8 + 3 * n])
            want = oracle64.cluster(lig.types, coords, recs[:, 0].copy(), limit)
            assert lead[li, :cnt[li]].tolist() == want


def test_dock_end_to_end(gpu_sys, oracle64):
    from ud2b200 import split_record
    eng = gpu_sys["eng"]
    res, ne = eng.dock(seed=3, nchain=32, mc_steps=15, opt_steps=5, refine_steps=3, num_pose=9, rmsd_limit=1.0,
                       energy_range=10.0)
    assert ne > 0
    env = oracle64.make_env(gpu_sys["rec"], gpu_sys["box"], mode="direct")
    for li, lig in enumerate(gpu_sys["ligs"]):
        r = res[li]
        assert 1 <= len(r.records) <= 9
        es = [split_record(lig, x)["energy"] for x in r.records]
        assert es == sorted(es)
        assert es[-1] <= es[0] + 10.0 + 1e-4
        for k, rec in enumerate(r.records):
            want = oracle64.score_terms(oracle64.ligand(lig), env, split_record(lig, rec)["coords"].astype(np.float64))
            assert np.allclose(r.terms[k], want, rtol=1e-4, atol=1e-4)


def test_autotuned_packing_gives_the_same_chains(gpu_sys):
    """The chain packing autotuner changes only how chains are laid over CTAs."""
    eng = gpu_sys["eng"]
    eng.search(seed=42, nchain=24, mc_steps=8, opt_steps=6, randomize=True)
    a = [eng.chain_poses(l).copy() for l in range(len(gpu_sys["ligs"]))]
    eng.set_autotune(True)
    try:
        eng.search(seed=42, nchain=24, mc_steps=8, opt_steps=6, randomize=True)
        b = [eng.chain_poses(l).copy() for l in range(len(gpu_sys["ligs"]))]
    finally:
        eng.set_autotune(False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y, equal_nan=True)


def test_packings_give_the_same_chains(gpu_sys):
    """Every chain packing (4, 8 or 12 warps per CTA; 1 or 2 chains per warp per work item)
    runs the same chains: bit-identical records.  The 12-warp CTAs use the 384-thread
    instantiation, the others the 256-thread ones."""
    eng = gpu_sys["eng"]
    nl = len(gpu_sys["ligs"])
    eng.search(seed=7, nchain=40, mc_steps=8, opt_steps=6, randomize=True)
    want = [eng.chain_poses(l).copy() for l in range(nl)]
    print("default shape:", eng.search_shape())
    try:
        for w, k in [(12, 1), (12, 2), (8, 1), (8, 2), (4, 1), (4, 2)]:
            eng.set_packing(w, k)
            eng.search(seed=7, nchain=40, mc_steps=8, opt_steps=6, randomize=True)
            sh = eng.search_shape()
            assert sh["warps_per_cta"] == w and sh["chains_per_warp"] == k and sh["ctas_per_sm"] >= 1, sh
            assert sh["register_class"] == (2 if w == 12 else sh["register_class"])
            for l in range(nl):
                assert np.array_equal(eng.chain_poses(l), want[l], equal_nan=True), (w, k, l)
    finally:
        eng.set_packing(0, 0)


def test_retained_poses_and_1024_pose_clustering(gpu_sys, oracle64):
    """256 chains keeping 4 poses each.  A chain's kept energies are distinct successive
    bests (unused records: 1e9); the lowest agrees with the one-pose search's best for
    (nearly) every chain (the chains move the same way; a few chaotic chains may part after
    a last-bit difference of the two kernel builds); a second run is bit-identical; and
    clustering all 1024 poses per ligand at 2.0 A is bit-exact against the oracle."""
    eng = gpu_sys["eng"]
    eng.search(seed=13, nchain=256, mc_steps=5, opt_steps=4, randomize=True)
    one = [eng.chain_poses(l)[:, 0].copy() for l in range(len(gpu_sys["ligs"]))]
    eng.set_retain(4)
    try:
        eng.search(seed=13, nchain=256, mc_steps=5, opt_steps=4, randomize=True)
        first = [eng.chain_poses(l).copy() for l in range(len(gpu_sys["ligs"]))]
        eng.search(seed=13, nchain=256, mc_steps=5, opt_steps=4, randomize=True)
        lead, cnt = eng.cluster(2.0)
        agree = total = 0
        for li, lig in enumerate(gpu_sys["ligs"]):
            recs = eng.chain_poses(li)
            assert recs.shape[0] == 1024
            # the reference's arithmetic can leave a NaN rotation vector in a record (a
            # rotation increment that overflowed: the rotation itself falls back to identity)
            assert np.array_equal(recs, first[li], equal_nan=True)
            e4 = recs[:, 0].reshape(256, 4)
            for row in e4:
                used = row[row < 1e9]
                assert len(set(used.tolist())) == len(used)
            agree += int(np.sum(e4.min(axis=1) == one[li]))
            total += 256
            n = lig.natom
            coords = np.ascontiguousarray(recs[:, 8:8 + 3 * n])
            want = oracle64.cluster(lig.types, coords, recs[:, 0].copy(), 2.0)
            assert lead[li, :cnt[li]].tolist() == want
        print(f"chains whose best of 4 equals the one-pose best: {agree}/{total}")
        assert agree >= 0.95 * total
    finally:
        eng.set_retain(1)


def test_constraint_docking_keeps_the_root_fragment(gpu_sys):
    """Constraint docking (no translation or rotation, src/cuda/mc.cu:159-166,
    bfgs.cuh:176,571): atoms that no torsion moves keep their input coordinates exactly in
    every chain's pose, and the rigid-body gradient is zero."""
    from ud2b200 import MODE_GRID
    eng = gpu_sys["eng"]
    eng.set_flags(True, 0, 0.1)
    try:
        eng.search(seed=8, nchain=16, mc_steps=6, opt_steps=5, randomize=True)
        for li, lig in enumerate(gpu_sys["ligs"]):
            moved = np.zeros(lig.natom, bool)
            for r in lig.rotated:
                moved[r] = True
            root = np.where(~moved)[0]
            recs = eng.chain_poses(li)
            x = recs[:, 8:8 + 3 * lig.natom].reshape(len(recs), lig.natom, 3)
            assert np.array_equal(x[:, root, :], np.broadcast_to(lig.coords[root], x[:, root, :].shape))
        lig = gpu_sys["ligs"][-1]
        _, gs = eng.score_batch([len(gpu_sys["ligs"]) - 1], [lig.coords], lig.center[None, :],
                                np.zeros((1, 3), np.float32), mode=MODE_GRID, vcap=10.0)
        assert np.all(gs[0][:6] == 0.0)
    finally:
        eng.set_flags(False, 0, 0.1)
