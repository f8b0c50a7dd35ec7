"""GPU parity: grid build, batched E + gradient, final-score terms (through the C ABI).

Tolerances (stated per the engine's accuracy contract):
  * grid maps (FP32 on the GPU) vs FP64 oracle maps: |d| <= 1e-4 * max(1, |v|)
  * per-pose energy vs FP64 oracle: |dE| <= 1e-4 * max(1, |E|)
  * per-pose generalised gradient: max|dg| <= 1e-4 * max(1, max|g|)
  * FP16 maps: error reported and bounded (5e-3 relative of the map range)
"""
import math

import numpy as np
import pytest

from gpu_helpers import engine_for, oracle_grid, perturbed_poses, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def gpu_sys(small_system, oracle64):
    eng, mt = engine_for(small_system)
    ogrid, gmaps = oracle_grid(oracle64, small_system, eng)
    return dict(eng=eng, mt=mt, ogrid=ogrid, gmaps=gmaps, **small_system)


def test_receptor_filter(gpu_sys):
    # hydrogens dropped and atoms beyond box +- 8 A removed (rapidjson_parser.cpp:25-52)
    assert gpu_sys["eng"].receptor_count == gpu_sys["rec"].natom


def test_grid_build_matches_oracle(gpu_sys):
    g = gpu_sys["gmaps"].astype(np.float64)
    o = gpu_sys["ogrid"]["maps"]
    assert g.shape == o.shape
    err = np.abs(g - o) / np.maximum(1.0, np.abs(o))
    assert float(err.max()) <= TOL


@pytest.mark.parametrize("mode", ["grid", "direct"])
@pytest.mark.parametrize("vcap", [1e30, 10.0])
def test_score_batch_matches_oracle(gpu_sys, oracle64, mode, vcap):
    from ud2b200 import MODE_DIRECT, MODE_GRID
    eng = gpu_sys["eng"]
    box = gpu_sys["box"]
    env = oracle64.make_env(gpu_sys["rec"], box, grid=gpu_sys["ogrid"], mode=mode)
    rng = np.random.default_rng(7)
    pl, xs, cs, rs, want_e, want_g = [], [], [], [], [], []
    for li, lig in enumerate(gpu_sys["ligs"]):
        olig = oracle64.ligand(lig)
        for p in perturbed_poses(oracle64, olig, env, lig, rng, 24, box):
            e, g, _ = oracle64.e_grad(olig, env, p["coords"].astype(np.float64), p["center"].astype(np.float64),
                                      p["rot_vec"].astype(np.float64), vcap=vcap)
            pl.append(li); xs.append(p["coords"]); cs.append(p["center"]); rs.append(p["rot_vec"])
            want_e.append(e); want_g.append(g)
    e, gs = eng.score_batch(pl, xs, np.array(cs), np.array(rs), mode=MODE_GRID if mode == "grid" else MODE_DIRECT,
                            vcap=vcap, slope=1e6)
    for k in range(len(pl)):
        assert abs(e[k] - want_e[k]) <= TOL * max(1.0, abs(want_e[k])), (k, e[k], want_e[k])
        assert rel_err(gs[k], want_g[k]) <= TOL, (k, gs[k], want_g[k])


def test_one_atom_kat_through_abi(oracle64):
    """cuda/test_bfgs.cpp:84-132 through the C ABI: E and centre gradient of one C_H atom
    at (r,0,0) over a C_H receptor atom, uncapped."""
    from ud2b200 import Engine, MODE_DIRECT
    from ud2b200.model import Box, Ligand
    box = Box(np.full(3, -30, np.float32), np.full(3, 30, np.float32))
    eng = Engine(box)
    eng.set_receptor(np.zeros((1, 3), np.float32), np.array([2], np.int32))
    lig = Ligand("one", np.array([[1.0, 0, 0]], np.float32), np.array([2], np.int32), np.zeros(1, np.int32),
                 np.zeros(1, np.float32), np.zeros((0, 2), np.int32), np.zeros(0, np.float32), [], [],
                 np.zeros(2, np.int32), np.zeros(0, np.int32))
    eng.add_ligands([lig])
    rs = [0.0, 0.5, 1.0, 1.5]
    e, gs = eng.score_batch([0] * 4, [np.array([[r, 0, 0]], np.float32) for r in rs],
                            np.array([[r, 0, 0] for r in rs], np.float32), np.zeros((4, 3), np.float32),
                            mode=MODE_DIRECT, vcap=1e30)
    for k, r in enumerate(rs):
        e_ref, g_ref = oracle64.eval_ef(r - 3.8, 2, 2)
        assert abs(e[k] - e_ref) < 1e-4
        assert abs(gs[k][0] - (0.0 if r == 0 else g_ref)) < 1e-4
        assert np.all(np.abs(gs[k][1:6]) < 1e-4)


def test_score_terms_match_reference_score(gpu_sys, oracle64):
    """Final scoring terms (no curl) vs the reference's own score() (oracle/_ref shim,
    src/score/score.cpp:12-108) and the oracle restatement."""
    import os
    import ctypes as C
    from ud2b200 import MODE_DIRECT
    eng = gpu_sys["eng"]
    box = gpu_sys["box"]
    env = oracle64.make_env(gpu_sys["rec"], box, mode="direct")
    rng = np.random.default_rng(11)
    pl, xs = [], []
    for li, lig in enumerate(gpu_sys["ligs"]):
        olig = oracle64.ligand(lig)
        for p in perturbed_poses(oracle64, olig, env, lig, rng, 8, box):
            pl.append(li); xs.append(p["coords"])
    terms, _ = eng.score_terms(pl, xs, mode=MODE_DIRECT)
    ref = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libudref_f64.so")
    R = C.CDLL(ref) if os.path.exists(ref) else None
    rec = gpu_sys["rec"]
    for k, li in enumerate(pl):
        lig = gpu_sys["ligs"][li]
        want = oracle64.score_terms(oracle64.ligand(lig), env, xs[k].astype(np.float64))
        if R is not None:
            out4 = np.zeros(4)
            x64 = xs[k].astype(np.float64).reshape(-1)
            rx = rec.xyz.astype(np.float64).reshape(-1)
            b6 = box.as6().astype(np.float64)
            R.udref_score(C.c_int(lig.natom), x64.ctypes.data_as(C.c_void_p), lig.types.ctypes.data_as(C.c_void_p),
                          lig.pair_off.ctypes.data_as(C.c_void_p), lig.pairs.ctypes.data_as(C.c_void_p),
                          C.c_int(rec.natom), rx.ctypes.data_as(C.c_void_p), rec.types.ctypes.data_as(C.c_void_p),
                          b6.ctypes.data_as(C.c_void_p), C.c_int(0), C.c_double(0.1), C.c_int(0), None, None,
                          out4.ctypes.data_as(C.c_void_p))
            assert np.allclose(out4, want, rtol=1e-9, atol=1e-9)
        for j in range(4):
            assert abs(terms[k, j] - want[j]) <= TOL * max(1.0, abs(want[j])), (k, j, terms[k], want)


def test_fp16_maps_error_reported(gpu_sys):
    """FP16 map storage: the interpolated energy error vs FP32 maps is measured and bounded."""
    from ud2b200 import GRID_F16, GRID_F32, MODE_GRID
    eng = gpu_sys["eng"]
    rng = np.random.default_rng(5)
    lig = gpu_sys["ligs"][3]
    xs, cs = [], []
    for _ in range(64):
        off = gpu_sys["box"].lo + 2 + (gpu_sys["box"].hi - gpu_sys["box"].lo - 4) * rng.random(3)
        x = (lig.coords - lig.coords.mean(axis=0) + off).astype(np.float32)
        xs.append(x); cs.append(x.mean(axis=0))
    rv = np.zeros((64, 3), np.float32)
    eng.set_grid_precision(GRID_F32)
    e32, _ = eng.score_batch([3] * 64, xs, np.array(cs), rv, mode=MODE_GRID, vcap=10.0)
    eng.set_grid_precision(GRID_F16)
    e16, _ = eng.score_batch([3] * 64, xs, np.array(cs), rv, mode=MODE_GRID, vcap=10.0)
    eng.set_grid_precision(GRID_F32)
    err = np.abs(e16 - e32) / np.maximum(1.0, np.abs(e32))
    print(f"FP16-vs-FP32 map energy error: max {err.max():.3e} mean {err.mean():.3e}")
    assert err.max() < 5e-3


def test_energy_decomposition_matches_reference(gpu_sys, oracle64):
    """Per-atom decomposition of the intermolecular energy (energy_decomp) against the
    reference's own score_decomp (src/score/score.cpp:114-147, through oracle/_ref)."""
    import os
    import ctypes as C
    from ud2b200 import MODE_DIRECT
    ref = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libudref_f64.so")
    if not os.path.exists(ref):
        pytest.skip("the reference's score_decomp was not built")
    R = C.CDLL(ref)
    eng, box, rec = gpu_sys["eng"], gpu_sys["box"], gpu_sys["rec"]
    env = oracle64.make_env(rec, box, mode="direct")
    rng = np.random.default_rng(19)
    pl, xs = [], []
    for li, lig in enumerate(gpu_sys["ligs"]):
        for p in perturbed_poses(oracle64, oracle64.ligand(lig), env, lig, rng, 4, box):
            pl.append(li); xs.append(p["coords"])
    _, dec = eng.score_terms(pl, xs, mode=MODE_DIRECT, decomp=True)
    rx = rec.xyz.astype(np.float64).reshape(-1)
    off = 0
    for k, li in enumerate(pl):
        lig = gpu_sys["ligs"][li]
        want = np.zeros(5 * lig.natom)
        x64 = xs[k].astype(np.float64).reshape(-1)
        R.udref_score_decomp(C.c_int(lig.natom), x64.ctypes.data_as(C.c_void_p), lig.types.ctypes.data_as(C.c_void_p),
                             C.c_int(rec.natom), rx.ctypes.data_as(C.c_void_p), rec.types.ctypes.data_as(C.c_void_p),
                             want.ctypes.data_as(C.c_void_p))
        got = dec[off:off + 5 * lig.natom]
        off += 5 * lig.natom
        assert np.all(np.abs(got - want) <= 1e-4 * np.maximum(1.0, np.abs(want))), (k, np.max(np.abs(got - want)))
