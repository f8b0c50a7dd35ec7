"""ud_score_batch_noalloc (scoring without device allocation) against ud_score_batch.

Collected last on purpose (file name), so it also runs after every other GPU test has used
and released device memory; it passes alone as well.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import engine_for

pytestmark = pytest.mark.gpu

TOL = 1e-6      # same kernel, same inputs: results are expected to be identical


def _poses(system, rng, per_lig):
    pl, xs, cs, rs = [], [], [], []
    box = system["box"]
    mid = (box.lo + box.hi) / 2.0
    for li, lig in enumerate(system["ligs"]):
        for _ in range(per_lig):
            shift = rng.uniform(-3.0, 3.0, 3).astype(np.float32)
            x = (lig.coords - lig.center + mid + shift).astype(np.float32)
            pl.append(li)
            xs.append(x)
            cs.append(x.mean(axis=0))
            rs.append(rng.uniform(-1.0, 1.0, 3).astype(np.float32))
    return pl, xs, np.array(cs, np.float32), np.array(rs, np.float32)


@pytest.mark.parametrize("mode_name", ["grid", "direct"])
def test_noalloc_matches_score_batch_twice(small_system, mode_name):
    from ud2b200 import MODE_DIRECT, MODE_GRID
    mode = MODE_GRID if mode_name == "grid" else MODE_DIRECT
    eng, _ = engine_for(small_system)
    try:
        pl, xs, cs, rs = _poses(small_system, np.random.default_rng(3), 40)
        want_e, want_g = eng.score_batch(pl, xs, cs, rs, mode=mode, vcap=10.0, slope=1e6)
        for _ in range(2):                       # two calls in a row reuse the same staging
            e, gs = eng.score_batch_noalloc(pl, xs, cs, rs, mode=mode, vcap=10.0, slope=1e6)
            np.testing.assert_allclose(e, want_e, rtol=TOL, atol=TOL)
            for g, w in zip(gs, want_g):
                np.testing.assert_allclose(g, w, rtol=TOL, atol=TOL)
    finally:
        eng.close()


def test_noalloc_more_poses_than_one_scan_block(small_system):
    """3000 poses: the offset prefix sums carry across 1024-pose blocks of the scan."""
    from ud2b200 import MODE_GRID
    eng, _ = engine_for(small_system)
    try:
        pl, xs, cs, rs = _poses(small_system, np.random.default_rng(11), 600)
        order = np.random.default_rng(12).permutation(len(pl))        # ligands interleaved
        pl = [pl[i] for i in order]
        xs = [xs[i] for i in order]
        cs, rs = cs[order], rs[order]
        assert len(pl) == 3000
        want_e, want_g = eng.score_batch(pl, xs, cs, rs, mode=MODE_GRID, vcap=10.0, slope=1e6)
        for _ in range(2):
            e, gs = eng.score_batch_noalloc(pl, xs, cs, rs, mode=MODE_GRID, vcap=10.0, slope=1e6)
            np.testing.assert_allclose(e, want_e, rtol=TOL, atol=TOL)
            for g, w in zip(gs, want_g):
                np.testing.assert_allclose(g, w, rtol=TOL, atol=TOL)
    finally:
        eng.close()


def test_noalloc_refuses_a_batch_whose_staging_exceeds_the_array(small_system):
    """16000 poses of the 41-atom ligand: under the pose limit, but coordinates alone take
    7.9 MB and the whole staging more than the fixed 8 MiB, so the call is refused with
    UD_EINVAL before anything is copied; a smaller batch then still goes through."""
    from ud2b200 import EngineError, MODE_GRID
    eng, _ = engine_for(small_system)
    try:
        li = 4
        lig = small_system["ligs"][li]
        assert lig.natom == 41
        pl, xs, cs, rs = _poses(small_system, np.random.default_rng(13), 4)
        want_e, _ = eng.score_batch(pl, xs, cs, rs, mode=MODE_GRID)     # uploads the ligand set
        n = 16000
        x = np.zeros((lig.natom, 3), np.float32)
        with pytest.raises(EngineError, match="bytes of staging"):
            eng.score_batch_noalloc([li] * n, [x] * n, np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32),
                                    mode=MODE_GRID)
        e, _ = eng.score_batch_noalloc(pl, xs, cs, rs, mode=MODE_GRID)
        np.testing.assert_allclose(e, want_e, rtol=TOL, atol=TOL)
    finally:
        eng.close()


def test_noalloc_limits_and_state(small_system):
    from ud2b200 import EngineError, MODE_GRID
    from ud2b200.engine import load_library
    eng, _ = engine_for(small_system)
    try:
        L = load_library()
        one = np.zeros(64, np.float32)
        idx = np.zeros(1, np.int32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        # over the pose limit: refused before any array is read
        rc = L.ud_score_batch_noalloc(eng.h, 16385, p(idx), p(one), p(one), p(one), MODE_GRID, 10.0, 1e6,
                                      p(one), p(one))
        assert rc != 0 and b"exceed" in L.ud_last_error()
        # ligand set not yet uploaded after add_ligands: refused with a state error
        pl, xs, cs, rs = _poses(small_system, np.random.default_rng(5), 2)
        with pytest.raises(EngineError, match="ligand set changed"):
            eng.score_batch_noalloc(pl, xs, cs, rs, mode=MODE_GRID)
        # after one allocating call the same batch goes through
        want_e, _ = eng.score_batch(pl, xs, cs, rs, mode=MODE_GRID)
        e, _ = eng.score_batch_noalloc(pl, xs, cs, rs, mode=MODE_GRID)
        np.testing.assert_allclose(e, want_e, rtol=TOL, atol=TOL)
    finally:
        eng.close()
