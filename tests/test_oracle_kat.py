"""The oracle against the reference's own known-answer tests.

Every expected value here is the one the reference engine's Catch2 unit tests assert
(paths relative to unidock/unidock_engine/test/unit/), restated as pytest cases on
the FP64 oracle, with the reference's tolerances (1e-4 absolute unless noted).
"""
import math

import numpy as np
import pytest

PI = 3.1415927
C_H, C_P = 2, 3
TOL = 1e-4


# score/test_vina.cpp:18-39
@pytest.mark.parametrize("d,e,f", [(-1, 0.018315, 0.146525), (0, 1.0, 0.0), (1, 0.018315, -0.146525),
                                   (1.5, 0.000123409804087, -0.00148091764904)])
def test_vina_gaussian1(oracle64, d, e, f):
    ee, ff = oracle64.vina_term(0, d)
    assert abs(ee - e) < TOL and abs(ff - f) < TOL


# score/test_vina.cpp:41-57
@pytest.mark.parametrize("d,e,f", [(0, 0.105399224562, 0.158098836843), (3, 1, 0), (6, 0.105399224562, -0.158098836843)])
def test_vina_gaussian2(oracle64, d, e, f):
    ee, ff = oracle64.vina_term(1, d)
    assert abs(ee - e) < TOL and abs(ff - f) < TOL


# score/test_vina.cpp:59-77
@pytest.mark.parametrize("d,e,f", [(-1, 1, -2), (0, 0, 0), (1, 0, 0)])
def test_vina_repulsion(oracle64, d, e, f):
    ee, ff = oracle64.vina_term(2, d)
    assert abs(ee - e) < TOL and abs(ff - f) < TOL


# score/test_vina.cpp:80-97
@pytest.mark.parametrize("d,e,f", [(0.2, 1, 0), (1, 0.5, -1), (2, 0, 0)])
def test_vina_hydrophobic(oracle64, d, e, f):
    ee, ff = oracle64.vina_term(3, d)
    assert abs(ee - e) < TOL and abs(ff - f) < TOL


# score/test_vina.cpp:99-116
@pytest.mark.parametrize("d,e,f", [(-1, 1, 0), (-0.5, 0.714285714286, -1.42857142857), (0.1, 0, 0)])
def test_vina_hbond(oracle64, d, e, f):
    ee, ff = oracle64.vina_term(4, d)
    assert abs(ee - e) < TOL and abs(ff - f) < TOL


# score/test_vina.cpp:119-135
def test_eval_ef_kat(oracle64):
    e, f = oracle64.eval_ef(0.0, C_P, C_P)
    assert abs(e - (-0.036122)) < TOL
    assert abs(f - (-0.000815)) < TOL


# score/test_bias.cpp:10-27
def test_zalign_kat(oracle64):
    r = np.array([-1.0, 0.0, 0.0])
    out = np.zeros(3)
    e = oracle64.lib.orc_eval_ef_zalign(r.ctypes.data, 1.0, C_H, out.ctypes.data)
    assert abs(e - 15.0) < TOL
    assert np.allclose(out, [22.5, 0, 0], atol=TOL)


# myutils/test_math.cpp:8-30
def test_normalize_angle(oracle64):
    L = oracle64.lib
    for x, want in [(0, 0), (PI, PI), (-PI, -PI), (2 * PI, 0), (-2 * PI, 0), (3 * PI, PI), (-3 * PI, -PI)]:
        assert abs(L.orc_normalize_angle(x) - want) < TOL
    for x, want in [(0, 0), (PI, PI), (-PI, PI), (2 * PI, 0), (-2 * PI, 0), (0.3 + 13 * PI, 3.441592),
                    (0.3 - 13 * PI, 3.441592)]:
        assert abs(L.orc_normalize_angle_2pi(x) - want) < TOL


# myutils/test_math.cpp:42-55
def test_get_radian_in_ranges(oracle64):
    ranges = np.array([-180, -160, 20, 90, 110, 150], np.float64)
    for r2, want in [((0.54, 0.1), 27), ((0.89, 1e-6), 110), ((0.21, 1.0), -160)]:
        rr = np.array(r2, np.float64)
        v = oracle64.lib.orc_get_radian_in_ranges(ranges.ctypes.data, 3, rr.ctypes.data)
        assert abs(v - want) < TOL


# myutils/test_math.cpp:58-68 (the reference test includes mymath.h, whose default n is 31)
def test_get_real_within_by_int(oracle64):
    f = oracle64.lib.orc_get_real_within_by_int
    assert abs(f(0, 0, 10, 31)) < TOL
    assert abs(f(11, 0, 10, 1001) - 11.0 / 1001 * 10) < TOL
    assert abs(f(1002, 0, 10, 1001) - 1.0 / 1001 * 10) < TOL
    assert abs(f(633093634, -30.5, -5.5, 31) - (-23.2419)) < TOL
    assert abs(f(633, -PI, PI, 31) - (-0.5067)) < TOL


# myutils/test_math.cpp:83-96
def test_gaussian_kat(oracle64):
    for args, e, f in [((0, 0, 3), 1, 0), ((1, 1, 3), 1, 0), ((0, 1, 4), 0.939413071, 0.117426634)]:
        ee, ff = oracle64.gaussian(*args)
        assert abs(ee - e) < TOL and abs(ff - f) < TOL


# geometry/test_quaternion.cpp:9-44
def test_quaternion_products(oracle64):
    q3 = np.array([0.9961947, 0, 0, 0.0871557])
    q4 = np.array([0.9848078, 0, 0, 0.1736482])
    oracle64.lib.orc_quaternion_multiply_left(q4.ctypes.data, q3.ctypes.data)
    assert np.allclose(q3, [0.9659258, 0, 0, 0.258819], atol=TOL)
    q1 = np.array([1.0, 2.0, 3.0, 4.0])
    oracle64.lib.orc_quaternion_normalize(q1.ctypes.data)
    assert np.allclose(q1, [0.1826, 0.3651, 0.5477, 0.7303], atol=TOL)
    a = np.array([0.9238795, 0, 0, 0.3826834])
    b = np.array([0.7071068, 0.5, -0.5, 0])
    oracle64.lib.orc_quaternion_normalize(a.ctypes.data)
    oracle64.lib.orc_quaternion_normalize(b.ctypes.data)
    oracle64.lib.orc_quaternion_multiply_left(b.ctypes.data, a.ctypes.data)   # quaternion_increment(a, b)
    assert np.allclose(a, [0.653282, 0.270598, -0.653282, 0.270598], atol=TOL)


# geometry/test_quaternion.cpp:47-80
@pytest.mark.parametrize("v,q,want", [
    ([2, 0, 0], [0.7071068, 0, 0, 0.7071068], [0, 2, 0]),
    ([2, 0, 0], [0.8660254, 0, 0, 0.5], [1, 1.7320508, 0]),
    ([1, 0, 0], [0.51421413, 0.21784632, 0.32676949, 0.76246214], [-0.37625361, 0.92650867, -0.00385983]),
    ([1, 2.3, -9.23], [0.51421413, 0.21784632, 0.32676949, 0.76246214], [-8.02033915, -2.19741106, -4.72529836]),
])
def test_rotate_vec_by_quaternion(oracle64, v, q, want):
    vv = np.array(v, np.float64)
    qq = np.array(q, np.float64)
    oracle64.lib.orc_rotate_vec_by_quaternion(vv.ctypes.data, qq.ctypes.data)
    assert np.allclose(vv, want, atol=TOL)


# geometry/test_quaternion.cpp:83-141
@pytest.mark.parametrize("q,want", [
    ([1, 0, 0, 0], [0, 0, 0]),
    ([0, 0, 0, 1], [0, 0, PI]),
    ([0.7071068, 0.7071068, 0, 0], [PI / 2, 0, 0]),
    ([0.9586831, 0.2370836, 0.0848071, -0.1323853], [0.4808074, 0.1719894, -0.2684785]),
    ([0.9999999, 0.0001, 0, 0], [0.0002, 0, 0]),
])
def test_quaternion_to_rotvec(oracle64, q, want):
    out = oracle64.vec_fn("orc_quaternion_to_rotvec", q)
    assert np.allclose(out, want, atol=TOL)


# geometry/test_rotation.cpp:9-51
def test_rodrigues(oracle64):
    L = oracle64.lib
    for v, axis, ang, want in [([1, 0, 0], [0, 0, 1], math.pi / 2, [0, 1, 0]),
                               ([1, 0, 0], [0, 0, 1], -7 * PI / 2, [0, 1, 0]),
                               ([0, 1, 0], [1, 0, 0], math.pi / 4, [0, 0.7071, 0.7071]),
                               ([0, 0, 0], [0, 0, 1], math.pi / 2, [0, 0, 0])]:
        vv = np.array(v, np.float64)
        ax = np.array(axis, np.float64)
        L.orc_rotate_vec_by_rodrigues(vv.ctypes.data, ax.ctypes.data, ang)
        assert np.allclose(vv, want, atol=TOL)


def _one_atom_system(oracle, r, ntors=0):
    """cuda/test_bfgs.cpp:47-81: receptor C_H at the origin, one C_H ligand atom at (r,0,0);
    the kernel's box is the default +-30 A (model.h:131-139)."""
    from ud2b200.model import Box, Ligand, Receptor
    rec = Receptor(np.zeros((1, 3), np.float32), np.array([C_H], np.int32), np.zeros(1, np.int32), np.zeros(1, np.float32))
    lig = Ligand("one", np.array([[r, 0, 0]], np.float32), np.array([C_H], np.int32), np.zeros(1, np.int32),
                 np.zeros(1, np.float32), np.zeros((0, 2), np.int32), np.zeros(0, np.float32), [], [],
                 np.zeros(2, np.int32), np.zeros(0, np.int32))
    box = Box(np.full(3, -30, np.float32), np.full(3, 30, np.float32))
    return rec, lig, box


# cuda/test_bfgs.cpp:84-132 (energy, gradient and one line-search step, uncapped curl)
def test_one_atom_energy_gradient_linesearch(oracle64):
    o = oracle64
    for r in [0.0, 0.5, 1.0, 1.5]:
        rec, lig, box = _one_atom_system(o, r)
        env = o.make_env(rec, box, mode="direct")
        ol = o.ligand(lig)
        e, g, _ = o.e_grad(ol, env, [[r, 0, 0]], [r, 0, 0], [0, 0, 0], vcap=1e30)
        e_ref, g_ref = o.eval_ef(r - 3.8, C_H, C_H)
        assert abs(e - e_ref) < TOL
        if r == 0:
            g_ref = 0.0
        assert abs(g[0] - g_ref) < TOL and abs(g[1]) < TOL and abs(g[2]) < TOL
        assert np.all(np.abs(g[3:6]) < TOL)
    # r = 1.5: a line search along -g accepts alpha = 1
    pose = dict(coords=np.array([[1.5, 0, 0]]), center=np.array([1.5, 0, 0]), rot_vec=np.zeros(3),
                dihedrals=np.zeros(0))
    p = -g
    moved = o.apply_update(ol, env, pose, p, 1.0)
    e_new, _, _ = o.e_grad(ol, env, moved["coords"], moved["center"], moved["rot_vec"], vcap=1e30)
    assert e_new - e < 1e-4 * 1.0 * float(p @ g)          # Armijo holds at alpha = 1
    assert np.allclose(moved["coords"][0], [1.5 + p[0], p[1], p[2]], atol=TOL)
    rn = float(np.linalg.norm(moved["coords"][0]))
    assert abs(e_new - o.eval_ef(rn - 3.8, C_H, C_H)[0]) < TOL


def _two_atom(o, ca, cb):
    from ud2b200.model import Box, Ligand, Receptor
    rec = Receptor(np.zeros((1, 3), np.float32), np.array([C_H], np.int32), np.zeros(1, np.int32), np.zeros(1, np.float32))
    coords = np.array([ca, cb], np.float32)
    lig = Ligand("two", coords, np.array([C_H, C_H], np.int32), np.zeros(2, np.int32), np.zeros(2, np.float32),
                 np.zeros((0, 2), np.int32), np.zeros(0, np.float32), [], [],
                 np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    box = Box(np.full(3, -30, np.float32), np.full(3, 30, np.float32))
    return rec, lig, box


def _rodrigues_np(v, axis, th):
    c, s = math.cos(th), math.sin(th)
    return c * v + (1 - c) * np.dot(axis, v) * axis + s * np.cross(axis, v)


# cuda/test_bfgs.cpp:214-298 (two atoms: energy, centre and orientation gradients vs FD, tol 0.01)
def test_two_atom_fd_gradients(oracle64):
    o = oracle64
    ca, cb = np.array([1.0, 0, 0]), np.array([1.0, 1.0, 0])
    rec, lig, box = _two_atom(o, ca, cb)
    env = o.make_env(rec, box, mode="direct")
    ol = o.ligand(lig)
    X = np.array([ca, cb])
    c = X.mean(axis=0)
    e1, g1, _ = o.e_grad(ol, env, X, c, [0, 0, 0], vcap=1e30)
    e_ref = (o.eval_ef(1 - 3.8, C_H, C_H)[0] + o.eval_ef(math.sqrt(2) - 3.8, C_H, C_H)[0]
             + o.eval_ef(1 - 3.8, C_H, C_H)[0])
    assert abs(e1 - e_ref) < TOL
    dr = 1e-3
    for i in range(3):
        X2 = X.copy()
        X2[:, i] += dr
        e2, _, _ = o.e_grad(ol, env, X2, X2.mean(axis=0), [0, 0, 0], vcap=1e30)
        assert abs(g1[i] - (e2 - e1) / dr) < 0.01
    rv = np.array([-1.1, 0.2, 0.3])

    def rotated(v):
        th = np.linalg.norm(v)
        ax = v / th
        return np.array([_rodrigues_np(x - c, ax, th) + c for x in X])

    Xr = rotated(rv)
    e1, g1, _ = o.e_grad(ol, env, Xr, c, rv, vcap=1e30)
    dr = 0.005
    for i in range(3):
        v2 = rv.copy()
        v2[i] += dr
        e2, _, _ = o.e_grad(ol, env, rotated(v2), c, v2, vcap=1e30)
        assert abs(g1[3 + i] - (e2 - e1) / dr) < 0.01


def test_philox_known_answer(oracle64):
    """Philox4x32-10 known-answer vectors published with Random123 (kat_vectors)."""
    assert oracle64.philox([0, 0, 0, 0], [0, 0]).tolist() == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle64.philox([0xffffffff] * 4, [0xffffffff] * 2).tolist() == [0x408f276d, 0x41c83b0e, 0xa20bc7c6,
                                                                              0x6d5451fd]
    assert oracle64.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]).tolist() == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]
