"""ctypes wrapper of the CPU oracle (udock_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, as the checker.  The product never
imports this module.

The oracle is an FP64 (or FP32, ``precision="f32"``) restatement of the reference
engine's hot path; see udock_oracle.h for the reference file:line of every piece.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def build(quiet: bool = True) -> None:
    """Compile the oracle libraries (and the reference shim when the reference is present)."""
    subprocess.run(["make", "-C", HERE, "all"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _libpath(prec: str) -> str:
    return os.path.join(HERE, f"liborc_{prec}.so")


class _Lig(C.Structure):
    _fields_ = [("natom", C.c_int), ("ntors", C.c_int), ("types", C.c_void_p), ("axis", C.c_void_p),
                ("range_off", C.c_void_p), ("ranges", C.c_void_p), ("rot_off", C.c_void_p),
                ("rot_atoms", C.c_void_p), ("pair_off", C.c_void_p), ("pairs", C.c_void_p),
                ("bias_off", C.c_void_p), ("bias", C.c_void_p)]


def _env_struct(real):
    class _Env(C.Structure):
        _fields_ = [("nrec", C.c_int), ("rec_xyz", C.c_void_p), ("rec_types", C.c_void_p),
                    ("box_lo", real * 3), ("box_hi", real * 3), ("mode", C.c_int),
                    ("nmaps", C.c_int), ("map_of_type", C.c_void_p), ("maps", C.c_void_p),
                    ("origin", real * 3), ("spacing", real), ("gdim", C.c_int * 3),
                    ("constraint", C.c_int), ("bias_type", C.c_int), ("bias_k", real)]
    return _Env


def _pose_struct(real):
    class _Pose(C.Structure):
        _fields_ = [("energy", real), ("center", real * 3), ("rot_vec", real * 3),
                    ("coords", C.c_void_p), ("dihedrals", C.c_void_p)]
    return _Pose


class _SearchParam(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("lig_uid", C.c_int), ("nchain", C.c_int), ("mc_steps", C.c_int),
                ("opt_steps", C.c_int), ("randomize", C.c_int)]


def _p(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size else 0


class OLigand:
    """Ligand topology held in the oracle's dtype."""

    def __init__(self, lig, dt):
        self.lig = lig
        T = lig.ntors
        self.types = np.ascontiguousarray(lig.types, np.int32)
        self.axis = np.ascontiguousarray(lig.axis.reshape(-1), np.int32) if T else np.zeros(2, np.int32)
        counts = [len(r) for r in lig.ranges]
        self.range_off = np.zeros(T + 1, np.int32)
        self.range_off[1:] = np.cumsum(counts) if T else []
        self.ranges = (np.concatenate([np.asarray(r, np.float64).reshape(-1) for r in lig.ranges]).astype(dt)
                       if T else np.zeros(2, dt))
        rc = [len(r) for r in lig.rotated]
        self.rot_off = np.zeros(T + 1, np.int32)
        self.rot_off[1:] = np.cumsum(rc) if T else []
        self.rot_atoms = (np.concatenate(lig.rotated).astype(np.int32) if T and sum(rc) else np.zeros(1, np.int32))
        self.pair_off = np.ascontiguousarray(lig.pair_off, np.int32)
        self.pairs = np.ascontiguousarray(lig.pairs, np.int32) if lig.pairs.size else np.zeros(1, np.int32)
        boff, bpar = lig.bias_csr()
        self.bias_off = np.ascontiguousarray(boff, np.int32)
        self.bias = np.ascontiguousarray(bpar.astype(dt).reshape(-1)) if bpar.size else np.zeros(5, dt)
        self.s = _Lig(lig.natom, T, _p(self.types), _p(self.axis), _p(self.range_off), _p(self.ranges),
                      _p(self.rot_off), _p(self.rot_atoms), _p(self.pair_off), _p(self.pairs),
                      _p(self.bias_off), _p(self.bias))


class Oracle:
    """FP64 (default) or FP32 CPU restatement of the docking hot path."""

    def __init__(self, precision: str = "f64"):
        path = _libpath(precision)
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        self.dt = np.float64 if precision == "f64" else np.float32
        self.real = C.c_double if precision == "f64" else C.c_float
        self.Env = _env_struct(self.real)
        self.Pose = _pose_struct(self.real)
        L = self.lib
        r = self.real
        L.orc_eval_ef.restype = r
        L.orc_eval_ef.argtypes = [r, C.c_int, C.c_int, C.POINTER(r)]
        L.orc_e_grad.restype = r
        L.orc_e_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, r, r, C.c_void_p, C.c_void_p]
        L.orc_e_f.restype = r
        L.orc_e_f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, r, r, C.c_void_p]
        L.orc_score_terms.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_grid_build.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, r,
                                     C.c_void_p, C.c_void_p]
        L.orc_bfgs.restype = C.c_int
        L.orc_bfgs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, r, r]
        L.orc_apply_update.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, r]
        L.orc_line_search.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, r, r, r,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_mc_chain.restype = C.c_long
        L.orc_mc_chain.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_randomize.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.orc_cluster.restype = C.c_int
        L.orc_cluster.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]
        L.orc_philox4x32_10.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_e_grad_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       r, r, C.c_void_p, C.c_void_p]
        for name, nargs in [("orc_normalize_angle", 1), ("orc_normalize_angle_2pi", 1)]:
            f = getattr(L, name)
            f.restype = r
            f.argtypes = [r] * nargs
        L.orc_vina_term.restype = r
        L.orc_vina_term.argtypes = [C.c_int, r, C.POINTER(r)]
        L.orc_gaussian.restype = r
        L.orc_gaussian.argtypes = [r, r, r, C.POINTER(r)]
        L.orc_clamp_by_ranges.restype = r
        L.orc_clamp_by_ranges.argtypes = [r, C.c_void_p, C.c_int]
        L.orc_get_radian_in_ranges.restype = r
        L.orc_get_radian_in_ranges.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_get_real_within_by_int.restype = r
        L.orc_get_real_within_by_int.argtypes = [C.c_int, r, r, C.c_int]
        for name in ["orc_rotvec_to_quaternion", "orc_quaternion_to_rotvec", "orc_rotate_vec_by_quaternion",
                     "orc_quaternion_multiply_left"]:
            getattr(L, name).argtypes = [C.c_void_p, C.c_void_p]
        L.orc_quaternion_normalize.argtypes = [C.c_void_p]
        L.orc_rotate_vec_by_rodrigues.argtypes = [C.c_void_p, C.c_void_p, r]
        L.orc_grad_rot_over_vec.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.orc_eval_ef_zalign.restype = r
        L.orc_eval_ef_zalign.argtypes = [C.c_void_p, r, C.c_int, C.c_void_p]
        L.orc_grid_interp.restype = r
        L.orc_grid_interp.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]

    # ------------------------------------------------------------- scalars
    def eval_ef(self, d: float, t1: int, t2: int) -> Tuple[float, float]:
        f = self.real(0)
        e = self.lib.orc_eval_ef(d, t1, t2, C.byref(f))
        return float(e), float(f.value)

    def vina_term(self, which: int, d: float):
        f = self.real(0)
        e = self.lib.orc_vina_term(which, d, C.byref(f))
        return float(e), float(f.value)

    def gaussian(self, d, off, w):
        f = self.real(0)
        e = self.lib.orc_gaussian(d, off, w, C.byref(f))
        return float(e), float(f.value)

    def vec_fn(self, name: str, *arrays, out_len: int = 3, extra=()):
        arrs = [np.ascontiguousarray(a, self.dt) for a in arrays]
        out = np.zeros(out_len, self.dt)
        getattr(self.lib, name)(_p(out), *[_p(a) for a in arrs], *extra)
        return out

    def philox(self, ctr: Sequence[int], key: Sequence[int]) -> np.ndarray:
        c = np.asarray(ctr, np.uint32)
        k = np.asarray(key, np.uint32)
        o = np.zeros(4, np.uint32)
        self.lib.orc_philox4x32_10(_p(c), _p(k), _p(o))
        return o

    # ------------------------------------------------------------- environment
    def make_env(self, receptor=None, box=None, grid=None, mode: str = "direct", constraint: bool = False,
                 bias_type: int = 0, bias_k: float = 0.1):
        """Scoring environment.  grid = dict(maps, map_of_type, origin, spacing, gdim)."""
        env = self.Env()
        keep = []
        if receptor is not None:
            rx = np.ascontiguousarray(receptor.xyz.reshape(-1), self.dt)
            rt = np.ascontiguousarray(receptor.types, np.int32)
            keep += [rx, rt]
            env.nrec = receptor.natom
            env.rec_xyz = _p(rx)
            env.rec_types = _p(rt)
        if box is not None:
            for a in range(3):
                env.box_lo[a] = float(box.lo[a])
                env.box_hi[a] = float(box.hi[a])
        env.mode = 0 if mode == "direct" else 1
        if grid is not None:
            maps = np.ascontiguousarray(grid["maps"], self.dt)
            mot = np.ascontiguousarray(grid["map_of_type"], np.int32)
            keep += [maps, mot]
            env.nmaps = int(maps.shape[0])
            env.maps = _p(maps)
            env.map_of_type = _p(mot)
            for a in range(3):
                env.origin[a] = float(grid["origin"][a])
                env.gdim[a] = int(grid["gdim"][a])
            env.spacing = float(grid["spacing"])
        env.constraint = int(constraint)
        env.bias_type = int(bias_type)
        env.bias_k = float(bias_k)
        env._keep = keep
        return env

    def grid_build(self, receptor, map_types: Sequence[int], origin, spacing: float, gdim) -> np.ndarray:
        rx = np.ascontiguousarray(receptor.xyz.reshape(-1), self.dt)
        rt = np.ascontiguousarray(receptor.types, np.int32)
        mt = np.asarray(map_types, np.int32)
        org = np.asarray(origin, self.dt)
        gd = np.asarray(gdim, np.int32)
        out = np.zeros((len(mt), int(gd[2]), int(gd[1]), int(gd[0])), self.dt)
        self.lib.orc_grid_build(receptor.natom, _p(rx), _p(rt), len(mt), _p(mt), _p(org), spacing, _p(gd), _p(out))
        return out

    # ------------------------------------------------------------- poses
    def ligand(self, lig) -> OLigand:
        return OLigand(lig, self.dt)

    def _pose(self, olig: OLigand, coords, center, rot_vec, dihedrals=None, energy=0.0):
        P = self.Pose()
        c = np.ascontiguousarray(np.asarray(coords, self.dt).reshape(-1)).copy()
        d = np.ascontiguousarray(np.asarray(dihedrals if dihedrals is not None else np.zeros(olig.lig.ntors),
                                            self.dt)).copy()
        if d.size == 0:
            d = np.zeros(1, self.dt)
        P.energy = energy
        for a in range(3):
            P.center[a] = float(center[a])
            P.rot_vec[a] = float(rot_vec[a])
        P.coords = _p(c)
        P.dihedrals = _p(d)
        P._c, P._d = c, d
        return P

    @staticmethod
    def _unpose(P, olig) -> dict:
        return dict(energy=float(P.energy), center=np.array(P.center[:]), rot_vec=np.array(P.rot_vec[:]),
                    coords=P._c.reshape(-1, 3).copy(), dihedrals=P._d[:olig.lig.ntors].copy())

    def e_grad(self, olig: OLigand, env, coords, center, rot_vec, vcap=1e30, slope=1e6):
        P = self._pose(olig, coords, center, rot_vec)
        g = np.zeros(6 + olig.lig.ntors, self.dt)
        f = np.zeros(3 * olig.lig.natom, self.dt)
        e = self.lib.orc_e_grad(C.byref(olig.s), C.byref(env), C.byref(P), vcap, slope, _p(g), _p(f))
        return float(e), g, f.reshape(-1, 3)

    def e_grad_batch(self, olig: OLigand, env, coords, centers, rotvecs, vcap=1e30, slope=1e6):
        n = coords.shape[0]
        c = np.ascontiguousarray(coords.reshape(n, -1), self.dt)
        ce = np.ascontiguousarray(centers, self.dt)
        rv = np.ascontiguousarray(rotvecs, self.dt)
        e = np.zeros(n, self.dt)
        g = np.zeros((n, 6 + olig.lig.ntors), self.dt)
        self.lib.orc_e_grad_batch(C.byref(olig.s), C.byref(env), n, _p(c), _p(ce), _p(rv), vcap, slope, _p(e), _p(g))
        return e, g

    def score_terms(self, olig: OLigand, env, coords) -> np.ndarray:
        c = np.ascontiguousarray(np.asarray(coords, self.dt).reshape(-1))
        out = np.zeros(4, self.dt)
        self.lib.orc_score_terms(C.byref(olig.s), C.byref(env), _p(c), _p(out))
        return out

    def apply_update(self, olig, env, pose: dict, g, alpha) -> dict:
        P = self._pose(olig, pose["coords"], pose["center"], pose["rot_vec"], pose["dihedrals"])
        gg = np.ascontiguousarray(g, self.dt)
        self.lib.orc_apply_update(C.byref(olig.s), C.byref(env), C.byref(P), _p(gg), alpha)
        return self._unpose(P, olig)

    def bfgs(self, olig, env, pose: dict, max_steps: int, vcap=10.0, slope=1e6) -> Tuple[dict, int]:
        P = self._pose(olig, pose["coords"], pose["center"], pose["rot_vec"], pose["dihedrals"],
                       pose.get("energy", 0.0))
        n = self.lib.orc_bfgs(C.byref(olig.s), C.byref(env), C.byref(P), max_steps, vcap, slope)
        return self._unpose(P, olig), int(n)

    def mc_chain(self, olig, env, pose: dict, seed: int, lig_uid: int, chain: int, nchain: int,
                 mc_steps: int, opt_steps: int, randomize: bool = True) -> Tuple[dict, int]:
        sp = _SearchParam(seed, lig_uid, nchain, mc_steps, opt_steps, int(randomize))
        X = self._pose(olig, pose["coords"], pose["center"], pose["rot_vec"], pose["dihedrals"], 999.0)
        O = self._pose(olig, pose["coords"], pose["center"], pose["rot_vec"], pose["dihedrals"], 999.0)
        n = self.lib.orc_mc_chain(C.byref(olig.s), C.byref(env), C.byref(sp), chain, C.byref(X), C.byref(O))
        return self._unpose(O, olig), int(n)

    def randomize(self, olig, env, pose: dict, seed: int, lig_uid: int, chain: int, nchain: int) -> dict:
        sp = _SearchParam(seed, lig_uid, nchain, 0, 0, 1)
        X = self._pose(olig, pose["coords"], pose["center"], pose["rot_vec"], pose["dihedrals"], 999.0)
        self.lib.orc_randomize(C.byref(olig.s), C.byref(env), C.byref(sp), chain, C.byref(X))
        return self._unpose(X, olig)

    def cluster(self, types, coords: np.ndarray, energies: np.ndarray, rmsd_limit: float) -> List[int]:
        t = np.ascontiguousarray(types, np.int32)
        c = np.ascontiguousarray(coords, np.float32)
        e = np.ascontiguousarray(energies, np.float32)
        out = np.zeros(len(e), np.int32)
        n = self.lib.orc_cluster(len(t), _p(t), len(e), _p(c), _p(e), rmsd_limit, _p(out))
        return out[:n].tolist()


def initial_pose(lig) -> dict:
    """The engine's starting pose for a ligand (task.cu:87-105)."""
    return dict(energy=999.0, center=lig.center.astype(np.float64), rot_vec=np.zeros(3),
                coords=lig.coords.astype(np.float64), dihedrals=lig.dihedrals.astype(np.float64))
