"""Shared helpers for the GPU parity tests (engine on cuda:0 vs the CPU oracle)."""
import math

import numpy as np

MAP_TYPES_ALL = [2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14, 15, 16, 17, 18]


def map_types_for(ligs):
    ts = sorted(set(int(t) for l in ligs for t in l.types if t != 0))
    return ts


def engine_for(system, spacing=0.375, precision=0):
    from ud2b200 import Engine
    eng = Engine(system["box"])
    rows = np.asarray([r[:4] for r in system["rows"]], np.float64)
    eng.set_receptor(rows[:, :3].astype(np.float32), rows[:, 3].astype(np.int32))
    mt = map_types_for(system["ligs"])
    eng.build_grid(spacing, mt, precision)
    eng.add_ligands(system["ligs"])
    return eng, mt


def oracle_grid(oracle, system, eng):
    maps, gd, org = eng.get_grid()
    mt = eng.map_types
    omaps = oracle.grid_build(system["rec"], mt, org.astype(np.float64), 0.375, gd)
    mot = -np.ones(24, np.int32)
    for i, t in enumerate(mt):
        mot[t] = i
    return dict(maps=omaps, map_of_type=mot, origin=org.astype(np.float64), spacing=0.375, gdim=gd), maps


def perturbed_poses(oracle, olig, env, lig, rng, n, box):
    """Random poses: random torsion increments through the oracle kinematics, then a
    random rigid placement inside the box; rot_vec random (it is pose state)."""
    from scipy.spatial.transform import Rotation as Rot
    poses = []
    for _ in range(n):
        pose = dict(coords=lig.coords.astype(np.float64), center=lig.center.astype(np.float64),
                    rot_vec=np.zeros(3), dihedrals=lig.dihedrals.astype(np.float64))
        g = np.zeros(6 + lig.ntors)
        g[6:] = rng.uniform(-math.pi, math.pi, lig.ntors)
        if lig.ntors:
            pose = oracle.apply_update(olig, env, pose, g, 1.0)
        X = pose["coords"]
        c = X.mean(axis=0)
        R = Rot.random(random_state=rng).as_matrix()
        mid = (box.lo + box.hi) / 2.0
        t = mid + rng.uniform(-3.0, 3.0, 3)
        X = (X - c) @ R.T + t
        rv = rng.uniform(-1.5, 1.5, 3)
        poses.append(dict(coords=X.astype(np.float32), center=X.astype(np.float32).mean(axis=0), rot_vec=rv.astype(np.float32),
                          dihedrals=pose["dihedrals"].astype(np.float32)))
    return poses


def rel_err(a, b, floor=1.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(floor, float(np.max(np.abs(b)))))
