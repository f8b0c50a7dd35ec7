"""Seeded synthetic receptors and ligands in the engine's input schema.

The docking benchmark workloads are defined on synthetic inputs (no public dataset
is used by the engine for performance).  Everything here is generated from a seed;
the same dicts feed this engine and, through ``json``, the reference engine.

Receptor: heavy atoms rejection-sampled uniformly in a cube with a minimum spacing
of 2.8 A and an empty spherical pocket of radius 8 A at the centre.  Element mix
C 62 % (C_H / C_P 50/50), N 17 % (N_D 95 %, N_P 4 %, N_A 1 %), O 19 % (O_A 86 %,
O_DA 14 %), S 2 % (S_P), the donor/acceptor split taken from the reference's 1W1P
fixture's type histogram.

Ligand: a random-walk tree (1.5 A bonds, 109.5 degree angles, random dihedrals,
no pair beyond 1-3 closer than 2.5 A), C/N/O at 70/15/15 %, typed with the XS rules
of the reference's processing package (C bonded to N/O is C_P else C_H; N is N_D
or N_A; O is O_A).  Rotatable bonds are a random subset of non-terminal tree edges;
the root is the largest rigid fragment; 1-2/1-3 and 1-4 lists come from graph
distances, the same semantics as the reference's topology builder.
"""
from __future__ import annotations

import math
from collections import deque
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# XS types (src/constants/constants.h:48-68)
C_H, C_P, N_P, N_D, N_A, O_A, O_DA, S_P = 2, 3, 4, 5, 6, 10, 11, 15


def make_receptor(natom: int, cube: float, seed: int, pocket_radius: float = 8.0,
                  min_dist: float = 2.8) -> Tuple[List[list], np.ndarray]:
    """Receptor rows [x,y,z,type,0,0.0] and the pocket centre."""
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0x7EC]))
    center = np.full(3, cube / 2.0)
    cell = min_dist
    ncell = int(math.ceil(cube / cell)) + 1
    grid: Dict[Tuple[int, int, int], List[int]] = {}
    pts = np.zeros((natom, 3))
    n = 0
    attempts = 0
    md2 = min_dist * min_dist
    while n < natom:
        attempts += 1
        if attempts > 400 * natom:
            raise RuntimeError("receptor rejection sampling did not converge")
        p = rng.uniform(0.0, cube, size=3)
        if np.sum((p - center) ** 2) < pocket_radius * pocket_radius:
            continue
        ci = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((ci[0] + dx, ci[1] + dy, ci[2] + dz), ()):
                        d = pts[j] - p
                        if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < md2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        pts[n] = p
        grid.setdefault(ci, []).append(n)
        n += 1
    u = rng.random(natom)
    v = rng.random(natom)
    types = np.empty(natom, np.int32)
    for i in range(natom):
        if u[i] < 0.62:
            types[i] = C_H if v[i] < 0.5 else C_P
        elif u[i] < 0.79:
            types[i] = N_D if v[i] < 0.95 else (N_P if v[i] < 0.99 else N_A)
        elif u[i] < 0.98:
            types[i] = O_A if v[i] < 0.86 else O_DA
        else:
            types[i] = S_P
    rows = [[float(pts[i, 0]), float(pts[i, 1]), float(pts[i, 2]), int(types[i]), 0, 0.0]
            for i in range(natom)]
    return rows, center


def _perp(v: np.ndarray) -> np.ndarray:
    a = np.array([1.0, 0.0, 0.0]) if abs(v[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    p = np.cross(v, a)
    return p / np.linalg.norm(p)


def _grow_tree(n: int, rng: np.random.Generator, core: Optional[Tuple[np.ndarray, List[Tuple[int, int]]]] = None,
               bond: float = 1.5, angle_deg: float = 109.5, clash: float = 2.5):
    """Random-walk tree; returns coords (n,3) and bond list."""
    ang = math.radians(angle_deg)
    if core is not None:
        xyz = [c.copy() for c in core[0]]
        bonds = list(core[1])
    else:
        xyz = [np.zeros(3)]
        bonds = []
    nbr: List[List[int]] = [[] for _ in range(n)]
    for a, b in bonds:
        nbr[a].append(b)
        nbr[b].append(a)
    start = len(xyz)
    for i in range(start, n):
        placed = False
        for _ in range(400):
            cands = [j for j in range(i) if len(nbr[j]) < 3]
            if not cands:
                cands = [j for j in range(i) if len(nbr[j]) < 4]
            # favour recently added atoms so the walk extends
            w = np.arange(1, len(cands) + 1, dtype=float) ** 2
            par = cands[int(rng.choice(len(cands), p=w / w.sum()))]
            if nbr[par]:
                gp = nbr[par][0]
                u = xyz[par] - xyz[gp]
                u /= np.linalg.norm(u)
                p1 = _perp(u)
                p2 = np.cross(u, p1)
                phi = rng.uniform(0, 2 * math.pi)
                d = math.cos(math.pi - ang) * u + math.sin(math.pi - ang) * (math.cos(phi) * p1 + math.sin(phi) * p2)
            else:
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
            p = xyz[par] + bond * d
            # distance check against atoms further than 1-3 in the graph
            near = {par}
            near.update(nbr[par])
            ok = True
            for j in range(i):
                if j in near:
                    continue
                if np.sum((xyz[j] - p) ** 2) < clash * clash:
                    ok = False
                    break
            if ok:
                xyz.append(p)
                bonds.append((par, i))
                nbr[par].append(i)
                nbr[i].append(par)
                placed = True
                break
        if not placed:
            raise RuntimeError("ligand growth failed")
    return np.asarray(xyz), bonds


def _graph_dist(n: int, bonds: List[Tuple[int, int]]) -> np.ndarray:
    nbr: List[List[int]] = [[] for _ in range(n)]
    for a, b in bonds:
        nbr[a].append(b)
        nbr[b].append(a)
    D = np.full((n, n), 99, np.int32)
    for s in range(n):
        D[s, s] = 0
        q = deque([s])
        while q:
            u = q.popleft()
            for v in nbr[u]:
                if D[s, v] == 99:
                    D[s, v] = D[s, u] + 1
                    q.append(v)
    return D


def _dihedral_deg(a, b, c, d) -> float:
    b0 = a - b
    b1 = c - b
    b2 = d - c
    b1n = b1 / np.linalg.norm(b1)
    v = b0 - np.dot(b0, b1n) * b1n
    w = b2 - np.dot(b2, b1n) * b1n
    x = np.dot(v, w)
    y = np.dot(np.cross(b1n, v), w)
    return math.degrees(math.atan2(y, x))


def make_ligand(natom: int, ntors: int, seed: int, center: Sequence[float],
                core: Optional[dict] = None) -> dict:
    """One ligand dict in the engine input schema.

    ``core`` (optional) = {"xyz": (k,3) absolute coords, "bonds": [...], "elements": [...]}:
    the ligand then grows from that fixed rigid core, keeps the core's absolute
    placement, takes the core as its root, and its torsions are all outside the core.
    """
    for attempt in range(64):       # a random walk can box itself in: restart it
        rng = np.random.default_rng(np.random.SeedSequence([seed, 0x11C, attempt]))
        try:
            if core is not None:
                k = len(core["xyz"])
                xyz, bonds = _grow_tree(natom, rng, core=(np.asarray(core["xyz"], float), list(core["bonds"])))
                elem = list(core["elements"]) + [None] * (natom - k)
            else:
                k = 0
                xyz, bonds = _grow_tree(natom, rng)
                elem = [None] * natom
            break
        except RuntimeError:
            continue
    else:
        raise RuntimeError("ligand growth failed")
    for i in range(natom):
        if elem[i] is None:
            r = rng.random()
            elem[i] = "C" if r < 0.70 else ("N" if r < 0.85 else "O")
    nbr: List[List[int]] = [[] for _ in range(natom)]
    for a, b in bonds:
        nbr[a].append(b)
        nbr[b].append(a)
    types = []
    for i in range(natom):
        e = elem[i]
        if e == "C":
            types.append(C_P if any(elem[j] in ("N", "O") for j in nbr[i]) else C_H)
        elif e == "N":
            types.append(N_D if rng.random() < 0.3 else N_A)
        else:
            types.append(O_A)
    # rotatable bonds: non-terminal edges, outside the core
    cand = [(a, b) for (a, b) in bonds if len(nbr[a]) > 1 and len(nbr[b]) > 1 and not (a < k and b < k)]
    T = min(ntors, len(cand))
    rot_idx = sorted(rng.choice(len(cand), size=T, replace=False).tolist()) if T > 0 else []
    rot_bonds = [cand[i] for i in rot_idx]
    rotset = set(rot_bonds) | set((b, a) for a, b in rot_bonds)
    # rigid fragments = components after cutting rotatable bonds
    comp = [-1] * natom
    nc = 0
    for s in range(natom):
        if comp[s] >= 0:
            continue
        comp[s] = nc
        q = deque([s])
        while q:
            u = q.popleft()
            for v in nbr[u]:
                if comp[v] < 0 and (u, v) not in rotset:
                    comp[v] = nc
                    q.append(v)
        nc += 1
    if core is not None:
        root_c = comp[0]
    else:
        sizes = np.bincount(comp, minlength=nc)
        root_c = int(np.argmax(sizes))
    root_atoms = [i for i in range(natom) if comp[i] == root_c]
    rootset = set(root_atoms)
    torsions = []
    for (a, b) in rot_bonds:
        # orient: side containing the root stays, the other side rotates
        seen = {a}
        q = deque([b])
        side_b = {b}
        while q:
            u = q.popleft()
            for v in nbr[u]:
                if v not in seen and v not in side_b and not (u == b and v == a):
                    side_b.add(v)
                    q.append(v)
        if rootset & side_b:
            frm, to = b, a
            side = set(range(natom)) - side_b
        else:
            frm, to = a, b
            side = side_b
        i0 = [j for j in nbr[frm] if j != to][0]
        i3 = [j for j in nbr[to] if j != frm][0]
        val = _dihedral_deg(xyz[i0], xyz[frm], xyz[to], xyz[i3])
        torsions.append([[i0, frm, to, i3], val, [[-180.0, 180.0]], sorted(side), []])
    if core is None:
        xyz = xyz - xyz.mean(axis=0) + np.asarray(center, float)
    D = _graph_dist(natom, bonds)
    atoms = []
    for i in range(natom):
        p1213 = [int(j) for j in range(natom) if 1 <= D[i, j] <= 2]
        p14 = [int(j) for j in range(natom) if D[i, j] == 3]
        atoms.append([float(xyz[i, 0]), float(xyz[i, 1]), float(xyz[i, 2]), int(types[i]), 0, 0.0, p1213, p14])
    return {"atoms": atoms, "torsions": torsions, "root_atoms": root_atoms}


def make_core(center: Sequence[float], seed: int, k: int = 14) -> dict:
    """A fixed rigid core for template-constrained screens."""
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0xC02E]))
    xyz, bonds = _grow_tree(k, rng)
    xyz = xyz - xyz.mean(axis=0) + np.asarray(center, float)
    elem = ["C" if rng.random() < 0.7 else ("N" if rng.random() < 0.5 else "O") for _ in range(k)]
    return {"xyz": xyz, "bonds": bonds, "elements": elem}


# ---------------------------------------------------------------- workload configs
WORKLOADS = {
    # name: receptor atoms, cube edge, box edge, chains, mc_steps
    "small": dict(nrec=2000, cube=40.0, box=22.5, chains=64, mc_steps=2000, num_pose=9, rmsd=1.0),
    "screen": dict(nrec=4000, cube=40.0 * 2 ** (1 / 3), box=30.0, chains=128, mc_steps=4000, num_pose=9, rmsd=1.0),
    "uneven": dict(nrec=4000, cube=40.0 * 2 ** (1 / 3), box=30.0, chains=128, mc_steps=4000, num_pose=9, rmsd=1.0),
    "template": dict(nrec=4000, cube=40.0 * 2 ** (1 / 3), box=30.0, chains=256, mc_steps=2000, num_pose=1024, rmsd=2.0),
}


def ligand_sizes(workload: str, count: int, seed: int) -> List[Tuple[int, int]]:
    """(heavy atoms, rotatable bonds) per ligand for a workload."""
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0x5172E]))
    out = []
    for _ in range(count):
        if workload == "small":
            out.append((24, 5))
        elif workload == "screen":
            out.append((int(rng.integers(12, 49)), int(min(12, rng.poisson(5)))))
        elif workload == "uneven":
            n = int(np.clip(round(math.exp(rng.normal(math.log(28), 0.45))), 8, 80))
            out.append((n, int(rng.integers(0, 21))))
        elif workload == "template":
            out.append((int(rng.integers(15, 41)), int(rng.integers(1, 9))))
        else:
            raise ValueError(workload)
    return out


def make_workload(workload: str, nlig: int, seed: int = 0):
    """Receptor rows, ligand dict, pocket centre and search settings for a workload."""
    w = WORKLOADS[workload]
    rows, center = make_receptor(w["nrec"], w["cube"], seed)
    sizes = ligand_sizes(workload, nlig, seed)
    core = make_core(center, seed) if workload == "template" else None
    ligs = {}
    for i, (n, t) in enumerate(sizes):
        ligs[f"lig{i:06d}"] = make_ligand(n, t, seed * (1 << 32) + i, center, core=core)
    return rows, ligs, center, w
