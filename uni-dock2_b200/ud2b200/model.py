"""Host data model: receptor and ligand topology, parsed from the engine's input schema.

The input schema is the one the reference engine's pybind ``pipeline`` consumes
(``unidock/unidock_engine/src/format/rapidjson_parser.cpp:25-225``):

* receptor rows ``[x, y, z, vina_type, ff_type, charge]``;
* ligand ``{"atoms": [[x,y,z,vt,fft,q,[1-2/1-3 idx],[1-4 idx](,[[bx,by,bz,V,r2],...])], ...],
  "torsions": [[[a,b,c,d], value_deg, [[lo,hi],...], [rotated idx], [gaff2...]], ...],
  "root_atoms": [...]}``.

Parsing restates the reference's semantics: hydrogens are dropped from the receptor
and only atoms inside the box grown by the 8 A Vina cutoff are kept
(``json.cpp:58-65``, ``rapidjson_parser.cpp:25-52``); the ligand intra pair list
excludes 1-2/1-3 pairs, 1-4 pairs and pairs inside one rigid fragment
(``rapidjson_parser.cpp:88-111, 201-221, 227-296``).  Angles are converted with the
reference's single-precision ``DEG2RAD = 3.1415927f / 180`` (``myutils/common.h:44-47``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

F32 = np.float32
PI_F = F32(3.1415927)
DEG2RAD_F = F32(PI_F / F32(180.0))
RAD2DEG_F = F32(F32(180.0) / PI_F)
VINA_CUTOFF = 8.0
VN_TYPE_H = 0
NUM_VN_TYPES = 21

# src/constants/constants.h:21-43
VDW_RADII = np.array([1.1, 1.92, 1.9, 1.9, 1.8, 1.8, 1.8, 1.8, 1.7, 1.7, 1.7,
                      1.7, 1.5, 2.2, 2.1, 2.0, 1.8, 2.0, 2.2, 2.3, 1.2], dtype=np.float64)


@dataclass
class Box:
    """Docking box; ligand heavy atoms outside it pay the box penalty (model.h:131-143)."""
    lo: np.ndarray
    hi: np.ndarray

    @staticmethod
    def from_center_size(center: Sequence[float], size: Sequence[float]) -> "Box":
        # the reference computes the bounds in Real (float): pipeline.cpp:88-93
        c = np.asarray(center, dtype=F32)
        s = np.asarray(size, dtype=F32)
        return Box(lo=(c - s / F32(2)).astype(F32), hi=(c + s / F32(2)).astype(F32))

    def as6(self) -> np.ndarray:
        return np.array([self.lo[0], self.hi[0], self.lo[1], self.hi[1], self.lo[2], self.hi[2]], dtype=F32)


@dataclass
class Receptor:
    xyz: np.ndarray          # (M, 3) float32, heavy atoms inside box +- 8 A
    types: np.ndarray        # (M,) int32 XS types
    ff_types: np.ndarray
    charges: np.ndarray

    @property
    def natom(self) -> int:
        return int(self.xyz.shape[0])


def parse_receptor(rows: Sequence[Sequence[float]], box: Box) -> Receptor:
    """Receptor rows -> heavy atoms inside box +- 8 A (rapidjson_parser.cpp:25-52)."""
    if len(rows) == 0:
        z = np.zeros((0,), np.int32)
        return Receptor(np.zeros((0, 3), F32), z, z.copy(), np.zeros((0,), F32))
    arr = np.asarray([r[:6] for r in rows], dtype=np.float64)
    xyz = arr[:, :3].astype(F32)
    types = arr[:, 3].astype(np.int32)
    lo = box.lo.astype(F32) - F32(VINA_CUTOFF)
    hi = box.hi.astype(F32) + F32(VINA_CUTOFF)
    inside = np.all((xyz >= lo) & (xyz <= hi), axis=1)
    keep = (types != VN_TYPE_H) & inside
    return Receptor(xyz=np.ascontiguousarray(xyz[keep]), types=np.ascontiguousarray(types[keep]),
                    ff_types=arr[keep, 4].astype(np.int32), charges=arr[keep, 5].astype(F32))


@dataclass
class Ligand:
    name: str
    coords: np.ndarray                 # (N, 3) float32
    types: np.ndarray                  # (N,) int32
    ff_types: np.ndarray
    charges: np.ndarray
    axis: np.ndarray                   # (T, 2) int32 (from, to) = torsion atoms[1], atoms[2]
    dihedrals: np.ndarray              # (T,) float32 radians
    ranges: List[np.ndarray]           # T arrays (n_k, 2) float32 radians
    rotated: List[np.ndarray]          # T arrays of rotated atom indices
    pair_off: np.ndarray               # (N+1,) int32 per-atom intra adjacency CSR
    pairs: np.ndarray                  # int32 neighbour indices (both directions)
    bias_atoms: np.ndarray = field(default_factory=lambda: np.zeros((0,), np.int32))
    bias_params: np.ndarray = field(default_factory=lambda: np.zeros((0, 5), F32))
    n_pairs_1213: int = 0
    n_pairs_14: int = 0

    @property
    def natom(self) -> int:
        return int(self.coords.shape[0])

    @property
    def ntors(self) -> int:
        return int(self.axis.shape[0])

    @property
    def n_heavy(self) -> int:
        return int(np.count_nonzero(self.types != VN_TYPE_H))

    @property
    def center(self) -> np.ndarray:
        # rapidjson_parser.cpp:67-83,197-199: float sums divided by natom
        s = np.zeros(3, F32)
        for row in self.coords:
            s = (s + row).astype(F32)
        return (s / F32(self.natom)).astype(F32)

    def bias_csr(self) -> Tuple[np.ndarray, np.ndarray]:
        """Per-atom offsets (records) into bias params, ordered by atom."""
        order = np.argsort(self.bias_atoms, kind="stable")
        counts = np.bincount(self.bias_atoms, minlength=self.natom) if self.bias_atoms.size else np.zeros(self.natom, np.int64)
        off = np.zeros(self.natom + 1, np.int32)
        off[1:] = np.cumsum(counts)
        return off, np.ascontiguousarray(self.bias_params[order].astype(F32))


def _order_pair(a: int, b: int) -> Tuple[int, int]:
    return (a, b) if a < b else (b, a)


def split_torsions_into_frags(root: set, axis: np.ndarray, rotated: List[np.ndarray]) -> List[set]:
    """Rigid fragments from the torsion tree (rapidjson_parser.cpp:227-296)."""
    frag0 = set(root)
    rest = list(range(len(rotated)))
    frags: List[set] = []
    for k in range(len(rotated)):
        a0, a1 = int(axis[k, 0]), int(axis[k, 1])
        if a0 in root or a1 in root:
            rest.remove(k)
            frag0.add(a0)
            frag0.add(a1)
            f = set(int(i) for i in rotated[k])
            f.add(a0)
            f.add(a1)
            frags.append(f)
    frags.append(frag0)
    for k in rest:
        a0, a1 = int(axis[k, 0]), int(axis[k, 1])
        tor = set(int(i) for i in rotated[k])
        for fi, frag in enumerate(frags):
            if a0 in frag and a1 in frag:
                f1 = (frag & tor) | {a0, a1}
                f2 = (frag - tor) | {a0, a1}
                frags[fi] = f1
                frags.append(f2)
                break
    return frags


def build_intra_pairs(natom: int, pairs_1213: set, pairs_14: set, frags: List[set]) -> Tuple[np.ndarray, np.ndarray]:
    """Per-atom adjacency of scored intra pairs (rapidjson_parser.cpp:201-221)."""
    member = np.zeros((len(frags), natom), dtype=bool)
    for fi, f in enumerate(frags):
        for a in f:
            if 0 <= a < natom:
                member[fi, a] = True
    excl = np.zeros((natom, natom), dtype=bool)
    for (a, b) in pairs_1213:
        if a < natom and b < natom:
            excl[a, b] = excl[b, a] = True
    for (a, b) in pairs_14:
        if a < natom and b < natom:
            excl[a, b] = excl[b, a] = True
    if len(frags):
        same = (member.T.astype(np.int32) @ member.astype(np.int32)) > 0
        excl |= same
    neigh: List[List[int]] = [[] for _ in range(natom)]
    iu, ju = np.triu_indices(natom, k=1)
    ok = ~excl[iu, ju]
    for i, j in zip(iu[ok].tolist(), ju[ok].tolist()):
        neigh[i].append(j)
        neigh[j].append(i)
    # the reference appends j to i's list in increasing (i, j) loop order: for a fixed
    # atom the neighbours below it come first (from earlier i), then those above it
    for i in range(natom):
        neigh[i].sort()
    off = np.zeros(natom + 1, np.int32)
    off[1:] = np.cumsum([len(n) for n in neigh])
    flat = np.asarray([j for n in neigh for j in n], dtype=np.int32)
    return off, flat


def parse_ligand(name: str, obj: dict, use_tor_lib: bool = False) -> Ligand:
    """One ligand of the input schema (rapidjson_parser.cpp:54-225)."""
    atoms = obj["atoms"]
    n = len(atoms)
    coords = np.asarray([a[:3] for a in atoms], dtype=F32).reshape(n, 3)
    types = np.asarray([int(a[3]) for a in atoms], dtype=np.int32)
    ff = np.asarray([int(a[4]) for a in atoms], dtype=np.int32)
    q = np.asarray([a[5] for a in atoms], dtype=F32)
    p1213: set = set()
    p14: set = set()
    b_atoms: List[int] = []
    b_params: List[List[float]] = []
    for ia, a in enumerate(atoms):
        for ib in a[6]:
            ib = int(ib)
            if ib != ia:
                p1213.add(_order_pair(ia, ib))
        for ib in a[7]:
            ib = int(ib)
            if ib != ia:
                p = _order_pair(ia, ib)
                if p not in p1213:
                    p14.add(p)
        if len(a) > 8:
            for bl in a[8]:
                b_atoms.append(ia)
                b_params.append([float(v) for v in bl[:5]])
    root = set(int(i) for i in obj.get("root_atoms", []))
    tors = obj.get("torsions", [])
    T = len(tors)
    axis = np.zeros((T, 2), np.int32)
    dihe = np.zeros((T,), F32)
    ranges: List[np.ndarray] = []
    rotated: List[np.ndarray] = []
    for k, t in enumerate(tors):
        four = [int(v) for v in t[0]]
        axis[k] = (four[1], four[2])
        dihe[k] = F32(F32(t[1]) * DEG2RAD_F)
        rl: List[Tuple[float, float]] = []
        if use_tor_lib:
            for r in t[2]:
                lo = F32(F32(r[0]) * DEG2RAD_F)
                hi = F32(F32(r[1]) * DEG2RAD_F)
                if lo < hi:
                    rl.append((lo, hi))
                elif lo > 0 and hi < 0:
                    rl.append((lo, PI_F))
                    rl.append((-PI_F, hi))
        else:
            rl.append((-PI_F, PI_F))
        if not rl:
            rl.append((-PI_F, PI_F))
        ranges.append(np.asarray(rl, dtype=F32).reshape(-1, 2))
        rotated.append(np.asarray([int(v) for v in t[3]], dtype=np.int32))
    frags = split_torsions_into_frags(root, axis, rotated)
    off, flat = build_intra_pairs(n, p1213, p14, frags)
    return Ligand(name=name, coords=coords, types=types, ff_types=ff, charges=q, axis=axis,
                  dihedrals=dihe, ranges=ranges, rotated=rotated, pair_off=off, pairs=flat,
                  bias_atoms=np.asarray(b_atoms, np.int32),
                  bias_params=np.asarray(b_params, F32).reshape(-1, 5),
                  n_pairs_1213=len(p1213), n_pairs_14=len(p14))


def parse_ligands(ligands: Dict[str, dict], use_tor_lib: bool = False) -> List[Ligand]:
    """All ligands of an input dict, skipping the reserved keys (rapidjson_parser.cpp:55-64)."""
    out = []
    for k, v in ligands.items():
        if k in ("score", "receptor"):
            continue
        out.append(parse_ligand(k, v, use_tor_lib))
    return out
