"""Ligand size groups, batches and the opt_steps heuristic of the reference screen.

The reference groups ligands by (atoms, torsions) into small <=40/8, medium <=80/16,
large <=120/24, extra <=160/32 and overflow (src/screening/screening.h:19-30,
screening.cpp:17-41), processes each group in batches of at most 1000 ligands
(screening.cpp:162-216) and, when opt_steps is -1, resolves it once, from the first
batch, as (25 + max atoms in that batch) / 3 (screening.cpp:206-208).
"""
from __future__ import annotations

from typing import List, Sequence

GROUP_LIMITS = [(40, 8), (80, 16), (120, 24), (160, 32)]
BATCH_MAX = 1000


def size_groups(natoms: Sequence[int], ntors: Sequence[int]) -> List[List[int]]:
    groups: List[List[int]] = [[] for _ in range(len(GROUP_LIMITS) + 1)]
    for i, (na, nt) in enumerate(zip(natoms, ntors)):
        for gi, (ma, mt) in enumerate(GROUP_LIMITS):
            if na <= ma and nt <= mt:
                groups[gi].append(i)
                break
        else:
            groups[-1].append(i)
    return groups


def batches(natoms: Sequence[int], ntors: Sequence[int], batch_max: int = BATCH_MAX) -> List[List[int]]:
    out = []
    for g in size_groups(natoms, ntors):
        for s in range(0, len(g), batch_max):
            out.append(g[s:s + batch_max])
    return out


def heuristic_opt_steps(natoms: Sequence[int], ntors: Sequence[int]) -> int:
    """opt_steps for opt_steps == -1: from the first batch, kept for all batches."""
    b = batches(natoms, ntors)
    if not b:
        return 0
    return (25 + max(natoms[i] for i in b[0])) // 3
