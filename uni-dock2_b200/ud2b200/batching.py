"""Ligand size groups, batches and the opt_steps heuristic of the reference screen, and
the memory-bounded launches of this engine.

The reference groups ligands by (atoms, torsions) into small <=40/8, medium <=80/16,
large <=120/24, extra <=160/32 and overflow (src/screening/screening.h:19-30,
screening.cpp:17-41), processes each group in batches of at most 1000 ligands that also
fit its predicted device memory (predict_gpu_flex, screening.cpp:53-127,162-216; the
budget is 95 % of the free device memory, capped by max_gpu_mem, core.cpp:32-63) and,
when opt_steps is -1, resolves it once, from the first batch, as (25 + max atoms in that
batch) / 3 (screening.cpp:206-208).

This engine keeps a chain's search state in shared memory, so a ligand needs far less
device memory than in the reference; it runs many of the reference's batches in one
persistent launch.  ``plan_launches`` merges consecutive batches of one size group while the
launch's predicted device memory (``predict_dock_bytes``) stays within the budget; the
output files and the opt_steps rule still follow the reference's batches.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

GROUP_LIMITS = [(40, 8), (80, 16), (120, 24), (160, 32)]
BATCH_MAX = 1000


def size_groups(natoms: Sequence[int], ntors: Sequence[int]) -> List[List[int]]:
    """Ligand indices per size group, in input order (the first group a ligand fits)."""
    na = np.asarray(natoms, np.int64).reshape(-1)
    nt = np.asarray(ntors, np.int64).reshape(-1)
    gid = np.full(na.shape, len(GROUP_LIMITS), np.int64)
    for gi in reversed(range(len(GROUP_LIMITS))):
        ma, mt = GROUP_LIMITS[gi]
        gid[(na <= ma) & (nt <= mt)] = gi
    return [np.nonzero(gid == g)[0].tolist() for g in range(len(GROUP_LIMITS) + 1)]


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


# per-chain bytes of the learned search beyond the records: the feature row (672 BF16) and
# the network's activations (x, 3 hidden, delta in BF16; output, its gradient, 2 hidden
# gradients in FP32; ud_mlp_host.cuh MlpState::ensure)
_LEARNED_CHAIN_BYTES = 672 * 2 + 672 * 2 + 3 * 256 * 2 + 256 * 2 + 2 * 64 * 4 + 2 * 256 * 4


def record_floats(natom, ntors):
    """Floats of one pose record, padded to 16 bytes (8 + 3N + T, ud_engine.cu rec_floats)."""
    v = 8 + 3 * np.asarray(natom, np.int64) + np.asarray(ntors, np.int64)
    return (v + 3) // 4 * 4


def predict_dock_bytes(natom, ntors, npairs, nrot, nrange, nbias, nchain: int, retain: int = 1, num_pose: int = 10,
                       learned: bool = False, decomp: bool = False) -> np.ndarray:
    """Device bytes one ligand adds to a dock launch (an upper bound): its topology blob
    (every section padded to 4 words), chain records (and the learned search's accepted
    poses, features and network activations), clustering and output buffers."""
    n = np.asarray(natom, np.int64)
    t = np.asarray(ntors, np.int64)
    p = np.asarray(npairs, np.int64)
    stride = record_floats(n, t)
    blob = 4 * (64 + 96 + 13 * n + 7 * t + 2 * np.asarray(nrange, np.int64) + 2 * np.asarray(nrot, np.int64)
                + 5 * np.asarray(nbias, np.int64) + 3 * p)
    chains = nchain * retain
    rec = 4 * chains * stride
    b = blob + rec + 4 * chains + 64 + 16 * nchain                      # records, leaders, ligand entry, items
    b += num_pose * (4 * stride + 4 + 16 + 24) + (20 * n * num_pose if decomp else 0)
    if learned:
        b += 4 * nchain * stride + nchain * _LEARNED_CHAIN_BYTES
    return b


def memory_budget(free_bytes: int, max_gpu_mem_mb: int = 0, host_bytes: int = 0) -> int:
    """Bytes a launch may use: 95 % of the free device memory, capped by the host memory
    and by max_gpu_mem (MB) when given (core.cpp:32-63)."""
    lim = int(0.95 * free_bytes)
    if host_bytes > 0:
        lim = min(lim, int(0.95 * host_bytes))
    if max_gpu_mem_mb > 0:
        lim = min(lim, int(max_gpu_mem_mb) << 20)
    return lim


def reference_batches(natoms: Sequence[int], ntors: Sequence[int], batch_max: int = BATCH_MAX):
    """The reference's batches with the size group of each: [(group, [ligands])]."""
    out = []
    for gi, g in enumerate(size_groups(natoms, ntors)):
        for s0 in range(0, len(g), batch_max):
            out.append((gi, g[s0:s0 + batch_max]))
    return out


def plan_launches(ref_batches, per_ligand_bytes, budget: int) -> List[List[int]]:
    """Launches (lists of ligand indices): consecutive ligands of one size group, in the
    reference's batch order, as many as fit `budget` together.  A launch may span several
    reference batches and a reference batch several launches.  Raises MemoryError when one
    ligand alone does not fit (the reference's "Not enough GPU Memory" check,
    screening.cpp:197)."""
    out: List[List[int]] = []
    cur: List[int] = []
    used = 0
    group = None
    for gi, b in ref_batches:
        if gi != group and cur:
            out.append(cur)
            cur, used = [], 0
        group = gi
        for i in b:
            need = int(per_ligand_bytes[i])
            if need > budget:
                raise MemoryError(f"not enough device memory for ligand {i}: {need >> 20} MB needed, "
                                  f"{budget >> 20} MB available")
            if cur and used + need > budget:
                out.append(cur)
                cur, used = [], 0
            cur.append(i)
            used += need
    if cur:
        out.append(cur)
    return out
