"""Training the learned move proposal from the plain engine's own search.

The network (C ABI `ud_mlp_*`) learns, from poses the plain search visits on a set of
training ligands, the move from each pose to its ligand's best pose found by the run
(`collect_moves(target=1)`), or to the next accepted pose (target 0).  Collection, training
(forward, backward and Adam kernels) and inference all run on the GPU; parameters are a
flat float32 vector that can be saved with numpy and loaded into any engine.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from .engine import Engine
from .model import Box, Ligand, Receptor


@dataclass
class TrainReport:
    samples: List[int] = field(default_factory=list)
    collect_s: float = 0.0
    train_s: float = 0.0
    epoch_loss: List[float] = field(default_factory=list)


def train_proposal(box: Box, rec: Receptor, ligand_sets: Sequence[Sequence[Ligand]], map_types: Sequence[int],
                   opt_steps: int, nchain: int = 128, mc_steps: int = 150, target: int = 1, epochs: int = 6,
                   batch: int = 1024, lr: float = 1e-3, seed: int = 1, spacing: float = 0.375,
                   max_moves: int = 1_500_000, device: int = 0):
    """One plain search over the union of the training ligand sets records up to max_moves
    poses with their targets on the device; a freshly initialised network is trained on
    them there.  Returns (params, TrainReport)."""
    rep = TrainReport()
    eng = Engine(box, device=device)
    try:
        eng.set_receptor(rec.xyz, rec.types)
        eng.build_grid(spacing, list(map_types))
        eng.add_ligands([l for ligs in ligand_sets for l in ligs])
        t = time.perf_counter()
        n = eng.collect_moves(seed=seed, nchain=nchain, mc_steps=mc_steps, opt_steps=opt_steps, max_moves=max_moves,
                              target=target)
        rep.collect_s = time.perf_counter() - t
        rep.samples.append(n)
        eng.mlp_init(seed)
        t = time.perf_counter()
        rep.epoch_loss = [float(v) for v in eng.mlp_train_moves(epochs=epochs, batch=batch, lr=lr, seed=seed)]
        rep.train_s = time.perf_counter() - t
        params = eng.mlp_get_params()
    finally:
        eng.close()
    return params, rep


def save_params(path: str, params: np.ndarray) -> None:
    np.save(path, np.asarray(params, np.float32))


def load_params(path: str) -> np.ndarray:
    return np.load(path).astype(np.float32)
