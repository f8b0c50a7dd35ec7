import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "uni-dock2_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libudock_b200.so")


@pytest.fixture(scope="session")
def oracle64():
    import oracle as O
    O.build()
    return O.Oracle("f64")


@pytest.fixture(scope="session")
def oracle32():
    import oracle as O
    O.build()
    return O.Oracle("f32")


@pytest.fixture(scope="session")
def small_system():
    """A small seeded receptor (600 atoms, 28 A cube, the density of the 2000-atom
    40 A benchmark receptor) and a few ligands of mixed size."""
    from ud2b200 import synth
    from ud2b200.model import Box, parse_ligands, parse_receptor
    rows, center = synth.make_receptor(600, 28.0, seed=3)
    box = Box.from_center_size(center, [20.0, 20.0, 20.0])
    rec = parse_receptor(rows, box)
    ligd = {}
    for i, (n, t) in enumerate([(8, 0), (14, 2), (20, 4), (30, 6), (41, 9)]):
        ligd[f"l{i}"] = synth.make_ligand(n, t, seed=100 + i, center=center)
    ligs = parse_ligands(ligd)
    return dict(rows=rows, center=center, box=box, rec=rec, ligs=ligs, ligd=ligd)


def random_poses(lig, box, rng, n, spread=0.6):
    """Rigidly rotated/translated copies of a ligand, with random torsion moves applied
    through the oracle's kinematics elsewhere; here only rigid moves inside the box."""
    from scipy.spatial.transform import Rotation as Rot
    out = []
    c0 = lig.coords.mean(axis=0)
    lo = box.lo + 2.0
    hi = box.hi - 2.0
    for _ in range(n):
        R = Rot.random(random_state=rng).as_matrix()
        t = lo + (hi - lo) * rng.random(3)
        x = (lig.coords - c0) @ R.T + t
        out.append(x.astype(np.float32))
    return out
