"""The multi-GPU path of bench.py on CPU: two gloo ranks shard the ligands (disjoint
ligands in every fresh batch, the same receptor) and reduce the timings (max over ranks,
ligands summed)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import hashlib
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "uni-dock2_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import bench
        w, box, rec, ligs = bench.make_inputs("small", 3, 1, rank)
        center = (box.lo.astype(np.float64) + box.hi) / 2.0
        # the timed steps' fresh batches, as run_ours builds them on each rank
        pool = [bench.ligand_batch("small", 3, 1000 + 11 * (j + 1), rank, center) for j in range(2)]
        names = [l.name for l in ligs] + [l.name for b in pool for l in b]
        rec_sum = hashlib.sha1(np.ascontiguousarray(rec.xyz).tobytes()).hexdigest()
        gathered = [None] * world
        dist.all_gather_object(gathered, (names, rec_sum))
        dev_ms, e2e_s, n = bench.reduce_over_ranks(dist, 100.0 * (rank + 1), 1.0 + rank, len(ligs), "cpu")
        if rank == 0:
            out.put((gathered, dev_ms, e2e_s, n))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, dev_ms, e2e_s, n = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (names0, rec0), (names1, rec1) = gathered
    assert rec0 == rec1                                  # every rank docks against the same receptor
    assert not set(names0) & set(names1)                 # ligand shards are disjoint
    assert len(names0) == len(names1) == 9
    assert dev_ms == 200.0 and e2e_s == 2.0 and n == 6   # slowest rank's times, all ranks' ligands
