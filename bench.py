"""Throughput benchmark of the docking engine on the plain virtual-screen workload:
ligands/s at a best-score gap of at most 0.3 kcal/mol to the plain 4000-step search for at
least 95 % of ligands; learned vs plain search.

Workload ("screen"): a 4000-atom synthetic receptor, ligands with 12-48 heavy atoms and
Poisson(5) rotatable bonds (clipped 0-12), a 30 A box with 0.375 A grid maps (81^3 x types),
128 MC chains per ligand with BFGS (opt_steps resolved by the -1 heuristic), 5 refinement
rounds of the cluster leaders, top-9 poses at RMSD 1.0 A, final scoring.  A step docks one
batch of ligands completely.  Inputs are seeded synthetic data.

Default (--mode learned): the plain fused engine docks the batch once at 4000 MC steps (the
reference result and the plain throughput); a proposal network is trained on the GPU from
the plain engine's searches of four other seeded ligand sets; the timed steps dock the batch
with the learned-proposal engine at --learned-steps MC steps.  `value` is the learned
engine's ligands/s, `quality` the share of ligands whose best score is within 0.3 kcal/mol of
the 4000-step result.  --mode plain times the fused 4000-step engine instead.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode learned|plain]

N > 1 runs under torchrun, one rank per GPU, each rank docking its own ligands (weak
scaling, no data-path collective); the timed region is bracketed by a barrier and
synchronisation and its time is the max over ranks.
"""
from __future__ import annotations

import argparse
import glob
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "uni-dock2_b200"))

METRIC = "ligands/s @ best-score within 0.3 kcal/mol of ref; learned vs plain search"
UNIT = "ligands/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--ref-ligands", type=int, default=8, help="ligands of the reference-gpu comparison")
    ap.add_argument("--ref-mc-steps", type=int, default=200, help="MC steps of the reference-gpu comparison")
    ap.add_argument("--workload", default="screen")
    ap.add_argument("--ligands", type=int, default=148, help="ligands per step per GPU")
    ap.add_argument("--mc-steps", type=int, default=0, help="override MC steps (0 = workload value)")
    ap.add_argument("--warmup-mc-steps", type=int, default=100,
                    help="MC steps per chain in the untimed warm-up steps (0 = as the timed steps)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--grid", default="f32", choices=["f32", "f16"])
    ap.add_argument("--mode", default="learned", choices=["learned", "plain"])
    ap.add_argument("--learned-steps", type=int, default=1000, help="MC steps of the learned-proposal engine")
    ap.add_argument("--p-learned", type=float, default=0.25, help="share of learned moves")
    ap.add_argument("--train-ligands", type=int, default=37, help="training ligands per seed (4 seeds)")
    ap.add_argument("--train-epochs", type=int, default=6, help="epochs of network training")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    return ap.parse_args()


# ------------------------------------------------------------------------- workload
def make_inputs(workload: str, nlig: int, seed: int, rank: int):
    import numpy as np
    from ud2b200 import synth
    from ud2b200.model import Box, parse_ligands, parse_receptor
    w = synth.WORKLOADS[workload]
    rows, center = synth.make_receptor(w["nrec"], w["cube"], seed)
    box = Box.from_center_size(center, [w["box"]] * 3)
    rec = parse_receptor(rows, box)
    sizes = synth.ligand_sizes(workload, nlig * (rank + 1), seed)[nlig * rank:]
    core = synth.make_core(center, seed) if workload == "template" else None
    ligd = {f"r{rank}_lig{i:05d}": synth.make_ligand(n, t, seed * 7919 + rank * 1000003 + i, center, core=core)
            for i, (n, t) in enumerate(sizes)}
    ligs = parse_ligands(ligd)
    return w, box, rec, ligs


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(summary: str = "k_search_screen.md"):
    """DRAM bytes (read + write) of one launch of the dominant kernel at the default batch
    (k_search, or k_learn_step: one MC step of every chain), from the committed ncu
    summary of that launch."""
    p = os.path.join(ROOT, "profiles", summary)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 4 + k and r[4 + k].lower().startswith("active"):
                    reasons.add(n)
        loaded = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------------------- CPU port
def cpu_port_rate(w, box, rec, ligs, mc_steps, opt_steps, seconds: float, mode: str = "direct"):
    """Chain-steps per second of the oracle's restatement of the reference search on all
    host cores (one chain per thread; the C calls release the GIL)."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    orc = O.Oracle("f32")
    env = orc.make_env(rec, box, mode=mode)
    cores = os.cpu_count() or 1
    sample = ligs[:cores]
    oligs = [orc.ligand(l) for l in sample]
    done_steps = 0
    t0 = time.perf_counter()
    steps = 1
    while True:
        def run(k):
            l = sample[k % len(sample)]
            pose = O.initial_pose(l)
            orc.mc_chain(oligs[k % len(sample)], env, pose, seed=11, lig_uid=k, chain=k, nchain=w["chains"],
                         mc_steps=steps, opt_steps=opt_steps, randomize=True)
            return steps
        ts = time.perf_counter()
        with ThreadPoolExecutor(max_workers=cores) as ex:
            done_steps += sum(ex.map(run, range(cores)))
        el = time.perf_counter() - t0
        if el >= seconds or steps >= mc_steps:
            break
        left = seconds - el
        per = (time.perf_counter() - ts) / steps
        steps = max(1, min(mc_steps, int(left / max(per, 1e-6))))
    el = time.perf_counter() - t0
    rate = done_steps / el
    return rate, cores, f"{done_steps} MC steps of {cores} chains (one per core) on {len(sample)} screen ligands, " \
                        f"{mode} scoring, in {el:.1f} s"


def reference_scoring_rate(rec, box, ligs, seconds: float = 8.0):
    """Poses scored per second by the reference's own host score() (src/score/score.cpp,
    compiled from the reference sources into oracle/_ref, OpenMP over poses on all host
    cores): energy of rigidly placed copies of the batch's first ligand.  None when that
    library was not built."""
    import ctypes as C
    import numpy as np
    path = os.path.join(ROOT, "oracle", "_ref", "libudref_f32.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    lig = ligs[0]
    rng = np.random.default_rng(5)
    npose = 2048
    mid = ((box.lo + box.hi) / 2.0).astype(np.float32)
    base = (lig.coords - lig.coords.mean(axis=0)).astype(np.float32)
    xs = np.ascontiguousarray(np.stack([base + mid + rng.uniform(-3, 3, 3).astype(np.float32) for _ in range(npose)]),
                              np.float32)
    types = np.ascontiguousarray(lig.types, np.int32)
    off = np.ascontiguousarray(lig.pair_off, np.int32)
    pairs = np.ascontiguousarray(lig.pairs, np.int32)
    rxyz = np.ascontiguousarray(rec.xyz, np.float32)
    rt = np.ascontiguousarray(rec.types, np.int32)
    box6 = np.ascontiguousarray(box.as6(), np.float32)
    out = np.zeros((npose, 4), np.float32)
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        L.udref_score_batch(C.c_int(npose), C.c_int(lig.natom), p(xs), p(types), p(off), p(pairs), C.c_int(rec.natom),
                            p(rxyz), p(rt), p(box6), p(out))
        done += npose
    el = time.perf_counter() - t0
    return {"value": done / el, "unit": "poses/s", "cores": os.cpu_count() or 1, "kind": "reference",
            "sample": f"{done} poses of a {lig.natom}-atom screen ligand against {rec.natom} receptor atoms, "
                      f"the reference's score() (energy only, direct pair sum), OpenMP over poses, {el:.1f} s"}


# ------------------------------------------------------------------------- main arms
def run_reference(a):
    """The reference's CPU path on this host: the oracle restatement of the reference's
    search (direct-sum scoring as the reference), timed on bounded samples."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ud2b200.batching import heuristic_opt_steps
    nl = max(8, os.cpu_count() or 8)
    w, box, rec, ligs = make_inputs(a.workload, nl, a.seed, 0)
    mc = a.mc_steps or w["mc_steps"]
    opt = heuristic_opt_steps([l.natom for l in ligs], [l.ntors for l in ligs])
    per_step = max(2.0, min(30.0, 120.0 / max(1, a.steps + a.warmup)))
    rates = []
    for s in range(a.warmup + a.steps):
        r, cores, sample = cpu_port_rate(w, box, rec, ligs, mc, opt, per_step)
        if s >= a.warmup:
            rates.append(r)
    rate = statistics.mean(rates)
    lig_s = rate / (w["chains"] * mc)
    out = {"metric": METRIC, "value": lig_s, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": 1000.0 / lig_s, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": {"workload": a.workload, "chains": w["chains"], "mc_steps": mc, "opt_steps": opt,
                      "receptor_atoms": rec.natom, "box_A": w["box"]},
           "cpu_baseline": {"value": lig_s, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": lig_s, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    ref_sc = reference_scoring_rate(rec, box, ligs)
    if ref_sc:
        out["reference_cpu_scoring"] = ref_sc
    print(json.dumps(out), flush=True)


def reduce_over_ranks(dist, dev_ms: float, e2e_s: float, ligs_done: int, device: str):
    """Whole-job numbers of a multi-rank run: the slowest rank's device and end-to-end
    times, the ligands of all ranks."""
    import torch
    t = torch.tensor([dev_ms, e2e_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([float(ligs_done)], dtype=torch.float64, device=device)
    dist.all_reduce(n)
    return float(t[0]), float(t[1]), int(n.item())


def train_sets(workload: str, n: int, center, seeds=(101, 102, 103, 104)):
    """Training ligands: four seeded sets of the workload's distribution (not the batch)."""
    from ud2b200 import synth
    from ud2b200.model import parse_ligands
    out = []
    for sd in seeds:
        sizes = synth.ligand_sizes(workload, n, sd)
        d = {f"t{sd}_{i}": synth.make_ligand(na, nt, sd * 7919 + i, center) for i, (na, nt) in enumerate(sizes)}
        out.append(parse_ligands(d))
    return out


def top_scores(res):
    """Final score of each ligand's top-ranked pose (intra + inter + penalty + bias)."""
    return [float(r.terms[0].sum()) if len(r.records) else float("inf") for r in res]


def run_reference_gpu(a):
    """The reference's own CUDA engine (core_pipeline, built from its sources into
    oracle/_ref/udref_dock) and this engine on the same small batch and settings, both on
    this GPU; ligands/s are extrapolated to the workload's MC steps (the time is linear in
    MC steps).  Run on demand only."""
    import tempfile
    import numpy as np
    from ud2b200 import synth, Engine, MODE_GRID
    from ud2b200.batching import heuristic_opt_steps
    from ud2b200.model import Box, parse_ligands, parse_receptor
    exe = os.path.join(ROOT, "oracle", "_ref", "udref_dock")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference-gpu", "unavailable": "oracle/_ref/udref_dock not built (make -C oracle refengine)"}))
        return
    w = synth.WORKLOADS[a.workload]
    rows, center = synth.make_receptor(w["nrec"], w["cube"], a.seed)
    box = Box.from_center_size(center, [w["box"]] * 3)
    sizes = synth.ligand_sizes(a.workload, a.ref_ligands, a.seed)
    ligd = {f"lig{i:04d}": synth.make_ligand(n, t, a.seed * 7919 + i, center) for i, (n, t) in enumerate(sizes)}
    ligs = parse_ligands(ligd)
    opt = heuristic_opt_steps([l.natom for l in ligs], [l.ntors for l in ligs])
    steps = a.ref_mc_steps
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "input.json")
        with open(inp, "w") as f:
            json.dump(dict(receptor=rows, **ligd), f)
        cmd = [exe, inp, os.path.join(tmp, "out"), *[str(float(v)) for v in center], *[str(float(w["box"]))] * 3,
               str(w["chains"]), str(steps), str(opt), "5", str(w["num_pose"]), str(w["rmsd"]), "10.0", str(a.seed), "0"]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
        line = [l for l in r.stdout.splitlines() if l.startswith("{")]
        ref = json.loads(line[-1]) if line else {"rc": r.returncode}
        ref_poses = {}
        for fp in sorted(glob.glob(os.path.join(tmp, "out", "udref_*.json"))):
            with open(fp) as f:
                ref_poses.update(json.load(f))
    rec = parse_receptor(rows, box)
    eng = Engine(box)
    eng.set_receptor(rec.xyz, rec.types)
    mt = sorted(set(int(t) for l in ligs for t in l.types if t != 0))
    t0 = time.perf_counter()
    eng.build_grid(0.375, mt)
    eng.add_ligands(ligs)
    res, _ = eng.dock(seed=a.seed, nchain=w["chains"], mc_steps=steps, opt_steps=opt, refine_steps=5,
                      num_pose=w["num_pose"], rmsd_limit=w["rmsd"], energy_range=10.0, fetch=True)
    ours_s = time.perf_counter() - t0
    eng.close()
    full = w["mc_steps"] / steps
    # best scores: total (intra + inter + penalty) of each ligand's top-ranked pose; the
    # reference's from its JSON files (energy[1]), 3 decimals
    quality = None
    if all(n in ref_poses and ref_poses[n] for n in ligd):
        ref_top = np.array([ref_poses[n][0]["energy"][1] for n in ligd], np.float64)
        gap = np.array(top_scores(res), np.float64) - ref_top
        quality = {"within_0.3_of_reference": float(np.mean(gap <= 0.3)), "mean_gap": float(gap.mean()),
                   "max_gap": float(gap.max()), "better_than_reference": float(np.mean(gap < -1e-3))}
    out = {"impl": "reference-gpu", "metric": METRIC, "unit": UNIT, "workload": a.workload, "ligands": len(ligs),
           "chains": w["chains"], "mc_steps_run": steps, "mc_steps_workload": w["mc_steps"], "opt_steps": opt,
           "reference": {"rc": ref.get("rc"), "seconds": ref.get("seconds"),
                         "value": (len(ligs) / (ref["seconds"] * full)) if ref.get("seconds") else None,
                         "engine": "the reference's core_pipeline (direct pair sums), built from its sources"},
           "ours": {"seconds": ours_s, "value": len(ligs) / (ours_s * full),
                    "engine": "this engine, ud_dock with grid maps (grid build included)"},
           "quality": quality,
           "note": "wall times of one call each on the same GPU and inputs; ligands/s extrapolated linearly "
                   f"from {steps} to {w['mc_steps']} MC steps"}
    print(json.dumps(out), flush=True)


def run_ours(a):
    import numpy as np
    import torch
    from ud2b200 import Engine, GRID_F16, GRID_F32, MODE_GRID
    from ud2b200.batching import heuristic_opt_steps
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    nl = a.ligands
    w, box, rec, ligs = make_inputs(a.workload, nl, a.seed, rank)
    mc = a.mc_steps or w["mc_steps"]
    opt = heuristic_opt_steps([l.natom for l in ligs], [l.ntors for l in ligs])
    learned = a.mode == "learned"
    tsets = train_sets(a.workload, a.train_ligands, (box.lo.astype(np.float64) + box.hi) / 2.0) if learned else []
    mt = sorted(set(int(t) for l in list(ligs) + [x for ts in tsets for x in ts] for t in l.types if t != 0))
    eng = Engine(box, device=local)
    template = a.workload == "template"
    if template:
        # template-constrained screen: the shared core stays on its reference pose (no
        # translation or rotation), every chain keeps 4 poses -> 1024 clustered per ligand
        eng.set_flags(constraint=True)
        eng.set_retain(4)
    eng.set_receptor(rec.xyz, rec.types)
    eng.build_grid(0.375, mt, GRID_F16 if a.grid == "f16" else GRID_F32)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")   # 256 MB > L2
    base_kw = dict(seed=a.seed, nchain=w["chains"], opt_steps=opt, refine_steps=5, num_pose=w["num_pose"],
                   rmsd_limit=w["rmsd"], energy_range=10.0, randomize=True, mode=MODE_GRID)
    from ud2b200.engine import pack_ligands
    packed = pack_ligands(ligs)
    h2d = int(sum(v.nbytes for v in packed.values()))
    extra = {}
    if learned:
        # reference result and plain throughput: the fused engine at the workload's MC steps
        eng.clear_ligands()
        eng.add_ligands(ligs)
        flush.fill_(0.0)
        torch.cuda.synchronize()
        res_ref, _ = eng.dock(**base_kw, mc_steps=mc, fetch=True)
        st = eng.stage_times()
        ref_scores = np.array(top_scores(res_ref))
        plain_ms = float(st[5])
        # proposal network trained on the GPU from the plain engine's own searches
        from ud2b200.learned import train_proposal
        params, trep = train_proposal(box, rec, tsets, mt, opt_steps=opt, nchain=w["chains"], mc_steps=150,
                                      target=1, epochs=a.train_epochs, batch=1024, lr=1e-3, seed=1, device=local)
        eng.mlp_set_params(params)
        # the method without the network: the fused plain engine at the learned engine's steps
        res_eq, _ = eng.dock(**base_kw, mc_steps=a.learned_steps, fetch=True)
        eq_ms = float(eng.stage_times()[5])
        gap_eq = np.array(top_scores(res_eq)) - ref_scores
        extra = {"plain": {"value": len(ligs) / (plain_ms / 1000.0), "unit": UNIT, "ms_per_step": plain_ms,
                           "mc_steps": mc, "engine": "fused plain search (k_search)"},
                 "learned_training": {"train_ligands": sum(len(t) for t in tsets), "ligand_seeds": [101, 102, 103, 104],
                                      "samples": trep.samples, "collect_s": trep.collect_s, "train_s": trep.train_s,
                                      "epoch_loss": trep.epoch_loss, "target": "move to the ligand's best pose"},
                 "plain_equal_steps": {"value": len(ligs) / (eq_ms / 1000.0), "unit": UNIT, "mc_steps": a.learned_steps,
                                       "within": float(np.mean(gap_eq <= 0.3)), "mean_gap": float(np.mean(gap_eq)),
                                       "engine": "fused plain search at the learned engine's MC steps (untimed)"}}
        run_kw = dict(base_kw, mc_steps=a.learned_steps)
        p_learned = a.p_learned
    else:
        run_kw = dict(base_kw, mc_steps=mc)
        p_learned = None
    # warm-up steps dock the same batch through the same kernels with shorter chains
    warm_kw = dict(run_kw, mc_steps=min(run_kw["mc_steps"], a.warmup_mc_steps or run_kw["mc_steps"]))
    dev_ms, e2e_s, stage, heavy, evals, launches = [], [], [], 0, 0, 0
    sampler = ClockSampler(local)
    res = None
    for s in range(a.warmup + a.steps):
        if s == a.warmup:
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            sampler.__enter__()
        flush.fill_(float(s))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.clear_ligands()
        eng.add_ligands(ligs)
        res, ne = eng.dock(**(run_kw if s >= a.warmup else warm_kw), fetch=True, p_learned=p_learned)
        t1 = time.perf_counter()
        st = eng.stage_times()
        cn = eng.counters()
        if s >= a.warmup:
            dev_ms.append(float(st[5]))
            e2e_s.append(t1 - t0)
            stage.append(st.tolist())
            heavy += cn["heavy_atom_evaluations"]
            evals += cn["evaluations"]
            launches += cn["launches"]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler.__exit__()
    d2h = int(sum(4 * (len(r.records) * (8 + 3 * l.natom + l.ntors) + 4 * len(r.records)) for r, l in zip(res, ligs)))
    tot_ms = sum(dev_ms)
    tot_e2e = sum(e2e_s)
    search_ms = sum(x[0] for x in stage)
    ligs_done = len(ligs) * a.steps
    if learned:
        gap = np.array(top_scores(res)) - ref_scores
        within = float(np.mean(gap <= 0.3))
        extra["quality"] = {"gap_kcal_mol": 0.3, "within": within, "gate": 0.95, "gate_met": within >= 0.95,
                            "mean_gap": float(np.mean(gap)), "max_gap": float(np.max(gap)),
                            "reference": f"plain fused search at {mc} MC steps, same batch, same seed"}
    if dist:
        tot_ms, tot_e2e, ligs_done = reduce_over_ranks(dist, tot_ms, tot_e2e, ligs_done, f"cuda:{local}")
    value = ligs_done / (tot_ms / 1000.0)
    peak, peak_kind = load_peaks()
    bytes_alg = heavy * 8 * (2 if a.grid == "f16" else 4)
    achieved = bytes_alg / (search_ms / 1000.0) / 1e9 if search_ms > 0 else 0.0
    # launches of the dominant kernel per step: k_search runs a dock's search in one launch,
    # k_learn_step one MC step of every chain per launch
    launches_per_step = run_kw["mc_steps"] if learned else 1
    tr = load_traffic("k_learn_step_screen.md" if learned else "k_search_screen.md")
    traffic = tr if (tr is not None and nl == 148 and a.workload == "screen" and a.grid == "f32"
                     and (learned or mc == w["mc_steps"])) else None
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": tot_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic",
           "config": {"workload": a.workload, "engine": "learned proposal" if learned else "fused plain search",
                      "ligands_per_step_per_gpu": len(ligs), "chains": w["chains"], "mc_steps": run_kw["mc_steps"],
                      "p_learned": p_learned, "opt_steps": opt, "refine_steps": 5, "num_pose": w["num_pose"],
                      "rmsd_limit": w["rmsd"], "receptor_atoms": rec.natom, "box_A": w["box"], "grid_spacing_A": 0.375,
                      "grid_maps": len(mt), "grid_precision": a.grid, "l2": "flushed between steps (256 MB write)",
                      "constraint_docking": template, "poses_kept_per_chain": 4 if template else 1,
                      "warmup": f"{a.warmup} steps, same batch, {warm_kw['mc_steps']} MC steps per chain",
                      "parallelism": f"ligand shards x{world}"},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": traffic,
                        "kernel": "k_learn_step" if learned else "k_search",
                        "peak_kind": f"{peak_kind} hbm copy bandwidth",
                        "algorithmic_bytes_per_launch": bytes_alg / a.steps / launches_per_step,
                        "launches_per_step": launches_per_step},
           "e2e": {"value": ligs_done / tot_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "gpu_launches": launches,
           "stage_ms_per_step": [sum(x[i] for x in stage) / a.steps for i in range(6)],
           "evaluations_per_step": evals / a.steps,
           "poses_scored_per_s": evals / (search_ms / 1000.0) if search_ms > 0 else None,
           "clocks": sampler.summary()}
    out.update(extra)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        rate, cores, sample = cpu_port_rate(w, box, rec, ligs, mc, opt, a.cpu_seconds)
        out["cpu_baseline"] = {"value": rate / (w["chains"] * mc), "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": sample + f"; ligands/s at {mc} MC steps per chain"}
        ref_sc = reference_scoring_rate(rec, box, ligs)
        if ref_sc:
            out["reference_cpu_scoring"] = ref_sc
    eng.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.impl == "reference-gpu":
        run_reference_gpu(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
