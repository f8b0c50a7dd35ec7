"""Drop-in replacement for the reference's pybind module ``unidock_engine.api.python.pipeline``.

Same class, keyword-only constructor arguments and defaults, methods and output files as
the reference (unidock/unidock_engine/api/python/pipeline.cpp:56-217, defaults
src/screening/core.h:9-92 and src/model/model.h:151-167).  ``run()`` drives the B200
engine (libudock_b200.so) instead of the reference's CUDA engine:

* presets: search_mode fast/balance/detail/free (src/screening/core.cpp:65-84), task
  screen/score/mc/randomize/optimize (core.cpp:165-212), bias no/pos/align (core.cpp:86-97),
  constraint docking disables randomisation (core.cpp:142-146);
* ligands are parsed, and their pair lists built, in bulk by the native parser
  (``ud_ligset_parse_json``; rapidjson_parser.cpp:54-296);
* ligands are ordered in the reference's size groups and batches of at most 1000
  (src/screening/screening.cpp:17-41,162-216), one output file per batch
  ``<output_dir>/<name_json>_<batch>.json``; ``opt_steps=-1`` resolves to
  ``(25 + max atoms of the first batch) / 3`` and keeps that value (screening.cpp:206-208);
  the engine docks as many consecutive batches of one size group in one launch as fit the
  device memory budget (95 % of the free memory, capped by ``max_gpu_mem`` MB;
  core.cpp:32-63), so a ligand's chains get their random streams from its place in the
  launch;
* output JSON ``{ligand: [{"energy": [affinity, total, intra, inter, penalty, conf_indep,
  bias], "coords": [...], "dihedrals": [deg...], ("decomp": [[5]...])}]}``, 3 decimals,
  non-finite values clamped to +-1e6 (src/format/json.cpp:88-191, src/task/DockTask.cpp:224-282);
* failures raise ``RuntimeError("Core pipeline failed...")`` (pipeline.cpp:141-143).

Additional optional keyword arguments (not in the reference): ``scoring`` ("grid" or
"direct" intermolecular term during search), ``grid_precision`` ("f32" or "f16"),
``grid_spacing`` (A), ``proposal_params`` (parameters of a trained move-proposal network, a
flat float32 array or the path of one saved with numpy; grid scoring only), ``p_learned``
(share of learned moves when a network is given, default 0.25), ``poses_per_chain`` (1-4
poses kept per chain before clustering) and ``autotune`` (time chain packings per batch).
"""
from __future__ import annotations

import json
import logging
import math
import os
import time
from decimal import ROUND_DOWN, Decimal
from typing import Dict, List, Optional

import numpy as np

from ud2b200.batching import memory_budget, plan_launches, predict_dock_bytes, reference_batches
from ud2b200.engine import Engine, EngineError, MODE_DIRECT, MODE_GRID, GRID_F16, GRID_F32
from ud2b200.ligset import LigandRef, parse_ligands_bulk
from ud2b200.model import Box, F32, RAD2DEG_F, parse_receptor

log = logging.getLogger("unidock_engine")

W_CONF = F32(0.05846)
MAX_SAFE = 1e6


def _safe(v: float) -> float:
    """json.cpp:78-85"""
    if not math.isfinite(v):
        return MAX_SAFE
    return max(-MAX_SAFE, min(MAX_SAFE, v))


def _fmt(v: float) -> str:
    """One value as the reference's writer prints it: the float widened to double, its
    shortest round-trip digits truncated to 3 decimals, trailing zeros dropped keeping one
    (rapidjson Writer::Double with SetMaxDecimalPlaces(3): include/rapidjson/internal/dtoa.h,
    Prettify).  The scalar statement of the rule; ``_fmt_array`` is the fast one."""
    v = _safe(float(np.float32(v)))
    q = int(Decimal(repr(abs(v))).scaleb(3).to_integral_value(rounding=ROUND_DOWN))
    ip, fr = divmod(q, 1000)
    return ("-" if math.copysign(1.0, v) < 0 else "") + str(ip) + _FRAC[fr]


# ".d", ".dd" or ".ddd" for 0..999 thousandths, trailing zeros dropped keeping one digit
_FRAC = ["." + (("%03d" % i).rstrip("0") or "0") for i in range(1000)]
_FRAC_NP = np.array(_FRAC)


def _fmt_array(vals) -> List[str]:
    """``_fmt`` of every value, vectorised.  A float32 value times 1000 is exact in double
    (24 + 10 significant bits), so flooring it gives the truncated thousandths of the exact
    value; those equal the truncation of the shortest digits, because a float32 value that
    is not a multiple of 1/1000 lies further from one (about 2^-34 of its magnitude at
    least: its ulp over 1000) than its shortest double digits lie from it (2^-53)."""
    v = np.asarray(vals, np.float32).astype(np.float64).reshape(-1)
    v = np.where(np.isfinite(v), np.clip(v, -MAX_SAFE, MAX_SAFE), MAX_SAFE)
    q = np.floor(np.abs(v) * 1000.0).astype(np.int64)
    s = np.strings.add(np.strings.add(np.where(np.signbit(v), "-", ""), (q // 1000).astype(str)),
                       _FRAC_NP[q % 1000])
    return s.tolist()


def _host_memory() -> int:
    try:
        return os.sysconf("SC_PHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        return 0


class DockingPipeline:
    """Uni-Dock2 molecular docking pipeline (B200 engine)."""

    def __init__(self, *, output_dir: str = "./res_ud2", center_x: float, center_y: float, center_z: float,
                 size_x: float, size_y: float, size_z: float, task: str = "screen", search_mode: str = "balance",
                 exhaustiveness: int = 512, randomize: bool = True, mc_steps: int = 20, opt_steps: int = -1,
                 refine_steps: int = 5, num_pose: int = 10, rmsd_limit: float = 1.0, energy_range: float = 10.0,
                 seed: int = 12345, bias: str = "no", bias_k: float = 0.1, constraint_docking: bool = False,
                 use_tor_lib: bool = False, energy_decomp: bool = False, gpu_device_id: int = 0,
                 name_json: str = "from_python_obj", max_gpu_mem: int = 0,
                 scoring: str = "grid", grid_precision: str = "f32", grid_spacing: float = 0.375,
                 proposal_params=None, p_learned: float = 0.25, poses_per_chain: int = 1, autotune: bool = False):
        self.output_dir = output_dir
        self.box = Box.from_center_size([center_x, center_y, center_z], [size_x, size_y, size_z])
        self.task = task
        self.search_mode = search_mode
        self.exhaustiveness = int(exhaustiveness)
        self.randomize = bool(randomize)
        self.mc_steps = int(mc_steps)
        self.opt_steps = int(opt_steps)
        self.refine_steps = int(refine_steps)
        self.num_pose = int(num_pose)
        self.rmsd_limit = float(rmsd_limit)
        self.energy_range = float(energy_range)
        self.seed = int(seed)
        self.bias = bias
        self.bias_k = float(bias_k)
        self.constraint_docking = bool(constraint_docking)
        self.use_tor_lib = bool(use_tor_lib)
        self.energy_decomp = bool(energy_decomp)
        self.gpu_device_id = int(gpu_device_id)
        self.name_json = name_json
        self.max_gpu_mem = int(max_gpu_mem)
        self.scoring = scoring
        self.grid_precision = grid_precision
        self.grid_spacing = float(grid_spacing)
        if isinstance(proposal_params, str):
            proposal_params = np.load(proposal_params)
        self.proposal_params = None if proposal_params is None else np.asarray(proposal_params, np.float32)
        self.p_learned = float(p_learned)
        self.poses_per_chain = int(poses_per_chain)
        self.autotune = bool(autotune)
        self._receptor: List = []
        self._ligands: Dict[str, dict] = {}
        self.last_stats: Dict[str, float] = {}

    def set_receptor(self, receptor_info: list) -> None:
        """Receptor atoms: rows [x, y, z, vina_type, ff_type, charge]."""
        self._receptor = receptor_info

    def add_ligands(self, ligands_info: dict) -> None:
        """Ligand topologies keyed by name (later keys overwrite earlier ones)."""
        for k, v in ligands_info.items():
            self._ligands[k] = v

    # ------------------------------------------------------------------ run
    def _params(self) -> dict:
        p = dict(seed=self.seed, exhaustiveness=self.exhaustiveness, randomize=self.randomize,
                 mc_steps=self.mc_steps, opt_steps=-1 if self.opt_steps < 0 else self.opt_steps,
                 refine_steps=self.refine_steps, num_pose=self.num_pose, energy_range=self.energy_range,
                 rmsd_limit=self.rmsd_limit)
        if self.bias not in ("no", "pos", "align"):
            raise ValueError(f"Not supported bias: {self.bias} doesn't belong to (no, pos, align)")
        p["bias_type"] = {"no": 0, "pos": 1, "align": 2}[self.bias]
        sm = self.search_mode
        if sm in ("", "free"):
            pass
        elif sm == "fast":
            p.update(exhaustiveness=128, mc_steps=20, opt_steps=-1)
        elif sm == "balance":
            p.update(exhaustiveness=256, mc_steps=30, opt_steps=-1)
        elif sm == "detail":
            p.update(exhaustiveness=512, mc_steps=40, opt_steps=-1)
        else:
            raise ValueError(f"Not supported search_mode: {sm} doesn't belong to (fast, balance, detail, free)")
        if self.constraint_docking:
            p["randomize"] = False
        t = self.task
        if t == "screen":
            pass
        elif t == "score":
            p.update(randomize=False, exhaustiveness=1, mc_steps=0, opt_steps=0, refine_steps=0, num_pose=1,
                     energy_range=999.0, rmsd_limit=999.0)
        elif t == "benchmark_one":
            p["skip"] = True
        elif t == "mc":
            p.update(randomize=True, opt_steps=0, refine_steps=0)
        elif t == "randomize":
            p.update(randomize=True, mc_steps=0, opt_steps=0, refine_steps=0, num_pose=p["exhaustiveness"],
                     energy_range=1e9, rmsd_limit=0.0)
        elif t == "optimize":
            p.update(randomize=False, exhaustiveness=1, mc_steps=0, opt_steps=0, num_pose=1, energy_range=1e9,
                     rmsd_limit=0.0)
        else:
            raise ValueError(f"Not supported task: {t} doesn't belong to (screen, local_only, mc)")
        return p

    def run(self) -> None:
        """Dock every ligand; writes <output_dir>/<name_json>_<batch>.json files."""
        try:
            self._run()
        except Exception as e:  # the reference surfaces any failure as this RuntimeError
            log.error("Core pipeline failed: %s", e)
            raise RuntimeError(f"Core pipeline failed. {e}") from e

    def _run(self) -> None:
        t0 = time.perf_counter()
        p = self._params()
        os.makedirs(self.output_dir, exist_ok=True)
        if p.get("skip"):
            log.warning("benchmark task is not implemented")
            return
        rec = parse_receptor(self._receptor, self.box)
        # all ligands parsed and their pair lists built natively, in document order
        ls = parse_ligands_bulk(self._ligands, self.use_tor_lib)
        if len(ls) == 0:
            log.error("No flexible molecules are found")
        ref_batches = reference_batches(ls.natoms, ls.ntors)
        eng = Engine(self.box, device=self.gpu_device_id)
        try:
            eng.set_flags(self.constraint_docking, p["bias_type"], self.bias_k)
            eng.set_receptor(rec.xyz, rec.types)
            if self.poses_per_chain != 1:
                eng.set_retain(self.poses_per_chain)
            if self.autotune:
                eng.set_autotune(True)
            mode = MODE_GRID if self.scoring == "grid" else MODE_DIRECT
            if mode == MODE_GRID:
                mt = sorted(int(t) for t in np.unique(ls.a["types"]) if t != 0)
                if mt:
                    eng.build_grid(self.grid_spacing, mt, GRID_F16 if self.grid_precision == "f16" else GRID_F32)
                else:
                    mode = MODE_DIRECT
            learned = None
            if self.proposal_params is not None and mode == MODE_GRID and p["mc_steps"] > 0:
                eng.mlp_set_params(self.proposal_params)
                learned = self.p_learned
            opt_steps = p["opt_steps"]
            if opt_steps == -1 and ref_batches:       # the first batch decides (screening.cpp:206-208)
                opt_steps = (25 + int(max(ls.natoms[i] for i in ref_batches[0][1]))) // 3
            # launches: as many of the reference's batches of one size group as fit the device
            # memory budget (max_gpu_mem caps it); output files still one per reference batch
            a = ls.a
            per_lig = predict_dock_bytes(ls.natoms, ls.ntors, np.diff(a["pair_off"][a["atom_off"]]),
                                         np.diff(a["rot_off"][a["tors_off"]]), np.diff(a["range_off"][a["tors_off"]]),
                                         np.diff(a["bias_off"][a["atom_off"]]), nchain=p["exhaustiveness"],
                                         retain=self.poses_per_chain, num_pose=p["num_pose"],
                                         learned=learned is not None, decomp=self.energy_decomp)
            free, _ = eng.device_memory()
            budget = memory_budget(free, self.max_gpu_mem, _host_memory())
            plan = plan_launches(ref_batches, per_lig, budget)
            batch_of = np.empty(len(ls), np.int64)
            left = []
            for k, (_, b) in enumerate(ref_batches):
                batch_of[b] = k
                left.append(len(b))
            done: Dict[int, object] = {}
            nevals = 0
            for run in plan:
                eng.clear_ligands()
                eng.add_ligands(ls.subset(run))
                res, ne = eng.dock(seed=p["seed"], nchain=p["exhaustiveness"], mc_steps=p["mc_steps"],
                                   opt_steps=opt_steps, refine_steps=p["refine_steps"], num_pose=p["num_pose"],
                                   rmsd_limit=p["rmsd_limit"], energy_range=p["energy_range"],
                                   randomize=p["randomize"], mode=mode, final_mode=MODE_DIRECT,
                                   energy_decomp=self.energy_decomp, p_learned=learned)
                nevals += ne
                for i, r in zip(run, res):
                    done[i] = r
                    k = int(batch_of[i])
                    left[k] -= 1
                    if left[k] == 0:                  # a reference batch is complete: its file
                        b = ref_batches[k][1]
                        fp = os.path.join(self.output_dir, f"{self.name_json}_{k + 1}.json")
                        self._dump(fp, [LigandRef(ls, j) for j in b], [done.pop(j) for j in b])
            self.last_launches = len(plan)
        finally:
            eng.close()
        self.last_stats = dict(seconds=time.perf_counter() - t0, evaluations=float(nevals), ligands=float(len(ls)),
                               launches=float(len(plan)))

    # ------------------------------------------------------------------ output
    def _dump(self, fp: str, ligs, results) -> None:
        parts = []
        for lig, r in zip(ligs, results):
            n3, nt = 3 * lig.natom, lig.ntors
            k = len(r.records)
            if k == 0:
                parts.append(json.dumps(lig.name) + ":[]")
                continue
            # the energy vector in float32 arithmetic (DockTask.cpp:224-282)
            intra, inter, pen, bias = (r.terms[:k, c].astype(np.float32) for c in range(4))
            total = (intra + inter) + pen
            e_inter = total - intra[0]
            aff = e_inter / (F32(1) + W_CONF * F32(nt))
            conf = aff - e_inter
            recs = np.stack(r.records)
            vals = [np.stack([aff, total, intra, inter, pen, conf, bias], axis=1), recs[:, 8:8 + n3],
                    recs[:, 8 + n3:8 + n3 + nt] * RAD2DEG_F]
            dec = self.energy_decomp and r.decomp is not None
            if dec:
                vals.append(r.decomp[:k].reshape(k, -1))
            txt = _fmt_array(np.concatenate([v.astype(np.float32) for v in vals], axis=1))
            w = len(txt) // k
            poses = []
            for j in range(k):
                t = txt[j * w:(j + 1) * w]
                s = '{"energy":[' + ",".join(t[:7]) + '],"coords":[' + ",".join(t[7:7 + n3]) + \
                    '],"dihedrals":[' + ",".join(t[7 + n3:7 + n3 + nt]) + "]"
                if dec:
                    d = t[7 + n3 + nt:]
                    s += ',"decomp":[' + ",".join("[" + ",".join(d[a:a + 5]) + "]" for a in range(0, len(d), 5)) + "]"
                poses.append(s + "}")
            parts.append(json.dumps(lig.name) + ":[" + ",".join(poses) + "]")
        text = "{" + ",".join(parts) + "}"
        wait = 5
        for attempt in range(5):     # DockTask.cpp:285-333: retry with back-off, check completeness
            try:
                with open(fp, "w") as f:
                    f.write(text)
                    f.flush()
                    os.fsync(f.fileno())
                with open(fp, "rb") as f:
                    f.seek(-1, os.SEEK_END)
                    if f.read(1) != b"}":
                        raise IOError("JSON file is incomplete.")
                return
            except Exception:
                if attempt == 4:
                    raise
                time.sleep(wait)
                wait *= 2
