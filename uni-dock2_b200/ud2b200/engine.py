"""ctypes binding of libudock_b200.so (the C ABI declared in include/udock_b200.h).

This is the host side of the docking engine: it packs parsed ligands into the flat
CSR arrays the C ABI takes, and unpacks pose records.  There is no CPU fallback:
if the CUDA library is missing or no GPU is present, calls raise EngineError.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .model import Box, Ligand

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libudock_b200.so"

MODE_DIRECT = 0
MODE_GRID = 1
GRID_F32 = 0
GRID_F16 = 1


class EngineError(RuntimeError):
    pass


_lib = None


def lib_path() -> str:
    """The engine library: UDOCK_B200_LIB if set, else the in-tree build."""
    return os.environ.get("UDOCK_B200_LIB") or os.path.join(HERE, LIB_NAME)


def read_bandwidth(device: int, nbytes: int, repeats: int = 20) -> float:
    """GB/s of streaming reads of an nbytes buffer on `device` (L2 when it fits, else HBM)."""
    L = load_library()
    out = C.c_float(0.0)
    if L.ud_read_bandwidth(int(device), int(nbytes), int(repeats), C.byref(out)) != 0:
        raise EngineError(L.ud_last_error().decode(errors="replace"))
    return float(out.value)


def learned_block(p_learned: float, recording: bool = False) -> int:
    """MC steps per launch of the learned search for p_learned (ud_learned_block)."""
    return int(load_library().ud_learned_block(float(p_learned), int(recording)))


def load_library() -> C.CDLL:
    """Load the CUDA engine; raises EngineError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        raise EngineError(f"{LIB_NAME} not built (run __graft_entry__.build() or uni-dock2_b200/build.py)")
    L = C.CDLL(path)
    vp, ip, fp, i, f = C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float
    sig = {
        "ud_version": ([], i),
        "ud_last_error": ([], C.c_char_p),
        "ud_create": ([i, fp, C.POINTER(C.c_void_p)], i),
        "ud_destroy": ([vp], i),
        "ud_set_flags": ([vp, i, i, f], i),
        "ud_set_receptor": ([vp, i, fp, ip], i),
        "ud_receptor_count": ([vp], i),
        "ud_build_grid": ([vp, f, i, ip, i], i),
        "ud_get_grid": ([vp, fp, ip, fp], i),
        "ud_set_grid_precision": ([vp, i], i),
        "ud_add_ligands": ([vp, i, ip, fp, ip, ip, ip, fp, ip, fp, ip, ip, ip, ip, ip, fp], i),
        "ud_clear_ligands": ([vp], i),
        "ud_ligand_count": ([vp], i),
        "ud_record_floats": ([vp, i], i),
        "ud_score_batch": ([vp, i, ip, fp, fp, fp, i, f, f, fp, fp], i),
        "ud_score_batch_noalloc": ([vp, i, ip, fp, fp, fp, i, f, f, fp, fp], i),
        "ud_score_terms": ([vp, i, ip, fp, i, fp, fp], i),
        "ud_bfgs_batch": ([vp, i, ip, fp, i, i, f, f, i, i, ip], i),
        "ud_search": ([vp, C.c_uint64, i, i, i, i, i, C.POINTER(C.c_longlong)], i),
        "ud_get_chain_poses": ([vp, i, fp], i),
        "ud_cluster": ([vp, f, ip, ip], i),
        "ud_dock": ([vp, vp, C.POINTER(C.c_longlong)], i),
        "ud_result_counts": ([vp, ip], i),
        "ud_get_results": ([vp, fp, fp, fp], i),
        "ud_result_floats": ([vp], C.c_longlong),
        "ud_sync": ([vp], i),
        "ud_stream": ([vp], C.c_void_p),
        "ud_stage_times": ([vp, fp], i),
        "ud_counters": ([vp, ip], i),
        "ud_set_autotune": ([vp, i], i),
        "ud_set_packing": ([vp, i, i], i),
        "ud_search_shape": ([vp, ip], i),
        "ud_set_retain": ([vp, i], i),
        "ud_mlp_param_count": ([], C.c_longlong),
        "ud_mlp_init": ([vp, C.c_uint64], i),
        "ud_mlp_set_gemm": ([vp, i], i),
        "ud_mlp_set_params": ([vp, fp], i),
        "ud_mlp_get_params": ([vp, fp], i),
        "ud_mlp_forward": ([vp, i, fp, fp], i),
        "ud_mlp_loss_grad": ([vp, i, fp, fp, fp, C.POINTER(C.c_double), fp], i),
        "ud_mlp_train": ([vp, i, fp, fp, fp, i, i, f, C.c_uint64, fp], i),
        "ud_search_learned": ([vp, C.c_uint64, i, i, i, i, f, C.POINTER(C.c_longlong)], i),
        "ud_collect_moves": ([vp, C.c_uint64, i, i, i, i, i, i, C.POINTER(C.c_int)], i),
        "ud_get_moves": ([vp, i, fp, fp, fp], i),
        "ud_dock_learned": ([vp, vp, f, C.POINTER(C.c_longlong)], i),
        "ud_learned_block": ([f, i], i),
        "ud_mlp_train_moves": ([vp, i, i, f, C.c_uint64, fp], i),
        "ud_read_bandwidth": ([i, C.c_longlong, i, fp], i),
        "ud_score_batch_timed": ([vp, i, ip, fp, fp, fp, i, f, f, i, fp, fp, fp], i),
        "ud_device_memory": ([i, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], i),
        "ud_ligset_parse_json": ([C.c_char_p, C.c_size_t, i, i, C.POINTER(C.c_void_p)], i),
        "ud_ligset_sizes": ([vp, vp], i),
        "ud_ligset_export": ([vp] + [vp] * 19, i),
        "ud_ligset_free": ([vp], None),
        "ud_ligset_last_error": ([], C.c_char_p),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


class DockParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("nchain", C.c_int), ("mc_steps", C.c_int), ("opt_steps", C.c_int),
                ("refine_steps", C.c_int), ("num_pose", C.c_int), ("rmsd_limit", C.c_float),
                ("energy_range", C.c_float), ("randomize", C.c_int), ("mode", C.c_int), ("final_mode", C.c_int),
                ("energy_decomp", C.c_int), ("refine_mode", C.c_int)]


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def record_len(lig: Ligand) -> int:
    return 8 + 3 * lig.natom + lig.ntors


def make_record(lig: Ligand, coords=None, center=None, rot_vec=None, dihedrals=None, energy: float = 999.0) -> np.ndarray:
    """Pose record [energy, centre(3), rot_vec(3), 0, coords(3N), dihedrals(T)]."""
    r = np.zeros(record_len(lig), np.float32)
    r[0] = energy
    r[1:4] = lig.center if center is None else center
    r[4:7] = 0.0 if rot_vec is None else rot_vec
    r[8:8 + 3 * lig.natom] = (lig.coords if coords is None else np.asarray(coords)).reshape(-1)
    if lig.ntors:
        r[8 + 3 * lig.natom:] = lig.dihedrals if dihedrals is None else dihedrals
    return r


def split_record(lig: Ligand, r: np.ndarray) -> dict:
    n = lig.natom
    return dict(energy=float(r[0]), center=r[1:4].copy(), rot_vec=r[4:7].copy(),
                coords=r[8:8 + 3 * n].reshape(n, 3).copy(), dihedrals=r[8 + 3 * n:8 + 3 * n + lig.ntors].copy())


def pack_ligands(ligs: Sequence[Ligand]) -> Dict[str, np.ndarray]:
    """Concatenate ligand topologies into the CSR arrays of ud_add_ligands."""
    nat = [l.natom for l in ligs]
    ntor = [l.ntors for l in ligs]
    atom_off = np.zeros(len(ligs) + 1, np.int32)
    atom_off[1:] = np.cumsum(nat)
    tors_off = np.zeros(len(ligs) + 1, np.int32)
    tors_off[1:] = np.cumsum(ntor)
    xyz = np.concatenate([l.coords.reshape(-1) for l in ligs]).astype(np.float32)
    types = np.concatenate([l.types for l in ligs]).astype(np.int32)
    T = int(tors_off[-1])
    axis = (np.concatenate([l.axis.reshape(-1) for l in ligs if l.ntors]).astype(np.int32)
            if T else np.zeros(2, np.int32))
    dihe = (np.concatenate([l.dihedrals for l in ligs if l.ntors]).astype(np.float32) if T else np.zeros(1, np.float32))
    rcounts = [len(r) for l in ligs for r in l.ranges]
    range_off = np.zeros(T + 1, np.int32)
    if T:
        range_off[1:] = np.cumsum(rcounts)
    ranges = (np.concatenate([np.asarray(r, np.float32).reshape(-1) for l in ligs for r in l.ranges])
              if T else np.zeros(2, np.float32))
    rot_counts = [len(r) for l in ligs for r in l.rotated]
    rot_off = np.zeros(T + 1, np.int32)
    if T:
        rot_off[1:] = np.cumsum(rot_counts)
    rot = (np.concatenate([r for l in ligs for r in l.rotated]).astype(np.int32)
           if T and sum(rot_counts) else np.zeros(1, np.int32))
    A = int(atom_off[-1])
    pair_off = np.zeros(A + 1, np.int32)
    cnts = np.concatenate([np.diff(l.pair_off) for l in ligs])
    pair_off[1:] = np.cumsum(cnts)
    pairs = np.concatenate([l.pairs for l in ligs]).astype(np.int32) if pair_off[-1] else np.zeros(1, np.int32)
    bias_off = np.zeros(A + 1, np.int32)
    bparts, bcounts = [], []
    for l in ligs:
        off, par = l.bias_csr()
        bcounts.append(np.diff(off))
        if par.size:
            bparts.append(par.reshape(-1))
    bias_off[1:] = np.cumsum(np.concatenate(bcounts))
    bias = np.concatenate(bparts).astype(np.float32) if bparts else np.zeros(5, np.float32)
    return dict(atom_off=atom_off, xyz=xyz, types=types, tors_off=tors_off, axis=axis, dihedrals=dihe,
                range_off=range_off, ranges=ranges, rot_off=rot_off, rot=rot, pair_off=pair_off, pairs=pairs,
                bias_off=bias_off, bias=bias)


@dataclass
class DockResult:
    """Output poses of one ligand in rank order."""
    records: List[np.ndarray]
    terms: np.ndarray          # (k, 4) intra, inter, penalty, bias
    decomp: Optional[np.ndarray]


class Engine:
    """One docking context on one GPU."""

    def __init__(self, box: Box, device: int = 0):
        self.L = load_library()
        self.box = box
        h = C.c_void_p()
        b6 = box.as6()
        self._check(self.L.ud_create(device, _p(b6), C.byref(h)))
        self.h = h
        self.device = int(device)
        self.ligands: List[Ligand] = []
        self.nchain = 0
        self.retain = 1

    def _check(self, rc: int):
        if rc != 0:
            msg = self.L.ud_last_error().decode(errors="replace")
            raise EngineError(msg or f"engine call failed ({rc})")

    def close(self):
        if getattr(self, "h", None):
            self.L.ud_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ setup
    def set_flags(self, constraint: bool = False, bias_type: int = 0, bias_k: float = 0.1):
        self._check(self.L.ud_set_flags(self.h, int(constraint), int(bias_type), float(bias_k)))

    def set_receptor(self, xyz: np.ndarray, types: np.ndarray):
        x = np.ascontiguousarray(xyz, np.float32).reshape(-1)
        t = np.ascontiguousarray(types, np.int32)
        self._check(self.L.ud_set_receptor(self.h, int(t.size), _p(x), _p(t)))

    @property
    def receptor_count(self) -> int:
        return self.L.ud_receptor_count(self.h)

    def build_grid(self, spacing: float, map_types: Sequence[int], precision: int = GRID_F32):
        mt = np.ascontiguousarray(map_types, np.int32)
        self._check(self.L.ud_build_grid(self.h, float(spacing), int(mt.size), _p(mt), int(precision)))
        self.map_types = list(int(v) for v in mt)

    def set_grid_precision(self, precision: int):
        self._check(self.L.ud_set_grid_precision(self.h, int(precision)))

    def get_grid(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        gd = np.zeros(3, np.int32)
        org = np.zeros(3, np.float32)
        self._check(self.L.ud_get_grid(self.h, None, _p(gd), _p(org)))
        out = np.zeros((len(self.map_types), gd[2], gd[1], gd[0]), np.float32)
        self._check(self.L.ud_get_grid(self.h, _p(out), _p(gd), _p(org)))
        return out, gd, org

    def add_ligands(self, ligs):
        """Append ligands: a sequence of Ligand, or a LigandSet from the native bulk
        parser (its packed arrays go to the engine as they are)."""
        if len(ligs) == 0:
            return
        from .ligset import LigandSet, LigandRef
        bulk = isinstance(ligs, LigandSet)
        p = ligs.packed() if bulk else pack_ligands(ligs)
        self._check(self.L.ud_add_ligands(self.h, len(ligs), _p(p["atom_off"]), _p(p["xyz"]), _p(p["types"]),
                                          _p(p["tors_off"]), _p(p["axis"]), _p(p["dihedrals"]), _p(p["range_off"]),
                                          _p(p["ranges"]), _p(p["rot_off"]), _p(p["rot"]), _p(p["pair_off"]),
                                          _p(p["pairs"]), _p(p["bias_off"]), _p(p["bias"])))
        if bulk:
            self.ligands.extend(LigandRef(ligs, i) for i in range(len(ligs)))
        else:
            self.ligands.extend(ligs)

    def device_memory(self):
        """(free, total) bytes of this context's device."""
        fr, tot = C.c_longlong(0), C.c_longlong(0)
        self._check(self.L.ud_device_memory(self.device, C.byref(fr), C.byref(tot)))
        return int(fr.value), int(tot.value)

    def clear_ligands(self):
        self._check(self.L.ud_clear_ligands(self.h))
        self.ligands = []

    # ------------------------------------------------------------ compute
    def score_batch(self, pose_lig: Sequence[int], coords: Sequence[np.ndarray], centers, rotvecs,
                    mode: int = MODE_GRID, vcap: float = 1e30, slope: float = 1e6):
        pl = np.ascontiguousarray(pose_lig, np.int32)
        x = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float32).reshape(-1) for c in coords]))
        ce = np.ascontiguousarray(centers, np.float32).reshape(-1)
        rv = np.ascontiguousarray(rotvecs, np.float32).reshape(-1)
        dims = [6 + self.ligands[l].ntors for l in pl]
        e = np.zeros(len(pl), np.float32)
        g = np.zeros(int(sum(dims)), np.float32)
        self._check(self.L.ud_score_batch(self.h, len(pl), _p(pl), _p(x), _p(ce), _p(rv), int(mode), float(vcap),
                                          float(slope), _p(e), _p(g)))
        gs = np.split(g, np.cumsum(dims)[:-1]) if len(dims) > 1 else [g]
        return e, gs

    def score_batch_timed(self, pose_lig: Sequence[int], coords: Sequence[np.ndarray], centers, rotvecs,
                          mode: int = MODE_GRID, vcap: float = 1e30, slope: float = 1e6, repeats: int = 5):
        """score_batch with the inputs resident on the device: (energies, gradients, mean
        kernel ms over `repeats` launches)."""
        pl = np.ascontiguousarray(pose_lig, np.int32)
        x = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float32).reshape(-1) for c in coords]))
        ce = np.ascontiguousarray(centers, np.float32).reshape(-1)
        rv = np.ascontiguousarray(rotvecs, np.float32).reshape(-1)
        dims = np.array([6 + self.ligands[l].ntors for l in range(len(self.ligands))], np.int64)[pl]
        e = np.zeros(len(pl), np.float32)
        g = np.zeros(int(dims.sum()), np.float32)
        ms = C.c_float(0.0)
        self._check(self.L.ud_score_batch_timed(self.h, len(pl), _p(pl), _p(x), _p(ce), _p(rv), int(mode),
                                                float(vcap), float(slope), int(repeats), _p(e), _p(g), C.byref(ms)))
        return e, g, float(ms.value)

    def score_batch_noalloc(self, pose_lig: Sequence[int], coords: Sequence[np.ndarray], centers, rotvecs,
                            mode: int = MODE_GRID, vcap: float = 1e30, slope: float = 1e6):
        """score_batch through ud_score_batch_noalloc: no device allocation inside the call;
        staging in the library's fixed per-device array (limits in include/udock_b200.h)."""
        pl = np.ascontiguousarray(pose_lig, np.int32)
        x = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float32).reshape(-1) for c in coords]))
        ce = np.ascontiguousarray(centers, np.float32).reshape(-1)
        rv = np.ascontiguousarray(rotvecs, np.float32).reshape(-1)
        dims = [6 + self.ligands[l].ntors for l in pl]
        e = np.zeros(len(pl), np.float32)
        g = np.zeros(int(sum(dims)), np.float32)
        self._check(self.L.ud_score_batch_noalloc(self.h, len(pl), _p(pl), _p(x), _p(ce), _p(rv), int(mode),
                                                  float(vcap), float(slope), _p(e), _p(g)))
        gs = np.split(g, np.cumsum(dims)[:-1]) if len(dims) > 1 else [g]
        return e, gs

    def set_retain(self, retain: int):
        """Poses kept per chain (1..4); chain_poses/cluster then hold nchain * retain poses."""
        self._check(self.L.ud_set_retain(self.h, int(retain)))
        self.retain = int(retain)

    def set_autotune(self, on: bool = True):
        """Time chain packings on each new batch shape and keep the fastest (results unchanged)."""
        self._check(self.L.ud_set_autotune(self.h, int(bool(on))))

    def set_packing(self, warps_per_cta: int = 0, chains_per_warp: int = 0):
        """Fix the chain packing (4, 8 or 12 warps per CTA; 1..4 chains per warp per item;
        0 = chosen per batch).  Results do not depend on it."""
        self._check(self.L.ud_set_packing(self.h, int(warps_per_cta), int(chains_per_warp)))

    def search_shape(self) -> dict:
        """Launch shape of the last search."""
        s = np.zeros(4, np.int32)
        self._check(self.L.ud_search_shape(self.h, _p(s)))
        return dict(warps_per_cta=int(s[0]), ctas_per_sm=int(s[1]), register_class=int(s[2]),
                    chains_per_warp=int(s[3]))

    # ------------------------------------------------------------------ learned proposal
    MLP_IN, MLP_OUT, MLP_NDIM = 672, 64, 26

    def mlp_param_count(self) -> int:
        return int(self.L.ud_mlp_param_count())

    def mlp_set_gemm(self, kind: int):
        """Network GEMMs (forward and training backward) on tcgen05 (1, default) or mma.sync (0)."""
        self._check(self.L.ud_mlp_set_gemm(self.h, int(kind)))

    def mlp_init(self, seed: int = 0):
        self._check(self.L.ud_mlp_init(self.h, C.c_uint64(seed & (2 ** 64 - 1))))

    def mlp_set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        if p.size != self.mlp_param_count():
            raise EngineError(f"expected {self.mlp_param_count()} parameters, got {p.size}")
        self._check(self.L.ud_mlp_set_params(self.h, _p(p)))

    def mlp_get_params(self) -> np.ndarray:
        p = np.zeros(self.mlp_param_count(), np.float32)
        self._check(self.L.ud_mlp_get_params(self.h, _p(p)))
        return p

    def mlp_forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.MLP_IN)
        out = np.zeros((x.shape[0], self.MLP_OUT), np.float32)
        self._check(self.L.ud_mlp_forward(self.h, x.shape[0], _p(x), _p(out)))
        return out

    def mlp_loss_grad(self, x, y, mask):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.MLP_IN)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, self.MLP_NDIM)
        m = np.ascontiguousarray(mask, np.float32).reshape(-1, self.MLP_NDIM)
        loss = C.c_double(0.0)
        g = np.zeros(self.mlp_param_count(), np.float32)
        self._check(self.L.ud_mlp_loss_grad(self.h, x.shape[0], _p(x), _p(y), _p(m), C.byref(loss), _p(g)))
        return float(loss.value), g

    def mlp_train(self, x, y, mask, epochs: int, batch: int = 1024, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.MLP_IN)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, self.MLP_NDIM)
        m = np.ascontiguousarray(mask, np.float32).reshape(-1, self.MLP_NDIM)
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(self.L.ud_mlp_train(self.h, x.shape[0], _p(x), _p(y), _p(m), int(epochs), int(batch), float(lr),
                                        C.c_uint64(seed), _p(losses)))
        return losses[:epochs]

    def search_learned(self, seed: int, nchain: int, mc_steps: int, opt_steps: int, p_learned: float,
                       randomize: bool = True) -> int:
        ne = C.c_longlong(0)
        self._check(self.L.ud_search_learned(self.h, C.c_uint64(seed & (2 ** 64 - 1)), int(nchain), int(mc_steps),
                                             int(opt_steps), int(randomize), float(p_learned), C.byref(ne)))
        self.nchain = nchain * self.retain
        return int(ne.value)

    def collect_moves(self, seed: int, nchain: int, mc_steps: int, opt_steps: int, max_moves: int,
                      randomize: bool = True, target: int = 0) -> int:
        """Record accepted moves of the plain search; target 0: to the next accepted pose,
        1: to the ligand's best pose at the end of the run."""
        n = C.c_int(0)
        self._check(self.L.ud_collect_moves(self.h, C.c_uint64(seed & (2 ** 64 - 1)), int(nchain), int(mc_steps),
                                            int(opt_steps), int(randomize), int(target), int(max_moves), C.byref(n)))
        self.nchain = nchain * self.retain
        return int(n.value)

    def get_moves(self, n: int):
        x = np.zeros((n, self.MLP_IN), np.float32)
        y = np.zeros((n, self.MLP_NDIM), np.float32)
        m = np.zeros((n, self.MLP_NDIM), np.float32)
        self._check(self.L.ud_get_moves(self.h, int(n), _p(x), _p(y), _p(m)))
        return x, y, m

    def mlp_train_moves(self, epochs: int, batch: int = 1024, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(self.L.ud_mlp_train_moves(self.h, int(epochs), int(batch), float(lr), C.c_uint64(seed), _p(losses)))
        return losses[:epochs]

    def score_terms(self, pose_lig, coords, mode: int = MODE_DIRECT, decomp: bool = False):
        pl = np.ascontiguousarray(pose_lig, np.int32)
        x = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float32).reshape(-1) for c in coords]))
        out = np.zeros((len(pl), 4), np.float32)
        nd = int(sum(5 * self.ligands[l].natom for l in pl))
        d = np.zeros(nd, np.float32) if decomp else None
        self._check(self.L.ud_score_terms(self.h, len(pl), _p(pl), _p(x), int(mode), _p(out), _p(d)))
        return out, d

    def bfgs_batch(self, pose_lig, records: Sequence[np.ndarray], max_steps: int, rounds: int = 1,
                   vcap: float = 10.0, slope0: float = 1e6, ramp: bool = False, mode: int = MODE_GRID):
        pl = np.ascontiguousarray(pose_lig, np.int32)
        recs = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float32) for r in records]))
        ne = np.zeros(len(pl), np.int32)
        self._check(self.L.ud_bfgs_batch(self.h, len(pl), _p(pl), _p(recs), int(max_steps), int(rounds), float(vcap),
                                          float(slope0), int(ramp), int(mode), _p(ne)))
        lens = [record_len(self.ligands[l]) for l in pl]
        out = np.split(recs, np.cumsum(lens)[:-1]) if len(lens) > 1 else [recs]
        return out, ne

    def search(self, seed: int, nchain: int, mc_steps: int, opt_steps: int, randomize: bool = True,
               mode: int = MODE_GRID) -> int:
        ne = C.c_longlong(0)
        self._check(self.L.ud_search(self.h, C.c_uint64(seed & (2 ** 64 - 1)), int(nchain), int(mc_steps),
                                     int(opt_steps), int(randomize), int(mode), C.byref(ne)))
        self.nchain = nchain * self.retain
        return int(ne.value)

    def chain_poses(self, lig: int) -> np.ndarray:
        stride = self.L.ud_record_floats(self.h, lig)
        if stride < 0:
            self._check(stride)
        out = np.zeros((self.nchain, stride), np.float32)
        self._check(self.L.ud_get_chain_poses(self.h, lig, _p(out)))
        return out

    def cluster(self, rmsd_limit: float):
        nl = len(self.ligands)
        lead = np.zeros((nl, self.nchain), np.int32)
        cnt = np.zeros(nl, np.int32)
        self._check(self.L.ud_cluster(self.h, float(rmsd_limit), _p(lead), _p(cnt)))
        return lead, cnt

    def dock(self, seed: int, nchain: int, mc_steps: int, opt_steps: int, refine_steps: int, num_pose: int,
             rmsd_limit: float, energy_range: float, randomize: bool = True, mode: int = MODE_GRID,
             final_mode: int = MODE_DIRECT, energy_decomp: bool = False,
             fetch: bool = True, p_learned: Optional[float] = None,
             refine_mode: int = MODE_DIRECT) -> Tuple[Optional[List[DockResult]], int]:
        """Dock the loaded ligands (search, clustering, refinement, filter, final scores);
        p_learned: None for the fused plain search, else the learned-proposal search;
        refine_mode: scoring of the refinement (exact pair sums by default, as the reference)."""
        p = DockParams(seed & (2 ** 64 - 1), nchain, mc_steps, opt_steps, refine_steps, num_pose, rmsd_limit,
                       energy_range, int(randomize), mode, final_mode, int(energy_decomp), int(refine_mode))
        ne = C.c_longlong(0)
        if p_learned is None:
            self._check(self.L.ud_dock(self.h, C.byref(p), C.byref(ne)))
        else:
            self._check(self.L.ud_dock_learned(self.h, C.byref(p), float(p_learned), C.byref(ne)))
        self.nchain = nchain * self.retain
        return (self.results(energy_decomp) if fetch else None), int(ne.value)

    @property
    def stream_ptr(self) -> int:
        """cudaStream_t of the context (wrap with torch.cuda.ExternalStream to time it)."""
        return int(self.L.ud_stream(self.h) or 0)

    def stage_times(self) -> np.ndarray:
        """Device ms of the last dock: search, cluster, refine, filter, final score, total."""
        t = np.zeros(6, np.float32)
        self._check(self.L.ud_stage_times(self.h, _p(t)))
        return t

    def counters(self) -> dict:
        c = np.zeros(4, np.int64)
        self._check(self.L.ud_counters(self.h, _p(c)))
        return dict(evaluations=int(c[0]), heavy_atom_evaluations=int(c[1]), launches=int(c[2]), chains=int(c[3]))

    def results(self, energy_decomp: bool = False) -> List[DockResult]:
        nl = len(self.ligands)
        cnt = np.zeros(nl, np.int32)
        self._check(self.L.ud_result_counts(self.h, _p(cnt)))
        total = self.L.ud_result_floats(self.h)
        recs = np.zeros(max(total, 1), np.float32)
        npose = int(cnt.sum())
        terms = np.zeros((max(npose, 1), 4), np.float32)
        nd = int(sum(5 * self.ligands[l].natom * int(cnt[l]) for l in range(nl)))
        dec = np.zeros(max(nd, 1), np.float32) if energy_decomp else None
        self._check(self.L.ud_get_results(self.h, _p(recs), _p(terms), _p(dec)))
        out = []
        w = 0
        k = 0
        dw = 0
        for l in range(nl):
            lig = self.ligands[l]
            stride = self.L.ud_record_floats(self.h, l)
            rl = []
            for j in range(int(cnt[l])):
                rl.append(recs[w:w + record_len(lig)].copy())
                w += stride
            t = terms[k:k + int(cnt[l])].copy()
            k += int(cnt[l])
            d = None
            if energy_decomp:
                m = 5 * lig.natom * int(cnt[l])
                d = dec[dw:dw + m].reshape(int(cnt[l]), lig.natom, 5).copy()
                dw += m
            out.append(DockResult(rl, t, d))
        return out
