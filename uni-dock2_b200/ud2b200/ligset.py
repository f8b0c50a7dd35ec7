"""Bulk ligand input: the native parser of the engine's JSON ligand schema.

``parse_ligands_bulk`` hands the whole document to ``ud_ligset_parse_json``
(libudock_b200.so), which parses it and builds every ligand's pair sets, rigid fragments
and scored intra pair lists on all host cores -- the work the reference does in C++ after
``json.dumps`` (``api/python/pipeline.cpp:125-139``,
``src/format/rapidjson_parser.cpp:54-225,227-296``).  The result, a :class:`LigandSet`,
holds the packed arrays of ``ud_add_ligands`` directly, so a batch goes to the engine
without a per-ligand Python step; single ligands are materialised on demand.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Dict, List, Sequence, Union

import numpy as np

from .model import Ligand

class LigandSet:
    """Ligands in the packed CSR layout of ``ud_add_ligands`` (document order)."""

    def __init__(self, names: List[str], arrays: Dict[str, np.ndarray]):
        self.names = names
        self.a = arrays
        self.natoms = np.diff(arrays["atom_off"]).astype(np.int32)
        self.ntors = np.diff(arrays["tors_off"]).astype(np.int32)

    def __len__(self) -> int:
        return len(self.names)

    def packed(self) -> Dict[str, np.ndarray]:
        """The arrays of ud_add_ligands (the keys and layout of engine.pack_ligands; an
        empty value array is given its minimal placeholder, as there)."""
        a = self.a
        pad = lambda v, n: v if v.size else np.zeros(n, v.dtype)
        return dict(atom_off=a["atom_off"], xyz=a["xyz"], types=a["types"], tors_off=a["tors_off"],
                    axis=pad(a["axis"], 2), dihedrals=pad(a["dihedrals"], 1), range_off=a["range_off"],
                    ranges=pad(a["ranges"], 2), rot_off=a["rot_off"], rot=pad(a["rot"], 1), pair_off=a["pair_off"],
                    pairs=pad(a["pairs"], 1), bias_off=a["bias_off"], bias=pad(a["bias"], 5))

    def __getitem__(self, i: int) -> Ligand:
        a = self.a
        if i < 0:
            i += len(self)
        a0, a1 = int(a["atom_off"][i]), int(a["atom_off"][i + 1])
        t0, t1 = int(a["tors_off"][i]), int(a["tors_off"][i + 1])
        ranges = [a["ranges"][2 * a["range_off"][k]:2 * a["range_off"][k + 1]].reshape(-1, 2).copy()
                  for k in range(t0, t1)]
        rotated = [a["rot"][a["rot_off"][k]:a["rot_off"][k + 1]].copy() for k in range(t0, t1)]
        p0 = int(a["pair_off"][a0])
        boff = a["bias_off"][a0:a1 + 1]
        b0, b1 = int(boff[0]), int(boff[-1])
        bias_atoms = np.repeat(np.arange(a1 - a0, dtype=np.int32), np.diff(boff))
        return Ligand(name=self.names[i], coords=a["xyz"][3 * a0:3 * a1].reshape(-1, 3).copy(),
                      types=a["types"][a0:a1].copy(), ff_types=a["ff_types"][a0:a1].copy(),
                      charges=a["charges"][a0:a1].copy(), axis=a["axis"][2 * t0:2 * t1].reshape(-1, 2).copy(),
                      dihedrals=a["dihedrals"][t0:t1].copy(), ranges=ranges, rotated=rotated,
                      pair_off=(a["pair_off"][a0:a1 + 1] - p0).astype(np.int32),
                      pairs=a["pairs"][p0:int(a["pair_off"][a1])].copy(),
                      bias_atoms=bias_atoms, bias_params=a["bias"][5 * b0:5 * b1].reshape(-1, 5).copy(),
                      n_pairs_1213=int(a["n_pairs_1213"][i]), n_pairs_14=int(a["n_pairs_14"][i]))

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def subset(self, idx: Sequence[int]) -> "LigandSet":
        """The ligands idx (in that order), re-packed with vectorised gathers."""
        idx = np.asarray(idx, np.int64)
        a = self.a

        def gather(off, vals, width, sel):
            # rows sel of a CSR (off over `vals` with `width` values per entry)
            lo, hi = off[sel].astype(np.int64), off[sel + 1].astype(np.int64)
            cnt = hi - lo
            new_off = np.zeros(len(sel) + 1, np.int32)
            new_off[1:] = np.cumsum(cnt)
            tot = int(new_off[-1])
            if tot == 0:
                return new_off, vals[:0].copy(), np.zeros(0, np.int64)
            start = np.repeat(lo - new_off[:-1], cnt)
            ent = np.arange(tot, dtype=np.int64) + start
            if width == 1:
                return new_off, vals[ent], ent
            cols = (ent[:, None] * width + np.arange(width)[None, :]).reshape(-1)
            return new_off, vals[cols], ent

        atom_off, _, aidx = gather(a["atom_off"], a["types"], 1, idx)
        out = dict(atom_off=atom_off, types=a["types"][aidx], ff_types=a["ff_types"][aidx],
                   charges=a["charges"][aidx],
                   xyz=a["xyz"][(aidx[:, None] * 3 + np.arange(3)[None, :]).reshape(-1)])
        tors_off, _, tidx = gather(a["tors_off"], a["dihedrals"], 1, idx)
        out["tors_off"] = tors_off
        out["dihedrals"] = a["dihedrals"][tidx]
        out["axis"] = a["axis"][(tidx[:, None] * 2 + np.arange(2)[None, :]).reshape(-1)]
        out["range_off"], out["ranges"], _ = gather(a["range_off"], a["ranges"], 2, tidx)
        out["rot_off"], out["rot"], _ = gather(a["rot_off"], a["rot"], 1, tidx)
        out["pair_off"], out["pairs"], _ = gather(a["pair_off"], a["pairs"], 1, aidx)
        out["bias_off"], out["bias"], _ = gather(a["bias_off"], a["bias"], 5, aidx)
        out["n_pairs_1213"] = a["n_pairs_1213"][idx]
        out["n_pairs_14"] = a["n_pairs_14"][idx]
        return LigandSet([self.names[int(i)] for i in idx], out)


class LigandRef:
    """Ligand i of a LigandSet: name, natom and ntors at once, every other attribute of
    the Ligand materialised on first use."""

    def __init__(self, ls: LigandSet, i: int):
        self._set = ls
        self._i = i
        self._lig = None
        self.name = ls.names[i]
        self.natom = int(ls.natoms[i])
        self.ntors = int(ls.ntors[i])

    def __getattr__(self, k):
        if k.startswith("_"):
            raise AttributeError(k)
        if self._lig is None:
            self._lig = self._set[self._i]
        return getattr(self._lig, k)


def parse_ligands_bulk(ligands: Union[Dict[str, dict], str, bytes], use_tor_lib: bool = False,
                       nthreads: int = 0) -> LigandSet:
    """All ligands of an input dict (or its JSON text) through the native parser."""
    from .engine import EngineError, load_library
    L = load_library()
    if isinstance(ligands, dict):
        doc = json.dumps(ligands).encode()
    elif isinstance(ligands, str):
        doc = ligands.encode()
    else:
        doc = bytes(ligands)
    h = C.c_void_p()
    if L.ud_ligset_parse_json(doc, C.c_size_t(len(doc)), int(bool(use_tor_lib)), int(nthreads), C.byref(h)) != 0:
        raise EngineError(L.ud_ligset_last_error().decode(errors="replace"))
    try:
        sz = np.zeros(8, np.int64)
        L.ud_ligset_sizes(h, sz.ctypes.data_as(C.c_void_p))
        nl, na, nt, nr, nrot, npair, nb, nbytes = (int(v) for v in sz)
        arr = dict(atom_off=np.zeros(nl + 1, np.int32), xyz=np.zeros(3 * na, np.float32),
                   types=np.zeros(na, np.int32), ff_types=np.zeros(na, np.int32), charges=np.zeros(na, np.float32),
                   tors_off=np.zeros(nl + 1, np.int32), axis=np.zeros(2 * nt, np.int32),
                   dihedrals=np.zeros(nt, np.float32), range_off=np.zeros(nt + 1, np.int32),
                   ranges=np.zeros(2 * nr, np.float32), rot_off=np.zeros(nt + 1, np.int32),
                   rot=np.zeros(nrot, np.int32), pair_off=np.zeros(na + 1, np.int32),
                   pairs=np.zeros(npair, np.int32), bias_off=np.zeros(na + 1, np.int32),
                   bias=np.zeros(5 * nb, np.float32), n_pairs_1213=np.zeros(nl, np.int32),
                   n_pairs_14=np.zeros(nl, np.int32))
        name_off = np.zeros(nl + 1, np.int64)
        names = C.create_string_buffer(max(1, nbytes))
        p = lambda k: arr[k].ctypes.data_as(C.c_void_p)
        rc = L.ud_ligset_export(h, p("atom_off"), p("xyz"), p("types"), p("ff_types"), p("charges"), p("tors_off"),
                                p("axis"), p("dihedrals"), p("range_off"), p("ranges"), p("rot_off"), p("rot"),
                                p("pair_off"), p("pairs"), p("bias_off"), p("bias"), p("n_pairs_1213"),
                                p("n_pairs_14"), name_off.ctypes.data_as(C.c_void_p), names)
        if rc != 0:
            raise EngineError(L.ud_ligset_last_error().decode(errors="replace"))
    finally:
        L.ud_ligset_free(h)
    raw = names.raw
    nm = [raw[name_off[i]:name_off[i + 1]].decode("utf-8") for i in range(nl)]
    return LigandSet(nm, arr)
