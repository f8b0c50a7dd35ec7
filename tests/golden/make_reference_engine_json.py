"""Writes tests/golden/ref_engine_small_<batch>.json, and ref_engine_small_decomp_ /
_constraint_ / _bias_ / _align_<batch>.json (energy_decomp on; constraint docking; bias records
with bias 'pos', k = 0.5, and 'align', k = 0.1): the output files of the reference's own CUDA
engine
(core_pipeline, built from its sources into oracle/_ref/udref_dock by `make -C oracle refengine`)
for the small test system (the `small_system` fixture of tests/conftest.py: 600-atom synthetic
receptor, five ligands of 8-41 atoms) at 32 chains x 20 MC steps.  Needs a GPU and the built
udref_dock; the CPU tests read the committed files (one per size-group batch the reference
makes, src/screening/screening.cpp:17-41).

    python tests/golden/make_reference_engine_json.py [out_dir]
"""
import glob
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "uni-dock2_b200"))


def bias_ligands(ligd):
    """The ligands with positional bias records ([x, y, z, V, r2] per atom, the input schema's
    optional 9th atom field) on every third atom, two on every sixth (seeded)."""
    import copy
    import numpy as np
    rng = np.random.default_rng(17)
    out = copy.deepcopy(ligd)
    for lig in out.values():
        for k, atom in enumerate(lig["atoms"]):
            if k % 3 == 0:
                recs = [[atom[0] + float(rng.uniform(-1, 1)), atom[1] + float(rng.uniform(-1, 1)),
                         atom[2] + float(rng.uniform(-1, 1)), float(rng.uniform(-2, 2)), float(rng.uniform(0.5, 3.0))]]
                if k % 6 == 0:
                    recs.append([atom[0], atom[1] + 0.5, atom[2], -1.0, 1.5])
                atom[:] = list(atom[:8]) + [recs]
    return out


def main(out_dir):
    from ud2b200 import synth
    rows, center = synth.make_receptor(600, 28.0, seed=3)
    ligd = {f"l{i}": synth.make_ligand(n, t, seed=100 + i, center=center)
            for i, (n, t) in enumerate([(8, 0), (14, 2), (20, 4), (30, 6), (41, 9)])}
    exe = os.path.join(ROOT, "oracle", "_ref", "udref_dock")
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "input.json")
        with open(inp, "w") as f:
            json.dump(dict(receptor=rows, **ligd), f)
        inp_bias = os.path.join(tmp, "input_bias.json")
        with open(inp_bias, "w") as f:
            json.dump(dict(receptor=rows, **bias_ligands(ligd)), f)
        c = [str(float(v)) for v in center]
        # (input, constraint, extra arguments, output prefix): plain; energy_decomp (per-atom
        # inter energy terms in the output); constraint docking; positional bias (k = 0.5);
        # z-align bias (k = 0.1)
        runs = ((inp, "0", ["0"], "ref_engine_small_"), (inp, "0", ["1"], "ref_engine_small_decomp_"),
                (inp, "1", ["0"], "ref_engine_small_constraint_"),
                (inp_bias, "0", ["0", "pos", "0.5"], "ref_engine_small_bias_"),
                (inp_bias, "0", ["0", "align", "0.1"], "ref_engine_small_align_"))
        for k, (src_in, constraint, extra, prefix) in enumerate(runs):
            out = os.path.join(tmp, f"out{k}")
            os.makedirs(out)
            cmd = [exe, src_in, out, *c, "20.0", "20.0", "20.0", "32", "20", "14", "2", "4", "1.0", "10.0", "5",
                   constraint, *extra]
            subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=600)
            files = sorted(glob.glob(os.path.join(out, "udref_*.json")))
            assert files
            for fp in files:
                batch = os.path.basename(fp)[len("udref_"):]
                with open(fp) as src, open(os.path.join(out_dir, prefix + batch), "w") as dst:
                    dst.write(src.read())


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
