"""The native bulk ligand parser (ud_ligset_parse_json) and the memory-bounded launch plan.

* the reference's own parser test (test/unit/format/test_json.cpp:9-71 on
  test/data/dev1/simple.json): atom counts, centres, dihedrals and the sizes of the
  1-2/1-3, 1-4 and scored-pair sets, for the bulk parser and the per-ligand parser;
* the bulk parser's packed arrays equal, entry for entry, those of the per-ligand parser
  (model.parse_ligands + engine.pack_ligands) on synthetic ligands of every workload
  (with and without the torsion library) and on the real molecules of the reference's
  acceptance cases (hydrogens, ring systems, bias records);
* reserved keys, names with escapes, malformed documents; subsets re-packed;
* launch plans: size groups kept apart, the budget respected, every ligand once.
"""
import json
import os
import time

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def _same_packed(ligs, ls):
    from ud2b200.engine import pack_ligands
    a, b = pack_ligands(ligs), ls.packed()
    bad = [k for k in a if not (a[k].dtype == b[k].dtype and np.array_equal(a[k], b[k]))]
    assert not bad, bad
    for i, l in enumerate(ligs):
        m = ls[i]
        assert m.name == l.name
        assert (m.n_pairs_1213, m.n_pairs_14) == (l.n_pairs_1213, l.n_pairs_14)
        assert np.array_equal(m.ff_types, l.ff_types) and np.array_equal(m.charges, l.charges)
        assert np.array_equal(m.bias_atoms, l.bias_atoms) and np.array_equal(m.bias_params, l.bias_params)


def test_reference_parser_test_counts():
    """test_json.cpp:9-71 on simple.json, for both parsers (its rotated-atom indices lie
    outside the ligands: only the parser sees them)."""
    from ud2b200.ligset import parse_ligands_bulk
    from ud2b200.model import DEG2RAD_F, F32, parse_ligands
    doc = _load("ref_simple.json")
    ls = parse_ligands_bulk(doc)
    py = parse_ligands(doc)
    assert ls.names == ["lig1", "lig2"] == [l.name for l in py]
    want = [dict(natom=3, center=(65.484336, 14.577332, 43.487335), dihe=(177.0, 70.0), n1213=8, n14=9, intra=2),
            dict(natom=2, center=(63.788497, 12.872499, 41.792999), dihe=(-13.5, 110.0), n1213=5, n14=6, intra=2)]
    for lig in (ls[0], ls[1]), py:
        for l, w in zip(lig, want):
            assert l.natom == w["natom"] and l.ntors == 2
            np.testing.assert_allclose(l.center, w["center"], atol=1e-4)
            assert [float(x) for x in l.dihedrals] == [float(F32(F32(d) * DEG2RAD_F)) for d in w["dihe"]]
            assert l.n_pairs_1213 == w["n1213"] and l.n_pairs_14 == w["n14"]
            assert len(l.pairs) == w["intra"] and len(l.pair_off) == l.natom + 1
    _same_packed(py, ls)


@pytest.mark.parametrize("workload", ["small", "screen", "uneven", "template"])
@pytest.mark.parametrize("tor_lib", [False, True])
def test_bulk_matches_per_ligand_parser_on_workloads(workload, tor_lib):
    from ud2b200 import synth
    from ud2b200.ligset import parse_ligands_bulk
    from ud2b200.model import parse_ligands
    w = synth.WORKLOADS[workload]
    _, center = synth.make_receptor(50, w["cube"], 1)
    sizes = synth.ligand_sizes(workload, 120, 5)
    core = synth.make_core(center, 5) if workload == "template" else None
    d = {f"{workload}_{i}": synth.make_ligand(n, t, 5 * 7919 + i, center, core=core) for i, (n, t) in enumerate(sizes)}
    if tor_lib:      # ranges that cross +-180 and invalid ones, as real torsion libraries give
        rng = np.random.default_rng(1)
        for v in d.values():
            for tor in v["torsions"]:
                tor[2] = [[-180.0, -150.0], [170.0, -170.0], [30.0, 10.0], [-20.0, float(rng.uniform(0, 40))]]
    _same_packed(parse_ligands(d, tor_lib), parse_ligands_bulk(d, tor_lib))


@pytest.mark.parametrize("fixture", ["ref_5s8i.json", "ref_bias_hbond.json", "ref_1w1p.json"])
def test_bulk_matches_per_ligand_parser_on_reference_molecules(fixture):
    from ud2b200.ligset import parse_ligands_bulk
    from ud2b200.model import parse_ligands
    ligd = _load(fixture)["ligands"]
    ls = parse_ligands_bulk(ligd)
    py = parse_ligands(ligd)
    _same_packed(py, ls)
    assert np.any(ls.a["types"] == 0)                    # hydrogens are kept in the topology


def test_reserved_keys_names_and_errors():
    from ud2b200 import synth
    from ud2b200.engine import EngineError
    from ud2b200.ligset import parse_ligands_bulk
    from ud2b200.model import parse_ligands
    _, c = synth.make_receptor(50, 30.0, 1)
    lig = synth.make_ligand(12, 2, 3, c)
    doc = {"score": ["vina"], "lié \"q\"/\\x": lig, "receptor": [[0, 0, 0, 2, 0, 0.0]], "b中": lig}
    ls = parse_ligands_bulk(doc)
    assert ls.names == ["lié \"q\"/\\x", "b中"]
    _same_packed(parse_ligands(doc), ls)
    text = json.dumps(doc, indent=2, ensure_ascii=True)          # escapes and whitespace
    assert parse_ligands_bulk(text).names == ls.names
    for bad in ['{"a": {"atoms": [[1, 2, 3, 4, 0, 0.1, [], []]', '{"a": {"torsions": []}}', '[1, 2]',
                '{"a": {"atoms": [[1, 2, 3, 4.5, 0, 0.1, [], []]]}}', '{"a": {"atoms": [[1, 2, 3]]}} x']:
        with pytest.raises(EngineError, match="ligand JSON"):
            parse_ligands_bulk(bad)
    assert len(parse_ligands_bulk("{}")) == 0


def test_subset_repacks_the_chosen_ligands():
    from ud2b200 import synth
    from ud2b200.engine import pack_ligands
    from ud2b200.ligset import parse_ligands_bulk
    from ud2b200.model import parse_ligands
    _, c = synth.make_receptor(50, 30.0, 1)
    sizes = synth.ligand_sizes("uneven", 40, 9)
    d = {f"u{i}": synth.make_ligand(n, t, 9000 + i, c) for i, (n, t) in enumerate(sizes)}
    d["hb"] = _load("ref_bias_hbond.json")["ligands"]["MOL_0"]      # bias records and hydrogens
    ls = parse_ligands_bulk(d)
    py = parse_ligands(d)
    idx = [40, 3, 17, 0, 39, 17]
    sub = ls.subset(idx)
    a, b = pack_ligands([py[i] for i in idx]), sub.packed()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert sub.names == [py[i].name for i in idx]


def test_bulk_parse_of_65536_ligands():
    """65,536 config-2-like ligands (lognormal sizes 8-80 atoms, 0-20 torsions) from their
    JSON text: parsed, fragments and pair lists built, exported to packed arrays."""
    from ud2b200 import synth
    from ud2b200.ligset import parse_ligands_bulk
    _, c = synth.make_receptor(50, 30.0, 1)
    sizes = synth.ligand_sizes("uneven", 256, 3)
    parts = [json.dumps(synth.make_ligand(n, t, 3000 + i, c)) for i, (n, t) in enumerate(sizes)]
    text = "{" + ",".join(f'"m{i}":{parts[i % len(parts)]}' for i in range(65536)) + "}"
    t0 = time.perf_counter()
    ls = parse_ligands_bulk(text)
    dt = time.perf_counter() - t0
    print(f"bulk parse of 65,536 ligands ({len(text) / 1e6:.0f} MB of JSON): {dt:.3f} s on {os.cpu_count()} cores")
    assert len(ls) == 65536 and ls.natoms.sum() == sum(sizes[i % 256][0] for i in range(65536))
    one = parse_ligands_bulk("{" + f'"m0":{parts[0]}' + "}")
    assert np.array_equal(ls[256].pairs, one[0].pairs)
    assert dt < 5.0


def test_launch_plan_keeps_groups_budget_and_order():
    from ud2b200.batching import plan_launches, predict_dock_bytes, reference_batches
    rng = np.random.default_rng(4)
    na = rng.integers(8, 100, 5000)
    nt = rng.integers(0, 20, 5000)
    ref = reference_batches(na, nt)
    assert all(len(b) <= 1000 for _, b in ref)
    per = predict_dock_bytes(na, nt, na * 4, nt * 5, nt, np.zeros(5000, int), nchain=128)
    for budget in (int(per.sum()) * 2, int(per.sum()) // 7, int(per.max()) + 1):
        plan = plan_launches(ref, per, budget)
        flat = [i for run in plan for i in run]
        assert flat == [i for _, b in ref for i in b]                  # every ligand once, in batch order
        group = {i: g for g, b in ref for i in b}
        for run in plan:
            assert len({group[i] for i in run}) == 1                  # one size group per launch
            assert per[run].sum() <= budget
    assert len(plan_launches(ref, per, int(per.sum()) * 2)) == len({g for g, _ in ref})
    with pytest.raises(MemoryError):
        plan_launches(ref, per, int(per.max()) - 1)
