"""Pins the CPU oracle to the reference: its louvian.py mode (FP64,
first-seen row order, decision max_gain > 0) must reproduce, bit for bit,
what louvian.py computed on every golden fixture (per-pass modularity,
level sizes, pass counts, final modularity, final communities)."""
import os

import numpy as np
import pytest

import pyoracle
from conftest import golden_mtx, golden_names, load_golden

REF_FIXTURE = os.path.join(os.environ.get("LOUVAIN_REFERENCE_DIR", "/root/reference"),
                           "tests", "bcsstk16.mtx")


@pytest.mark.parametrize("name", golden_names())
def test_oracle_reproduces_louvian_py(name):
    gold = load_golden(name)
    g = pyoracle.read_mtx(golden_mtx(name), as_float=False)
    assert g.n == gold["n_vertices"]
    res = pyoracle.louvain(g, gold["min_gain"], rule="py", prec="fp64",
                           rows="first_seen")
    assert res.q == gold["q_final"]  # exact: same FP64 operations in the same order
    assert [l.n_vertices for l in res.levels] == [l["n_vertices"] for l in gold["levels"]]
    assert [l.passes for l in res.levels] == [l["passes"] for l in gold["levels"]]
    assert np.array_equal(res.assignment, np.array(gold["assignment"], np.uint32))


@pytest.mark.parametrize("name", golden_names())
def test_oracle_pass_traces(name):
    """Every level's per-pass Q sequence equals louvian.py's printout."""
    gold = load_golden(name)
    g = pyoracle.read_mtx(golden_mtx(name), as_float=False)
    for lev in gold["levels"]:
        more, comm, trace, qs, qe = pyoracle.move_phase(g, gold["min_gain"], rule="py",
                                                       prec="fp64")
        assert qs == lev["q_start"]
        assert list(trace) == lev["q_trace"]
        assert more == lev["moved"]
        if not more:
            break
        g, _ = pyoracle.contract(g, comm, rows="first_seen", prec="fp64")


def test_zero_based_and_banner_read_identically():
    base = pyoracle.read_mtx(golden_mtx("two_cliques"))
    for variant in ("two_cliques_zero_based", "two_cliques_banner"):
        g = pyoracle.read_mtx(golden_mtx(variant))
        assert g.n == base.n
        assert np.array_equal(g.off, base.off)
        assert np.array_equal(g.col, base.col)
        assert np.array_equal(g.w, base.w)


def test_fp32_mode_stays_within_tolerance(golden):
    """The FP32 gain arithmetic (the engine's) ends within 1e-4 of the
    reference's final modularity on every fixture."""
    for name, gold in golden.items():
        g = pyoracle.read_mtx(golden_mtx(name), as_float=True)
        res = pyoracle.louvain(g, gold["min_gain"], rule="py", prec="fp32")
        assert abs(res.q - gold["q_final"]) < 1e-4, name


@pytest.mark.skipif(not os.path.exists(REF_FIXTURE),
                    reason="reference checkout not present")
def test_reference_fixture_bcsstk16():
    """louvian.py on the reference's own fixture gives Q=0.7408630099495417
    with levels 4884 -> 117 -> 86 -> 80 and 36/4/2/1 passes."""
    g = pyoracle.read_mtx(REF_FIXTURE, as_float=False)
    res = pyoracle.louvain(g, 1e-6, rule="py", prec="fp64", rows="first_seen")
    assert res.q == 0.7408630099495417
    assert [l.n_vertices for l in res.levels] == [4884, 117, 86, 80]
    assert [l.passes for l in res.levels] == [36, 4, 2, 1]
    hist = np.bincount(pyoracle.buckets(g), minlength=8)
    assert list(hist[1:7]) == [74, 0, 4, 224, 4582, 0]
    assert g.nnz == 290378 and g.max_deg == 81


def test_oracle_contract_preserves_modularity(golden):
    """Contraction keeps Q: the singleton partition of the contracted graph
    has the modularity of the partition it was built from."""
    g = pyoracle.read_mtx(golden_mtx("planted_small"))
    more, comm, trace, qs, qe = pyoracle.move_phase(g, 1e-6, rule="py", prec="fp64")
    g2, nid = pyoracle.contract(g, comm, rows="sorted", prec="fp64")
    q2 = pyoracle.modularity(g2, np.arange(g2.n, dtype=np.uint32))
    assert abs(q2 - qe) < 1e-12
    assert abs(pyoracle.modularity(g, comm) - qe) < 1e-12


def test_oracle_rules_differ_only_in_decision(golden):
    """On the reference fixture the two decision rules coincide; on a
    power-law graph they do not (the rule is a real semantic switch)."""
    g = pyoracle.read_mtx(golden_mtx("two_cliques"))
    a = pyoracle.louvain(g, 1e-6, rule="py")
    b = pyoracle.louvain(g, 1e-6, rule="cuda")
    assert a.q == b.q
