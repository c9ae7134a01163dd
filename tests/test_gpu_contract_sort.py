"""Contraction by sorting (lv_config.contract_sort) against the oracle and
against the hash merge.

The reference contracts by hashing each community's member edges
(aggregation.cu:57-357); the sort form keys every entry by
(new id of its row's community, new id of its column's community), sorts
the keys stably on the device and sums each run.  Bars: for a given
partition the new vertex count, offsets, columns and FP32 weights are
bit-exact against the oracle (rows come out sorted by column, so no
reordering is needed); whole runs give the same partitions, levels and
passes as the hash merge and the oracle.
"""
import numpy as np
import pytest

import lvb200
import lvgen
import pyoracle
from conftest import golden_mtx, golden_names

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng_sort():
    with lvb200.Engine(rule="py", contract_sort=True) as e:
        yield e


@pytest.mark.parametrize("name", golden_names())
def test_sorted_contraction_of_given_partition_bit_exact(eng_sort, name):
    og = pyoracle.read_mtx(golden_mtx(name), as_float=True)
    more, comm, _, _, _ = pyoracle.move_phase(og, 1e-6, rule="py", prec="fp32")
    eng_sort.load(lvb200.Graph.load_mtx(golden_mtx(name)))
    eng_sort.set_level_comm(comm)
    eng_sort.phase_aggregate()
    n2, off2, col2, w2 = eng_sort.level_csr()
    o2, nid = pyoracle.contract(og, comm, rows="sorted", prec="fp32")
    assert n2 == o2.n
    assert np.array_equal(off2, o2.off)
    assert np.array_equal(col2, o2.col)
    assert np.array_equal(w2.astype(np.float64), o2.w)
    assert np.array_equal(eng_sort.assignment(), nid[comm])


@pytest.mark.parametrize("name", golden_names())
def test_sorted_contraction_runs_equal_oracle(eng_sort, name):
    res = eng_sort.run(lvb200.Graph.load_mtx(golden_mtx(name)), 1e-6)
    orc = pyoracle.louvain(pyoracle.read_mtx(golden_mtx(name), as_float=True), 1e-6,
                           rule="py", prec="fp32", rows="sorted")
    assert [l["passes"] for l in res.levels] == [l.passes for l in orc.levels]
    assert abs(res.modularity - orc.q) < 1e-9
    assert np.array_equal(res.assignment, orc.assignment)


@pytest.mark.parametrize("kind", ["planted", "rmat"])
def test_sorted_and_hash_contraction_give_the_same_run(kind):
    if kind == "planted":
        n, s, d, w = lvgen.planted_powerlaw(seed=0)
    else:
        n, s, d, w = lvgen.rmat(16, edge_factor=16, seed=1)
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    g = lvb200.Graph.from_csr(n, off, col, ww)
    out = []
    for cs in (False, True):
        with lvb200.Engine(rule="py", contract_sort=cs) as e:
            out.append(e.run(g, 1e-6))
    a, b = out
    assert np.array_equal(a.assignment, b.assignment)
    assert [l["passes"] for l in a.levels] == [l["passes"] for l in b.levels]
    assert [l["n_entries"] for l in a.levels] == [l["n_entries"] for l in b.levels]
    assert abs(a.modularity - b.modularity) < 1e-12
