"""The engine's FP64 gain arithmetic (LV_GAIN_FP64) against louvian.py.

louvian.py evaluates the move gain in FP64 (louvian.py:135-138); the
reference CUDA program evaluates the same expression in FP32
(modularity.cu:149-152), which is the engine's default.  With every weight
sum exact in FP32 (integer weights, sums below 2^24) the FP64 mode must
reproduce louvian.py's runs exactly: the golden traces generated by
importing the unmodified louvian.py (partition, levels, passes, final Q),
and the oracle's louvian.py restatement on full-size graphs where no golden
file is kept (the power-law workload, R-MAT scale 20).
"""
import numpy as np
import pytest

import lvb200
import lvgen
import pyoracle
from conftest import golden_mtx, golden_names, load_golden

pytestmark = pytest.mark.gpu

Q_TOL = 1e-4
INTEGER_WEIGHTS = ["two_cliques", "ring_of_cliques", "planted_small", "rmat11"]


@pytest.fixture(scope="module")
def eng64():
    with lvb200.Engine(rule="py", gain="fp64") as e:
        yield e


@pytest.mark.parametrize("name", INTEGER_WEIGHTS)
def test_fp64_gains_reproduce_louvian_py(eng64, name):
    gold = load_golden(name)
    res = eng64.run(lvb200.Graph.load_mtx(golden_mtx(name)), gold["min_gain"])
    assert [l["n_vertices"] for l in res.levels] == [l["n_vertices"] for l in gold["levels"]]
    assert [l["passes"] for l in res.levels] == [l["passes"] for l in gold["levels"]]
    for a, b in zip(res.levels, gold["levels"]):
        assert abs(a["q_start"] - b["q_start"]) < 1e-12
        assert abs(a["q_end"] - b["q_trace"][-1]) < 1e-12
    assert abs(res.modularity - gold["q_final"]) < 1e-12
    assert np.array_equal(res.assignment, np.array(gold["assignment"], np.uint32))


@pytest.mark.parametrize("name", golden_names())
def test_fp64_gains_within_tolerance_on_every_fixture(eng64, name):
    gold = load_golden(name)
    res = eng64.run(lvb200.Graph.load_mtx(golden_mtx(name)), gold["min_gain"])
    assert abs(res.modularity - gold["q_final"]) < Q_TOL


@pytest.mark.parametrize("kind", ["planted", "rmat20"])
def test_fp64_gains_equal_louvian_restatement_at_full_size(kind):
    if kind == "planted":
        n, s, d, w = lvgen.planted_powerlaw(seed=0)
    else:
        n, s, d, w = lvgen.rmat(20, seed=0)
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    with lvb200.Engine(rule="py", gain="fp64") as e:
        res = e.run(lvb200.Graph.from_csr(n, off, col, ww), 1e-6)
    ref = pyoracle.louvain(pyoracle.CSR(n, off, col, ww.astype(np.float64)), 1e-6,
                           rule="py", prec="fp64", rows="first_seen")
    assert [l["n_vertices"] for l in res.levels] == [l.n_vertices for l in ref.levels]
    assert [l["passes"] for l in res.levels] == [l.passes for l in ref.levels]
    assert abs(res.modularity - ref.q) < 1e-9
    assert np.array_equal(res.assignment, ref.assignment)


@pytest.mark.parametrize("name", ["hub3000", "rmat11"])
def test_fp64_gains_cuda_rule_matches_oracle(name):
    """modularity.cu's decision rule with FP64 gains, hubs included."""
    with lvb200.Engine(rule="cuda", gain="fp64") as e:
        res = e.run(lvb200.Graph.load_mtx(golden_mtx(name)), 1e-6)
    ref = pyoracle.louvain(pyoracle.read_mtx(golden_mtx(name), as_float=True), 1e-6,
                           rule="cuda", prec="fp64", rows="sorted")
    assert abs(res.modularity - ref.q) < Q_TOL
    if name == "rmat11":
        assert np.array_equal(res.assignment, ref.assignment)
