"""Batched form: many graphs packed into one block-diagonal union and run
together give, graph by graph, the result of running each graph alone
(lv_run): the same partition, the same number of levels, and the same
modularity.

Each graph keeps its own m, modularity and stop rule inside the batch, so
partitions and level counts are compared exactly.  Per-graph modularity is
summed with FP64 atomics in the batch (a fixed-order reduction alone), so
it may differ from the single-graph value, and from one batched run to the
next, in the last bits when squared community totals round; it is compared
to 1e-12 relative, and bit-exactly on unit-weight graphs, whose totals and
squares are exact integers.  (Moves never read modularity; only the stop
rule does, so a partition could differ only if a pass's gain fell within
those last bits of the threshold.)
"""
import numpy as np
import pytest

import lvb200
import lvgen
from conftest import golden_mtx, golden_names

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _sbm_mix(count, seed, lo=64, hi=4096):
    """SBM graphs with log-uniform sizes, 4-32 blocks, weights U(0.5, 1.5)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        blocks = int(rng.integers(4, 33))
        blocks = max(1, min(blocks, n // 4))
        out.append(lvgen.sbm(n, blocks, mean_deg=16.0, seed=seed * 1000 + i))
    return out


def _graphs(edge_lists):
    return [lvb200.Graph.from_edges(n, s, d, w) for n, s, d, w in edge_lists]


def _mix():
    graphs = [lvb200.Graph.load_mtx(golden_mtx(name)) for name in golden_names()]
    graphs += _graphs(_sbm_mix(12, 1))
    # edgeless, a single vertex with a self-loop, an isolated pair
    graphs.append(lvb200.Graph.from_edges(5, np.zeros(0), np.zeros(0), None))
    graphs.append(lvb200.Graph.from_edges(1, [0], [0], [2.0]))
    graphs.append(lvb200.Graph.from_edges(2, [0], [1], [1.0]))
    return graphs


def _alone(graphs, min_gain, **kw):
    with lvb200.Engine(**kw) as e:
        return [e.run(g, min_gain) for g in graphs]


def _assert_batch_equals_alone(graphs, alone, parts, q, lv, exact_q=False):
    for g, a in enumerate(alone):
        assert np.array_equal(parts[g], a.assignment), f"graph {g}"
        assert lv[g] == len(a.levels), f"graph {g}"
        if exact_q:
            assert q[g] == a.modularity, f"graph {g}"
        else:
            assert abs(q[g] - a.modularity) <= 1e-12 * max(1.0, abs(a.modularity)), f"graph {g}"


@pytest.mark.parametrize("rule", ["py", "cuda"])
@pytest.mark.parametrize("use_graphs", [True, False])
def test_batch_equals_alone(rule, use_graphs):
    graphs = _mix()
    alone = _alone(graphs, 1e-6, rule=rule, use_graphs=use_graphs)
    with lvb200.Engine(rule=rule, use_graphs=use_graphs) as e:
        parts, q, lv, r = e.batch_run(graphs, 1e-6)
    _assert_batch_equals_alone(graphs, alone, parts, q, lv)
    assert r.n_vertices == sum(len(p) for p in parts)
    assert r.n_communities == sum(int(p.max()) + 1 if len(p) else 0 for p in parts)


def test_batch_unit_weights_bit_exact():
    edge_lists = []
    for i, (n, s, d, w) in enumerate(_sbm_mix(10, 2)):
        edge_lists.append((n, s, d, np.ones_like(w)))
    edge_lists.append(lvgen.ring_of_cliques(10, 5))
    edge_lists.append(lvgen.two_cliques_bridge(6))
    graphs = _graphs(edge_lists)
    alone = _alone(graphs, 1e-6)
    with lvb200.Engine() as e:
        parts, q, lv, _ = e.batch_run(graphs, 1e-6)
    _assert_batch_equals_alone(graphs, alone, parts, q, lv, exact_q=True)


@pytest.mark.parametrize("max_levels", [1, 2])
def test_batch_max_levels(max_levels):
    graphs = _mix()
    alone = _alone(graphs, 1e-6, max_levels=max_levels)
    with lvb200.Engine(max_levels=max_levels) as e:
        parts, q, lv, _ = e.batch_run(graphs, 1e-6)
    _assert_batch_equals_alone(graphs, alone, parts, q, lv)
    assert max(lv) <= max_levels


def test_batch_nonpositive_threshold():
    """Threshold 0: a level that merges nothing ends the graph's run."""
    graphs = [lvb200.Graph.load_mtx(golden_mtx(n))
              for n in ("ring_of_cliques", "two_cliques", "sbm_small")]
    alone = _alone(graphs, 0.0, max_passes=50)
    with lvb200.Engine(max_passes=50) as e:
        parts, q, lv, _ = e.batch_run(graphs, 0.0)
    _assert_batch_equals_alone(graphs, alone, parts, q, lv)


def test_batch_repeated_and_order():
    """Two batches in a row on one engine, and the same graphs in reverse
    order, give the same per-graph results."""
    graphs = _graphs(_sbm_mix(16, 3))
    with lvb200.Engine() as e:
        p1, q1, l1, _ = e.batch_run(graphs, 1e-6)
        p2, q2, l2, _ = e.batch_run(graphs, 1e-6)
        p3, q3, l3, _ = e.batch_run(graphs[::-1], 1e-6)
    for g in range(len(graphs)):
        assert np.array_equal(p1[g], p2[g]) and l1[g] == l2[g]
        assert abs(q1[g] - q2[g]) <= 1e-12
        r = len(graphs) - 1 - g
        assert np.array_equal(p1[g], p3[r]) and l1[g] == l3[r]
        assert abs(q1[g] - q3[r]) <= 1e-12


def test_batch_device_equals_host():
    edge_lists = _sbm_mix(20, 4)
    csrs = [lvgen.csr_from_edges(n, s, d, w) for n, s, d, w in edge_lists]
    goff, off, col, w = lvb200.pack_graphs(
        [(n,) + tuple(c) for (n, _, _, _), c in zip(edge_lists, csrs)])
    N, E = int(goff[-1]), len(col)
    dev = torch.device("cuda:0")
    d_off = torch.from_numpy(off.view(np.int64)).to(dev)
    d_col = torch.from_numpy(col.view(np.int32)).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_out = torch.zeros(N, dtype=torch.int32, device=dev)
    graphs = _graphs(edge_lists)
    with lvb200.Engine() as e:
        q, lv, r = e.batch_run_device(goff, N, E, d_off.data_ptr(), d_col.data_ptr(),
                                      d_w.data_ptr(), 1e-6, d_out.data_ptr())
        torch.cuda.synchronize()
        parts, qh, lh, _ = e.batch_run(graphs, 1e-6)
    out = d_out.cpu().numpy().view(np.uint32)
    for g in range(len(edge_lists)):
        assert np.array_equal(out[goff[g]:goff[g + 1]], parts[g])
        # per-graph Q of a union is summed with FP64 atomics: last bits only
        assert abs(q[g] - qh[g]) <= 1e-12 * max(1.0, abs(qh[g])) and lv[g] == lh[g]


def test_batch_bad_offsets():
    dev = torch.device("cuda:0")
    d_off = torch.zeros(4, dtype=torch.int64, device=dev)
    d_out = torch.zeros(3, dtype=torch.int32, device=dev)
    with lvb200.Engine() as e:
        for goff in ([0, 5, 3], [1, 2, 3], [0, 1, 2]):  # decreasing, bad start, bad end
            with pytest.raises(lvb200.LouvainError):
                e.batch_run_device(np.array(goff, dtype=np.uint64), 3, 0, d_off.data_ptr(),
                                   0, 0, 1e-6, d_out.data_ptr())
        with pytest.raises(lvb200.LouvainError):
            e.batch_run([], 1e-6)
