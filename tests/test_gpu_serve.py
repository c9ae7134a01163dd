"""Served form (lv_serve_*): continuous batching.  Requests submitted while
others are resident join the union at a level boundary; every result must
equal a run of the same graph alone (lv_run): the same partition and
number of levels, modularity to 1e-12 relative (per-graph sums are FP64
atomics in the union, see test_gpu_batch.py)."""
import numpy as np
import pytest

import lvb200
import lvgen
from conftest import golden_mtx, golden_names

pytestmark = pytest.mark.gpu


def _sbm_graphs(count, seed, lo=64, hi=3000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        blocks = max(1, min(int(rng.integers(4, 33)), n // 4))
        out.append(lvb200.Graph.from_edges(*lvgen.sbm(n, blocks, mean_deg=16.0,
                                                      seed=seed * 1000 + i)))
    return out


def _mix():
    graphs = [lvb200.Graph.load_mtx(golden_mtx(name)) for name in golden_names()]
    graphs += _sbm_graphs(10, 5)
    graphs.append(lvb200.Graph.from_edges(5, np.zeros(0), np.zeros(0), None))
    graphs.append(lvb200.Graph.from_edges(2, [0], [1], [1.0]))
    return graphs


def _alone(graphs, min_gain, **kw):
    with lvb200.Engine(**kw) as e:
        return [e.run(g, min_gain) for g in graphs]


def _check(alone, served, tickets):
    for a, t in zip(alone, tickets):
        r = served[t]
        assert np.array_equal(r.assignment, a.assignment), t
        assert r.levels == len(a.levels), t
        assert abs(r.modularity - a.modularity) <= 1e-12 * max(1.0, abs(a.modularity)), t
        assert r.n_communities == (int(a.assignment.max()) + 1 if len(a.assignment) else 0)
        assert r.submit_ms <= r.admit_ms <= r.done_ms


def _staggered(server, graphs, waves=(4, 6)):
    """Submits in waves with steps in between, so later graphs join while
    earlier ones are mid-run; then drains."""
    tickets, served, i = [], {}, 0
    for w in waves:
        for g in graphs[i:i + w]:
            tickets.append(server.submit(g))
        i += w
        for _ in range(2):
            server.step()
            while (x := server.poll()) is not None:
                served[x.ticket] = x
    for g in graphs[i:]:
        tickets.append(server.submit(g))
    served.update(server.drain())
    return tickets, served


@pytest.mark.parametrize("rule", ["py", "cuda"])
def test_serve_alone_vs_mix(rule):
    graphs = _mix()
    alone = _alone(graphs, 1e-6, rule=rule)
    with lvb200.Server(1e-6, 256 << 20, rule=rule) as s:
        tickets, served = _staggered(s, graphs)
        st = s.stats()
    assert st["completed"] == len(graphs)
    assert set(tickets) <= set(served)
    _check(alone, served, tickets)


def test_serve_budget_admission():
    """A budget that holds only a few graphs at a time: the others wait in
    the queue and are admitted as memory frees up."""
    graphs = _sbm_graphs(12, 6, lo=600, hi=1000)
    alone = _alone(graphs, 1e-6)
    budget = 3000 * 5 * 192  # about 3,000 vertices / 57k entries resident
    with lvb200.Server(1e-6, budget) as s:
        st0 = s.stats()
        tickets = [s.submit(g) for g in graphs]
        served, max_res, saw_queue = {}, 0, False
        while True:
            r, q = s.step()
            st = s.stats()
            assert st["resident_vertices"] <= st0["cap_vertices"]
            assert st["resident_entries"] <= st0["cap_entries"]
            max_res = max(max_res, r)
            saw_queue = saw_queue or q > 0
            while (x := s.poll()) is not None:
                served[x.ticket] = x
            if r == 0 and q == 0:
                break
    assert saw_queue and 1 <= max_res < len(graphs)
    _check(alone, served, tickets)


def test_serve_max_levels_and_threshold():
    graphs = _mix()
    alone = _alone(graphs, 0.0, max_levels=2, max_passes=40)
    with lvb200.Server(0.0, 256 << 20, max_levels=2, max_passes=40) as s:
        tickets, served = _staggered(s, graphs, waves=(3, 3))
    _check(alone, served, tickets)


def test_serve_oversized_and_empty():
    with lvb200.Server(1e-6, 64 * 232 * 4) as s:  # about sixty vertices
        big = _sbm_graphs(1, 7, lo=3000, hi=3001)[0]
        with pytest.raises(lvb200.LouvainError):
            s.submit(big)
        t = s.submit(lvb200.Graph.from_edges(0, np.zeros(0), np.zeros(0), None))
        r = s.poll()
        assert r is not None and r.ticket == t and len(r.assignment) == 0
        assert s.step() == (0, 0)


def test_serve_slot_limit():
    graphs = _sbm_graphs(9, 8, lo=100, hi=400)
    alone = _alone(graphs, 1e-6)
    with lvb200.Server(1e-6, 64 << 20, max_graphs=2) as s:
        tickets = [s.submit(g) for g in graphs]
        served = {}
        while True:
            r, q = s.step()
            assert r <= 2
            while (x := s.poll()) is not None:
                served[x.ticket] = x
            if r == 0 and q == 0:
                break
    _check(alone, served, tickets)


@pytest.mark.parametrize("background", [False, True])
def test_serve_lanes(background):
    """Three lanes routed by entry count (tiny bounds so every lane gets
    graphs), stepped by the caller or by worker threads: every result still
    equals the lone run, and the lanes' unions are independent."""
    graphs = _mix()
    alone = _alone(graphs, 1e-6)
    entries = [g.csr()[2].size for g in graphs]
    with lvb200.Server(1e-6, 512 << 20, lanes=3, background=background,
                       lane_max_entries=[2_000, 20_000], lane_share=[0.2, 0.3, 0.5]) as s:
        tickets, served = _staggered(s, graphs)
        st = s.stats()
    assert st["n_lanes"] == 3 and st["completed"] == len(graphs)
    _check(alone, served, tickets)
    for t, e in zip(tickets, entries):
        want = 0 if e <= 2_000 else (1 if e <= 20_000 else 2)
        assert served[t].lane == want
    assert len({served[t].lane for t in tickets}) == 3


def test_serve_lane_group():
    """Two unbounded lanes form a group: requests too large for lane 0 go
    to whichever of lanes 1 and 2 holds fewer entries, so both take work;
    results still equal the lone runs."""
    graphs = _mix()
    alone = _alone(graphs, 1e-6)
    entries = [g.csr()[2].size for g in graphs]
    unbounded = 2**64 - 1
    with lvb200.Server(1e-6, 512 << 20, lanes=3, background=True,
                       lane_max_entries=[2_000, unbounded, unbounded],
                       lane_share=[0.2, 0.4, 0.4]) as s:
        tickets = [s.submit(g) for g in graphs]
        served = s.drain()
    _check(alone, served, tickets)
    big = [served[t].lane for t, e in zip(tickets, entries) if e > 2_000]
    assert all(served[t].lane == 0 for t, e in zip(tickets, entries) if e <= 2_000)
    assert set(big) == {1, 2}


@pytest.mark.parametrize("background", [False, True])
def test_serve_solo_lanes(background):
    """Solo lanes run one request at a time through the single-graph path
    beside a union lane; routing by size still holds and every result
    equals the lone run, whether the lanes are stepped by the caller or by
    worker threads."""
    graphs = _mix()
    alone = _alone(graphs, 1e-6)
    entries = [g.csr()[2].size for g in graphs]
    unbounded = 2**64 - 1
    with lvb200.Server(1e-6, 512 << 20, lanes=3, background=background,
                       lane_max_entries=[2_000, unbounded, unbounded],
                       lane_share=[0.2, 0.4, 0.4], lane_solo=0b110) as s:
        tickets, served = _staggered(s, graphs)
        st = s.stats()
    assert st["completed"] == len(graphs)
    _check(alone, served, tickets)
    for t, e in zip(tickets, entries):
        assert (served[t].lane == 0) == (e <= 2_000)


def test_serve_all_solo():
    graphs = _mix()
    alone = _alone(graphs, 1e-6)
    with lvb200.Server(1e-6, 512 << 20, lanes=2, background=True,
                       lane_max_entries=[2**64 - 1, 2**64 - 1], lane_share=[0.5, 0.5],
                       lane_solo=0b11) as s:
        tickets = [s.submit(g) for g in graphs]
        served = s.drain()
    _check(alone, served, tickets)
