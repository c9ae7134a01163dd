"""Autotuner (lv_autotune / lv_set_tuning): every kernel variant that can
hold a bucket's degrees gives the same proposals, so any tuning must give
the same run as the defaults -- partitions, levels and modularity
identical (the move kernels' sums are exact FP64 sums of FP32 weights and
the argmax breaks ties by community id, whatever the work mapping)."""
import itertools

import numpy as np
import pytest

import lvb200
import lvgen
from conftest import golden_mtx

pytestmark = pytest.mark.gpu

FIXTURES = ["planted_small", "planted_weighted", "hub3000", "rmat11", "sbm_small",
            "banded_small", "loops_dups_isolated"]


def _fits(k, b):
    return lvb200.KERNEL_MAX_DEGREE[k] >= lvb200.BUCKET_MAX_DEGREE[b]


def _tunings():
    smallest = [min(k for k in range(7) if _fits(k, b)) for b in range(1, 8)]
    largest = [6] * 7
    warps = [4 if _fits(4, b) else (5 if _fits(5, b) else 6) for b in range(1, 8)]
    rng = np.random.default_rng(0)
    rand = [[int(rng.choice([k for k in range(7) if _fits(k, b)])) for b in range(1, 8)]
            for _ in range(3)]
    return [smallest, largest, warps] + rand


def _same(a, b):
    assert np.array_equal(a.assignment, b.assignment)
    assert a.modularity == b.modularity
    assert [l["passes"] for l in a.levels] == [l["passes"] for l in b.levels]


@pytest.mark.parametrize("rule", ["py", "cuda"])
@pytest.mark.parametrize("name", FIXTURES)
def test_every_tuning_gives_the_same_run(name, rule):
    g = lvb200.Graph.load_mtx(golden_mtx(name))
    with lvb200.Engine(rule=rule) as e:
        ref = e.run(g, 1e-6)
        for t in _tunings():
            e.set_tuning(t)
            _same(e.run(g, 1e-6), ref)


def test_autotune_then_run():
    n, s, d, w = lvgen.planted_powerlaw(n=60_000, target_edges=170_000, seed=3)
    g = lvb200.Graph.from_edges(n, s, d, w)
    with lvb200.Engine() as e:
        ref = e.run(g, 1e-6)
        e.load(g)
        picked = e.autotune(reps=3)
        assert picked and all(ms > 0 for _, ms in picked.values())
        for b, (k, _) in picked.items():
            assert _fits(lvb200.KERNELS.index(k), b)
        assert e.tuning() == [picked.get(b, (e.tuning()[b - 1], 0))[0] for b in range(1, 8)]
        _same(e.run(g, 1e-6), ref)


def test_set_tuning_rejects_unfit_kernels():
    with lvb200.Engine() as e:
        for b in range(2, 8):
            bad = [6] * 7
            bad[b - 1] = 0  # 4-lane groups cannot hold degrees above 4
            with pytest.raises(lvb200.LouvainError):
                e.set_tuning(bad)
        assert e.tuning() == ["lanes4", "lanes8", "lanes16", "lanes32", "warp128", "warp512",
                              "block"]


def test_batch_with_tuning_equals_alone():
    graphs = [lvb200.Graph.load_mtx(golden_mtx(n)) for n in FIXTURES]
    with lvb200.Engine() as e:
        alone = [e.run(g, 1e-6) for g in graphs]
        e.set_tuning([6] * 7)
        parts, q, lv, _ = e.batch_run(graphs, 1e-6)
    for a, p in zip(alone, parts):
        assert np.array_equal(a.assignment, p)
