"""Parity of the CUDA engine (through the C ABI) with the oracle.

Bars:
  * integer work bit-exact: degree buckets, community sizes, renumbering and
    the contracted CSR of a given partition (rows compared as sets, as the
    reference's row order depends on atomicCAS winners);
  * whole runs: the engine's partitions equal the oracle's FP32 restatement
    exactly (same FP32 gain arithmetic), level by level;
  * final modularity within 1e-4 absolute of the reference (louvian.py's
    value stored in the golden fixtures; Louvain labels are not unique, the
    FP32/FP64 arithmetic may break ties differently).
"""
import os
import subprocess

import numpy as np
import pytest

import lvb200
import lvgen
import pyoracle
from conftest import golden_mtx, golden_names, load_golden

pytestmark = pytest.mark.gpu

Q_TOL = 1e-4


def _oracle_graph(path):
    return pyoracle.read_mtx(path, as_float=True)


@pytest.fixture(scope="module")
def eng():
    with lvb200.Engine(rule="py") as e:
        yield e


@pytest.fixture(scope="module")
def eng_cuda():
    with lvb200.Engine(rule="cuda") as e:
        yield e


def _assert_same_run(res, orc):
    assert [l["n_vertices"] for l in res.levels] == [l.n_vertices for l in orc.levels]
    assert [l["passes"] for l in res.levels] == [l.passes for l in orc.levels]
    for a, b in zip(res.levels, orc.levels):
        assert abs(a["q_start"] - b.q_start) < 1e-9
        assert abs(a["q_end"] - b.q_end) < 1e-9
    assert abs(res.modularity - orc.q) < 1e-9
    assert np.array_equal(res.assignment, orc.assignment)


@pytest.mark.parametrize("name", golden_names())
def test_run_equals_oracle_py_rule(eng, name):
    res = eng.run(lvb200.Graph.load_mtx(golden_mtx(name)), 1e-6)
    orc = pyoracle.louvain(_oracle_graph(golden_mtx(name)), 1e-6, rule="py",
                           prec="fp32", rows="sorted")
    _assert_same_run(res, orc)


@pytest.mark.parametrize("name", golden_names())
def test_run_equals_oracle_cuda_rule(eng_cuda, name):
    res = eng_cuda.run(lvb200.Graph.load_mtx(golden_mtx(name)), 1e-6)
    orc = pyoracle.louvain(_oracle_graph(golden_mtx(name)), 1e-6, rule="cuda",
                           prec="fp32", rows="sorted")
    _assert_same_run(res, orc)


@pytest.mark.parametrize("name", golden_names())
def test_final_q_within_tolerance_of_reference(eng, name):
    gold = load_golden(name)
    res = eng.run(lvb200.Graph.load_mtx(golden_mtx(name)), gold["min_gain"])
    assert abs(res.modularity - gold["q_final"]) < Q_TOL
    # the reported Q is the modularity of the returned partition
    g = _oracle_graph(golden_mtx(name))
    assert abs(pyoracle.modularity(g, res.assignment) - res.modularity) < 1e-6


@pytest.mark.parametrize("name", golden_names())
def test_buckets_and_degrees_bit_exact(eng, name):
    g = lvb200.Graph.load_mtx(golden_mtx(name))
    eng.load(g)
    og = _oracle_graph(golden_mtx(name))
    assert np.array_equal(eng.buckets(), pyoracle.buckets(og))
    comm, sz, k = eng.level_state()
    n = og.n
    assert np.array_equal(comm, np.arange(n, dtype=np.uint32))
    assert np.array_equal(sz, np.ones(n, np.uint32))
    ref_k = np.zeros(n, np.float64)
    deg = np.diff(og.off.astype(np.int64))
    np.add.at(ref_k, np.repeat(np.arange(n), deg), og.w)
    assert np.array_equal(k, ref_k.astype(np.float32))


@pytest.mark.parametrize("name", golden_names())
def test_contraction_of_given_partition_bit_exact(eng, name):
    og = _oracle_graph(golden_mtx(name))
    more, comm, _, _, _ = pyoracle.move_phase(og, 1e-6, rule="py", prec="fp32")
    g = lvb200.Graph.load_mtx(golden_mtx(name))
    eng.load(g)
    eng.set_level_comm(comm)
    _, sz, _ = eng.level_state()
    assert np.array_equal(sz, np.bincount(comm, minlength=og.n).astype(np.uint32))
    eng.phase_aggregate()
    n2, off2, col2, w2 = eng.level_csr()
    o2, nid = pyoracle.contract(og, comm, rows="sorted", prec="fp32")
    assert n2 == o2.n
    assert np.array_equal(off2, o2.off)
    for v in range(n2):
        a, b = int(off2[v]), int(off2[v + 1])
        order = np.argsort(col2[a:b], kind="stable")
        assert np.array_equal(col2[a:b][order], o2.col[a:b])
        assert np.array_equal(w2[a:b][order].astype(np.float64), o2.w[a:b])
    # assignment after aggregation = renumbered communities
    assert np.array_equal(eng.assignment(), nid[comm])


def test_modularity_fp64_of_arbitrary_partitions(eng):
    og = _oracle_graph(golden_mtx("planted_weighted"))
    eng.load(lvb200.Graph.load_mtx(golden_mtx("planted_weighted")))
    rng = np.random.default_rng(0)
    for k in (1, 7, 100, og.n):
        part = rng.integers(0, k, og.n).astype(np.uint32)
        assert abs(eng.modularity(part) - pyoracle.modularity(og, part)) < 1e-12


def test_phase_api_matches_run(eng):
    """lv_phase_move / lv_phase_aggregate driven one level at a time (as the
    reference's main.cu:43-48 drives modularityOptimization/aggregation)."""
    path = golden_mtx("planted_small")
    ref = eng.run(lvb200.Graph.load_mtx(path), 1e-6)
    eng.load(lvb200.Graph.load_mtx(path))
    q = None
    while True:
        more, q = eng.phase_move(1e-6)
        if not more:
            break
        eng.phase_aggregate()
    assert q == ref.modularity
    assert np.array_equal(eng.assignment(), ref.assignment)


@pytest.mark.parametrize("case", ["no_edges", "single_vertex", "only_loops",
                                  "isolated_pairs"])
def test_edge_cases(eng, case):
    if case == "no_edges":
        g = lvb200.Graph.from_edges(5, [], [], [])
    elif case == "single_vertex":
        g = lvb200.Graph.from_edges(1, [0], [0], [2.0])
    elif case == "only_loops":
        g = lvb200.Graph.from_edges(4, [0, 1, 2, 3], [0, 1, 2, 3], [1, 2, 3, 4])
    else:
        g = lvb200.Graph.from_edges(6, [0, 2, 4], [1, 3, 5], [1, 1, 1])
    res = eng.run(g, 1e-6)
    n, off, col, w, _ = g.csr()
    og = pyoracle.CSR(n, off, col, w.astype(np.float64))
    orc = pyoracle.louvain(og, 1e-6, rule="py", prec="fp32")
    assert abs(res.modularity - orc.q) < 1e-12
    assert np.array_equal(res.assignment, orc.assignment)


def test_nonpositive_threshold_terminates():
    """With min_gain <= 0 the reference never stops; here the pass cap and
    the "level merged nothing" rule end the run, identically to the oracle."""
    with lvb200.Engine(rule="py", max_passes=50) as e:
        res = e.run(lvb200.Graph.load_mtx(golden_mtx("ring_of_cliques")), 0.0)
    orc = pyoracle.louvain(_oracle_graph(golden_mtx("ring_of_cliques")), 0.0,
                           rule="py", prec="fp32", max_passes=50)
    assert np.array_equal(res.assignment, orc.assignment)
    assert abs(res.modularity - orc.q) < 1e-12


@pytest.mark.parametrize("kind", ["planted", "rmat", "banded", "rmat20"])
def test_bench_scale_graphs(kind):
    """Benchmark-shaped graphs at full size: the power-law workload
    (334,863 vertices), the banded FEM-like matrix (4,884 vertices, half-band
    60, about 290k stored entries, U(0.1, 1.0) weights), an R-MAT graph whose
    hubs exceed the shared-table class (several blocks per vertex), and
    R-MAT scale 20 (1,048,576 vertices, about 31 M entries, hubs of tens of
    thousands of entries)."""
    if kind == "planted":
        n, s, d, w = lvgen.planted_powerlaw(seed=0)
    elif kind == "banded":
        n, s, d, w = lvgen.banded_fem(seed=0)
    elif kind == "rmat20":
        n, s, d, w = lvgen.rmat(20, seed=0)
    else:
        n, s, d, w = lvgen.rmat(16, edge_factor=16, seed=1)
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    g = lvb200.Graph.from_csr(n, off, col, ww)
    og = pyoracle.CSR(n, off, col, ww.astype(np.float64))
    with lvb200.Engine(rule="py") as e:
        res = e.run(g, 1e-6)
    orc = pyoracle.louvain(og, 1e-6, rule="py", prec="fp32", rows="sorted")
    _assert_same_run(res, orc)
    if kind != "rmat20":
        # R-MAT 20's m (about 1.6e7) puts many candidates' gain differences
        # below FP32 resolution, so FP32 gains (the reference CUDA program's
        # arithmetic) and louvian.py's FP64 gains resolve those ties
        # differently; its louvian.py comparison runs the FP64 gain mode.
        ref = pyoracle.louvain(og, 1e-6, rule="py", prec="fp64", rows="first_seen")
        assert abs(res.modularity - ref.q) < Q_TOL
    if kind.startswith("rmat"):
        assert int(np.diff(off.astype(np.int64)).max()) > 2048
    if kind == "banded":
        assert n == 4884 and 280_000 <= len(col) <= 300_000


def test_run_device_equals_run():
    import torch

    n, s, d, w = lvgen.planted_powerlaw(n=50000, target_edges=150000, seed=3)
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    g = lvb200.Graph.from_csr(n, off, col, ww)
    with lvb200.Engine(rule="py") as e:
        ref = e.run(g, 1e-6)
        d_off = torch.from_numpy(off.view(np.int64)).cuda()
        d_col = torch.from_numpy(col.view(np.int32)).cuda()
        d_w = torch.from_numpy(ww).cuda()
        d_asg = torch.empty(n, dtype=torch.int32, device="cuda")
        r = e.run_device(n, len(col), d_off.data_ptr(), d_col.data_ptr(),
                         d_w.data_ptr(), 1e-6, d_asg.data_ptr())
        torch.cuda.synchronize()
    assert r.modularity == ref.modularity
    assert np.array_equal(d_asg.cpu().numpy().view(np.uint32), ref.assignment)


@pytest.mark.parametrize("name", ["planted_small", "rmat11", "hub3000", "star1000"])
def test_pass_loop_forms_agree(name):
    """Every way of running a level's pass loop gives the same run: the
    level graph (WHILE node, the default), the persistent level kernel with
    and without its phase timers, the host loop, and the per-pass replay of
    a captured pass (the mode kernel timing uses)."""
    out = []
    for lk, ug, prof in ((False, True, False), (True, True, False), (True, True, True),
                         (False, False, False), (False, True, True)):
        with lvb200.Engine(rule="py", use_graphs=ug, level_kernel=lk) as e:
            e.set_profiling(prof)
            out.append(e.run(lvb200.Graph.load_mtx(golden_mtx(name)), 1e-6))
    # identical runs; Q values to the last bits only, since the level
    # kernel's modularity reduction splits the sum over a different grid
    for o in out[1:]:
        assert abs(o.modularity - out[0].modularity) < 1e-12
        assert np.array_equal(o.assignment, out[0].assignment)
        assert [l["passes"] for l in o.levels] == [l["passes"] for l in out[0].levels]
        assert np.allclose([l["q_end"] for l in o.levels], [l["q_end"] for l in out[0].levels],
                           rtol=0, atol=1e-12)


@pytest.mark.parametrize("rule", ["py", "cuda"])
@pytest.mark.parametrize("gain", ["fp32", "fp64"])
def test_fused_steps_equal_apply_launches(rule, gain):
    """Bucket steps that apply their own moves into the second copy of the
    community state (the default) run exactly as steps followed by a
    separate apply launch: same partition, passes and Q, with the level
    graph and with the host loop, on a graph with every degree class and on
    one with hubs (whose decide kernel applies their moves)."""
    for kind in ("planted", "rmat"):
        if kind == "planted":
            n, s, d, w = lvgen.planted_powerlaw(n=60000, target_edges=200000, seed=5,
                                                unit=False)
        else:
            n, s, d, w = lvgen.rmat(15, edge_factor=16, seed=2)
        off, col, ww = lvgen.csr_from_edges(n, s, d, w)
        g = lvb200.Graph.from_csr(n, off, col, ww)
        res = []
        for al, ug in ((True, True), (False, True), (False, False)):
            with lvb200.Engine(rule=rule, gain=gain, apply_launch=al, use_graphs=ug) as e:
                res.append(e.run(g, 1e-6))
        for r in res[1:]:
            assert r.modularity == res[0].modularity
            assert np.array_equal(r.assignment, res[0].assignment)
            assert [l["passes"] for l in r.levels] == [l["passes"] for l in res[0].levels]
            assert [l["q_end"] for l in r.levels] == [l["q_end"] for l in res[0].levels]


@pytest.mark.parametrize("rule", ["py", "cuda"])
@pytest.mark.parametrize("gain", ["fp32", "fp64"])
def test_incremental_modularity_equals_full_sweeps(rule, gain):
    """Pass sweeps that update the intra-community weight from the moved
    vertices' rows (the default, after passes that moved under a quarter of
    the entries) give the same runs as a full sweep every pass: partition,
    passes and every level's Q, with the level graph and the host loop, on
    unit weights, U(0.1, 1) weights and R-MAT graphs with hubs.  The
    update runs on levels of at least 2^23 entries (R-MAT 19: 15.7 M at
    level 0); the small graphs check that the other levels keep full sweeps."""
    cases = [lvgen.rmat(19, seed=3),
             lvgen.planted_powerlaw(n=60000, target_edges=200000, seed=5),
             lvgen.planted_powerlaw(n=40000, target_edges=150000, seed=9, unit=False),
             lvgen.rmat(15, edge_factor=16, seed=2)]
    for n, s, d, w in cases:
        off, col, ww = lvgen.csr_from_edges(n, s, d, w)
        g = lvb200.Graph.from_csr(n, off, col, ww)
        res = []
        for full, ug in ((True, True), (False, True), (False, False)):
            with lvb200.Engine(rule=rule, gain=gain, modularity_full=full, use_graphs=ug) as e:
                res.append(e.run(g, 1e-6))
        assert sum(l["passes"] for l in res[0].levels) > 2 * len(res[0].levels)
        for r in res[1:]:
            assert np.array_equal(r.assignment, res[0].assignment)
            assert [l["passes"] for l in r.levels] == [l["passes"] for l in res[0].levels]
            assert abs(r.modularity - res[0].modularity) < 1e-12
            for a, b in zip(r.levels, res[0].levels):
                assert abs(a["q_end"] - b["q_end"]) < 1e-12


def test_fused_steps_level_state():
    """After a fused pass loop the level's state (the first copy, which the
    contraction and the level-state reads use) equals the one the separate
    apply launches leave, sizes and totals included."""
    n, s, d, w = lvgen.rmat(13, edge_factor=16, seed=4)
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    g = lvb200.Graph.from_csr(n, off, col, ww)
    states = []
    for al in (True, False):
        with lvb200.Engine(rule="py", apply_launch=al) as e:
            e.load(g)
            e.phase_move(1e-6)
            states.append(e.level_state())
    for a, b in zip(states[0], states[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("rule", ["py", "cuda"])
@pytest.mark.parametrize("gain", ["fp32", "fp64"])
def test_level_kernel_equals_level_graph_at_scale(rule, gain):
    """The power-law workload (every degree class) and an R-MAT graph with
    hubs, under both rules and both gain arithmetics."""
    for kind in ("planted", "rmat"):
        if kind == "planted":
            n, s, d, w = lvgen.planted_powerlaw(n=60000, target_edges=200000, seed=5)
        else:
            n, s, d, w = lvgen.rmat(15, edge_factor=16, seed=2)
        off, col, ww = lvgen.csr_from_edges(n, s, d, w)
        g = lvb200.Graph.from_csr(n, off, col, ww)
        res = []
        for lk, al in ((True, False), (False, False), (True, True)):
            with lvb200.Engine(rule=rule, gain=gain, level_kernel=lk, apply_launch=al) as e:
                res.append(e.run(g, 1e-6))
        for r in res[1:]:
            assert abs(res[0].modularity - r.modularity) < 1e-12
            assert np.array_equal(res[0].assignment, r.assignment)
            assert [l["passes"] for l in res[0].levels] == [l["passes"] for l in r.levels]


@pytest.mark.parametrize("apply_launch", [False, True])
def test_level_kernel_phase_timers(apply_launch):
    """With profiling on, the level kernel's barrier timestamps give every
    phase kind a device time and a count; its bucket phases apply their own
    moves unless lv_config.apply_launch asks for separate apply phases."""
    with lvb200.Engine(rule="py", level_kernel=True, apply_launch=apply_launch) as eng:
        eng.set_profiling(True)
        eng.reset_kernel_stats()
        res = eng.run(lvb200.Graph.load_mtx(golden_mtx("hub3000")), 1e-6)
        st = eng.kernel_stats()
    passes = sum(l["passes"] for l in res.levels)
    # one sweep per pass, plus each level's initial one
    assert st["modularity"]["launches"] == passes + len(res.levels)
    if apply_launch:
        assert st["apply"]["launches"] >= passes
    else:
        assert st["apply"]["launches"] == 0
    assert st["move_hub"]["launches"] >= 2
    assert all(v["total_ms"] >= 0.0 for v in st.values())
    assert st["modularity"]["total_ms"] > 0.0


def test_kernel_profiling_counts(eng):
    eng.set_profiling(True)
    eng.reset_kernel_stats()
    res = eng.run(lvb200.Graph.load_mtx(golden_mtx("rmat11")), 1e-6)
    st = eng.kernel_stats()
    eng.set_profiling(False)
    assert st["modularity"]["launches"] >= sum(l["passes"] for l in res.levels)
    assert st["contract"]["launches"] == len(res.levels) - 1
    assert all(v["total_ms"] >= 0 for v in st.values())


def test_cli_matches_reference_output_format(tmp_path):
    cli = os.path.join(lvb200.PKG_DIR, "bin", "louvain")
    gold = load_golden("planted_small")
    r = subprocess.run([cli, "-f", golden_mtx("planted_small"), "-g", "1e-6", "-v"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    q = float(lines[0])
    assert lines[0] == f"{np.float32(q):.6g}" or abs(q - gold["q_final"]) < Q_TOL
    assert abs(q - gold["q_final"]) < Q_TOL + 1e-6
    alg, total = (float(x) for x in lines[1].split())
    assert 0 <= alg <= total
    ncomm = int(lines[2])
    seen = []
    for i, ln in enumerate(lines[3:], start=1):
        parts = ln.split()
        assert int(parts[0]) == i and ln.endswith(" ")
        seen.extend(int(x) for x in parts[1:])
    assert len(lines) - 3 == ncomm
    assert sorted(seen) == list(range(1, gold["n_vertices"] + 1))


def test_cli_cache_gives_the_same_output(tmp_path):
    """--cache: the first run parses and writes <file>.lvbcsr, the second
    loads it; both print the same modularity and communities."""
    import shutil

    cli = os.path.join(lvb200.PKG_DIR, "bin", "louvain")
    mtx = str(tmp_path / "g.mtx")
    shutil.copy(golden_mtx("planted_weighted"), mtx)
    outs = []
    for _ in range(2):
        r = subprocess.run([cli, "-f", mtx, "-g", "1e-6", "-v", "--cache"],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = r.stdout.splitlines()
        outs.append([lines[0]] + lines[2:])  # line 2 holds times
        assert os.path.exists(mtx + ".lvbcsr")
    assert outs[0] == outs[1]


@pytest.mark.parametrize("name", ["planted_small", "ring_of_cliques", "hub3000"])
def test_host_waits_per_level(name):
    """A single graph on device inputs makes the host wait twice a level:
    for the level's class counts (with the hub plan's totals and the
    previous contraction's entry count and error flag riding along), and
    for the level graph's result together with the contraction's class
    sizes and the plan of its largest communities (the contraction's front
    is launched behind the level graph before its result is known).  Hubs
    and multi-block communities (hub3000) add no wait.  The results stay
    those of the oracle."""
    import torch

    g = lvb200.Graph.load_mtx(golden_mtx(name))
    n, off, col, w, _ = g.csr()
    d_off = torch.from_numpy(off.view(np.int64)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_w = torch.from_numpy(w).cuda()
    d_asg = torch.empty(n, dtype=torch.int32, device="cuda")
    with lvb200.Engine(rule="py") as e:
        e.run_device(n, len(col), d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr(), 1e-6,
                     d_asg.data_ptr())  # warm-up: buffers, level graphs
        s0 = lvb200.sync_count()
        r = e.run_device(n, len(col), d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr(), 1e-6,
                         d_asg.data_ptr())
        syncs = lvb200.sync_count() - s0
    levels = r.n_levels
    assert syncs <= 2 * levels + 2, (syncs, levels)
    orc = pyoracle.louvain(_oracle_graph(golden_mtx(name)), 1e-6, rule="py", prec="fp32",
                           rows="sorted")
    assert np.array_equal(d_asg.cpu().numpy().view(np.uint32), orc.assignment)
    assert abs(r.modularity - orc.q) < 1e-9
