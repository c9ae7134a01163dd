"""Ingest and output on the device: the CSR of an edge list built by a
stable device sort (the reference reader's layout, utils.cu:168-229) and
the community listing grouped on the device (utils.cu:270-293).

Bars: the device CSR is identical, row by row in order, to the host reader's
(lv_graph_*), for every fixture (0- and 1-based files, banner lines,
duplicate lines, self-loops, isolated vertices, missing weights) and for
random edge lists with signed weights; the listing equals a host grouping
of the assignment exactly; the CLI prints the same output either way.
"""
import os
import subprocess

import numpy as np
import pytest

import lvb200
from conftest import golden_mtx, golden_names

pytestmark = pytest.mark.gpu

FIXTURES = golden_names() + ["two_cliques_zero_based", "two_cliques_banner"]


def _host_csr(g):
    n, off, col, w, _ = g.csr()
    return n, off.astype(np.uint64), col, w


def _engine_csr(e):
    n, off, col, w = e.level_csr()
    return n, off, col, w


def _same_csr(a, b):
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
    assert np.array_equal(a[3], b[3])


@pytest.mark.parametrize("name", FIXTURES)
def test_device_csr_of_mtx_equals_host_reader(name):
    host = _host_csr(lvb200.Graph.load_mtx(golden_mtx(name)))
    with lvb200.Engine() as e:
        e.load_mtx(golden_mtx(name))
        _same_csr(_engine_csr(e), host)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_device_csr_of_random_edges_equals_host(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 5000))
    m = int(rng.integers(0, 40000))
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    dst[: m // 10] = src[: m // 10]  # self-loops
    w = rng.normal(size=m).astype(np.float32)  # signed: stored as |w|
    host = _host_csr(lvb200.Graph.from_edges(n, src, dst, w))
    with lvb200.Engine() as e:
        e.load_edges(n, src, dst, w)
        _same_csr(_engine_csr(e), host)
        e.load_edges(n, src, dst)  # no weights: 1
        _same_csr(_engine_csr(e), _host_csr(lvb200.Graph.from_edges(n, src, dst)))


def test_device_csr_entry_point_and_errors():
    import ctypes

    import torch

    rng = np.random.default_rng(9)
    n, m = 100_000, 1_200_000  # several radix tiles, hubs of repeated rows
    src = (rng.zipf(1.6, m) % n).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    w = rng.uniform(0.5, 1.5, m).astype(np.float32)
    host = _host_csr(lvb200.Graph.from_edges(n, src, dst, w))
    d_src = torch.from_numpy(src.view(np.int32)).cuda()
    d_dst = torch.from_numpy(dst.view(np.int32)).cuda()
    d_w = torch.from_numpy(w).cuda()
    d_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_col = torch.zeros(2 * m, dtype=torch.int32, device="cuda")
    d_wo = torch.zeros(2 * m, dtype=torch.float32, device="cuda")
    nnz = ctypes.c_uint64()
    lvb200._check(lvb200.lib().lv_csr_from_edges_device(
        n, m, d_src.data_ptr(), d_dst.data_ptr(), d_w.data_ptr(), d_off.data_ptr(),
        d_col.data_ptr(), d_wo.data_ptr(), ctypes.byref(nnz), None))
    e = int(nnz.value)
    got = (n, d_off.cpu().numpy().view(np.uint64), d_col.cpu().numpy().view(np.uint32)[:e],
           d_wo.cpu().numpy()[:e])
    _same_csr(got, host)
    d_dst[5] = n  # an index past the vertex count
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200._check(lvb200.lib().lv_csr_from_edges_device(
            n, m, d_src.data_ptr(), d_dst.data_ptr(), d_w.data_ptr(), d_off.data_ptr(),
            d_col.data_ptr(), d_wo.data_ptr(), ctypes.byref(nnz), None))
    assert ei.value.status == 3  # LV_ERR_PARSE


def _host_grouping(asg):
    k = int(asg.max()) + 1 if len(asg) else 0
    order = np.argsort(asg, kind="stable").astype(np.uint32)
    off = np.zeros(k + 1, np.uint32)
    np.add.at(off, asg.astype(np.int64) + 1, 1)
    return np.cumsum(off).astype(np.uint32), order


@pytest.mark.parametrize("name", ["planted_small", "rmat11", "hub3000", "loops_dups_isolated"])
def test_device_listing_equals_host_grouping(name):
    with lvb200.Engine() as e:
        res = e.run(lvb200.Graph.load_mtx(golden_mtx(name)), 1e-6)
        off, members = e.communities()
    hoff, hmem = _host_grouping(res.assignment)
    assert len(off) == res.n_communities + 1
    assert np.array_equal(off, hoff)
    assert np.array_equal(members, hmem)


def test_cli_device_csr_prints_the_same(tmp_path):
    cli = os.path.join(lvb200.PKG_DIR, "bin", "louvain")
    outs = []
    for extra in ([], ["--gpu-csr"]):
        r = subprocess.run([cli, "-f", golden_mtx("planted_weighted"), "-g", "1e-6", "-v"] + extra,
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = r.stdout.splitlines()
        outs.append([lines[0]] + lines[2:])
    assert outs[0] == outs[1]
    r = subprocess.run([cli, "-f", str(tmp_path / "missing.mtx"), "-g", "1e-6", "--gpu-csr"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "Error opening file" in r.stdout
