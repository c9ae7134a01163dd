"""CPU tests of the C ABI library: it loads, exports every symbol the
header declares, and its host-side parts (Matrix Market reader, CSR
construction, status reporting) match the reference's reader semantics
(utils.cu:132-229) as restated by the oracle -- bit-exact CSR."""
import ctypes
import os

import numpy as np
import pytest

import lvb200
import lvgen
import pyoracle
from conftest import golden_mtx, golden_names


def test_library_exports_every_header_symbol():
    L = lvb200.lib()
    names = lvb200.header_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(lvb200._SIGS), "binding and header disagree"


def test_abi_version_and_status_strings():
    L = lvb200.lib()
    assert L.lv_abi_version() == 2
    assert L.lv_status_string(0) == b"ok"
    assert L.lv_status_string(2) == b"Error opening file"


@pytest.mark.parametrize("name", golden_names() + ["two_cliques_zero_based",
                                                   "two_cliques_banner"])
def test_mtx_reader_matches_reference_semantics(name):
    g = lvb200.Graph.load_mtx(golden_mtx(name))
    n, off, col, w, md = g.csr()
    o = pyoracle.read_mtx(golden_mtx(name), as_float=True)
    assert n == o.n and md == o.max_deg
    assert np.array_equal(off, o.off)
    assert np.array_equal(col, o.col)
    assert np.array_equal(w.astype(np.float64), o.w)


def test_from_edges_equals_mtx(tmp_path):
    n, s, d, w = lvgen.planted_powerlaw(n=500, target_edges=1500, max_deg=60,
                                        comm_min=5, comm_max=50, seed=11, unit=False)
    p = str(tmp_path / "g.mtx")
    lvgen.write_mtx(p, n, s, d, w)
    a = lvb200.Graph.load_mtx(p).csr()
    b = lvb200.Graph.from_edges(n, s, d, w).csr()
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    assert np.array_equal(a[1], off) and np.array_equal(a[2], col)
    assert np.array_equal(a[3], ww)
    c = lvb200.Graph.from_csr(n, off, col, ww).csr()
    assert np.array_equal(c[1], off) and np.array_equal(c[2], col)


def _write(tmp_path, text, name="x.mtx"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_weight_carry_over_and_abs(tmp_path):
    # a line without a weight repeats the previous one (utils.cu:289,294)
    p = _write(tmp_path, "3 3 3\n1 2 -2.5\n2 3\n3 3 0.5\n")
    n, off, col, w, _ = lvb200.Graph.load_mtx(p).csr()
    o = pyoracle.read_mtx(p, as_float=True)
    assert np.array_equal(off, o.off) and np.array_equal(col, o.col)
    assert np.array_equal(w.astype(np.float64), o.w)
    assert list(w) == [2.5, 2.5, 2.5, 2.5, 0.5]


def test_pattern_file_defaults_to_unit_weights(tmp_path):
    p = _write(tmp_path, "%%MatrixMarket matrix coordinate pattern symmetric\n"
                         "4 4 3\n2 1\n3 2\n4 4\n")
    n, off, col, w, _ = lvb200.Graph.load_mtx(p).csr()
    assert n == 4 and list(off) == [0, 1, 3, 4, 5]
    assert list(col) == [1, 0, 2, 1, 3]
    assert np.all(w == 1.0)


@pytest.mark.parametrize("text,status", [
    ("", 3),
    ("% only a comment\n", 3),
    ("3 3\n1 2 1\n", 3),
    ("3 3 2\n1 2 1\n", 3),          # fewer entry lines than nnz
    ("3 3 1\n1 4 1\n", 3),          # index past the vertex count
    ("3 3 1\n1 x 1\n", 3),          # malformed index
    ("3 3 1\n1 2 abc\n", 3),        # malformed weight
])
def test_reader_errors_are_status_codes(tmp_path, text, status):
    p = _write(tmp_path, text)
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200.Graph.load_mtx(p)
    assert ei.value.status == status
    # the oracle rejects the same inputs
    with pytest.raises(pyoracle.OracleError):
        pyoracle.read_mtx(p)


def test_missing_file_is_io_error(tmp_path):
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200.Graph.load_mtx(str(tmp_path / "nope.mtx"))
    assert ei.value.status == 2
    assert "Error opening file" in str(ei.value)


def test_csr_validation():
    with pytest.raises(lvb200.LouvainError):
        lvb200.Graph.from_csr(2, np.array([0, 2, 1], np.uint64),
                              np.array([1, 0], np.uint32), np.ones(2, np.float32))
    with pytest.raises(lvb200.LouvainError):
        lvb200.Graph.from_csr(2, np.array([0, 1, 2], np.uint64),
                              np.array([1, 5], np.uint32), np.ones(2, np.float32))


def test_engine_without_device_fails_loudly():
    """With no usable CUDA device the engine reports an error status; there
    is no CPU fallback."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200.Engine()
    assert ei.value.status in (5, 4)


def test_cli_usage_and_missing_file(tmp_path):
    import subprocess

    cli = os.path.join(lvb200.PKG_DIR, "bin", "louvain")
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stdout.strip() == "Usage: ./gpulouvain -f mtx-matrix-file -g min-gain [-v]"
    r = subprocess.run([cli, "-f", str(tmp_path / "none.mtx"), "-g", "1e-6"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout.strip() == "Error opening file"
    r = subprocess.run([cli, "-f", "x", "-g", "abc"], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stdout.strip() == "-g option invalid argument: stof"


def test_pack_graphs_block_diagonal():
    """The batched input layout: graph g's rows and column ids are shifted
    by its vertex offset, entry order kept."""
    parts = [lvgen.two_cliques_bridge(4), lvgen.star(7), (3, np.zeros(0), np.zeros(0),
                                                          np.zeros(0, np.float32))]
    csrs = [(n,) + tuple(lvgen.csr_from_edges(n, s, d, w)) for n, s, d, w in parts]
    goff, off, col, w = lvb200.pack_graphs(csrs)
    assert goff.tolist() == [0, 8, 16, 19]
    assert off[-1] == len(col) == sum(len(c[2]) for c in csrs)
    for g, (n, o, c, x) in enumerate(csrs):
        vb = int(goff[g])
        rows = off[vb:vb + n + 1] - off[vb]
        assert np.array_equal(rows, o - o[0])
        seg = slice(int(off[vb]), int(off[vb + n]))
        assert np.array_equal(col[seg], c.astype(np.uint32) + vb)
        assert np.array_equal(w[seg], x)
        assert (col[seg] >= vb).all() and (col[seg] < vb + n).all()


def test_binary_csr_round_trip(tmp_path):
    """lv_graph_save / lv_graph_load give back the same CSR; damaged files
    are rejected."""
    n, s, d, w = lvgen.planted_powerlaw(n=3000, target_edges=9000, seed=5, unit=False)
    mtx = str(tmp_path / "g.mtx")
    lvgen.write_mtx(mtx, n, s, d, w)
    g = lvb200.Graph.load_mtx(mtx)
    path = str(tmp_path / "g.lvbcsr")
    g.save(path)
    h = lvb200.Graph.load(path)
    a, b = g.csr(), h.csr()
    assert a[0] == b[0] and a[4] == b[4]
    for x, y in zip(a[1:4], b[1:4]):
        assert np.array_equal(x, y)
    raw = open(path, "rb").read()
    bad = str(tmp_path / "bad.lvbcsr")
    for blob in (raw[:40], b"XXXXXXXX" + raw[8:], raw[:-4]):
        open(bad, "wb").write(blob)
        with pytest.raises(lvb200.LouvainError):
            lvb200.Graph.load(bad)


def test_parallel_reader_weights_carry_across_chunks(tmp_path):
    """A multi-chunk file (the reader splits large files across threads)
    whose lines alternate between explicit and missing weights reads the
    same as the oracle's serial reader."""
    rng = np.random.default_rng(1)
    n, m = 50_000, 400_000
    src = rng.integers(1, n + 1, m)
    dst = rng.integers(1, n + 1, m)
    path = str(tmp_path / "big.mtx")
    with open(path, "w") as f:
        f.write(f"{n} {n} {m}\n")
        for i in range(m):
            if (i // 7) % 3 == 0:
                f.write(f"{src[i]} {dst[i]}\n")
            else:
                f.write(f"{src[i]} {dst[i]} {rng.uniform(-2, 2):.6f}\n")
    g = lvb200.Graph.load_mtx(path)
    o = pyoracle.read_mtx(path, as_float=True)
    n2, off, col, w, _ = g.csr()
    assert n2 == o.n
    assert np.array_equal(off, np.asarray(o.off))
    assert np.array_equal(col, np.asarray(o.col))
    assert np.array_equal(w, np.asarray(o.w).astype(np.float32))
