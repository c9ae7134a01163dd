"""The allocation-free modularity entry point (lv_modularity_noalloc).

It exists for callers that must not allocate device memory while they run
it — latency-bound serving loops that cannot stall in the allocator, and
processes whose device memory is owned by another allocator — and keeps its
scratch in a fixed array inside the library.  Its result must equal the regular entry point's
(lv_modularity_fp64, engine-owned scratch) on the same graph and partition,
on two calls in a row (the second call reuses the array the first one
left behind).  This file is collected last so that a stop-at-first-failure
run has already run every other test.
"""
import numpy as np
import pytest

import lvb200
import pyoracle
from conftest import golden_mtx

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the tolerance of the other modularity tests


def _device_csr(path):
    import torch

    g = lvb200.Graph.load_mtx(path)
    n, off, col, w, _ = g.csr()
    d = (torch.from_numpy(off.view(np.int64)).cuda(),
         torch.from_numpy(col.view(np.int32)).cuda(),
         torch.from_numpy(w).cuda())
    return g, n, d


@pytest.mark.parametrize("name", ["planted_weighted", "rmat11", "hub3000"])
def test_noalloc_matches_engine_entry_point(name):
    import torch

    g, n, (d_off, d_col, d_w) = _device_csr(golden_mtx(name))
    rng = np.random.default_rng(3)
    parts = [rng.integers(0, k, n).astype(np.uint32) for k in (5, n)]
    # a partition produced by the engine itself
    with lvb200.Engine(rule="py") as e:
        res = e.run(g, 1e-6)
        parts.append(res.assignment.astype(np.uint32))
        e.load(g)
        expected = [e.modularity(p) for p in parts]
    d_q = torch.zeros(1, dtype=torch.float64, device="cuda")
    for part, want in zip(parts, expected):
        d_part = torch.from_numpy(part.view(np.int32)).cuda()
        for _ in range(2):  # two calls in a row on the shared scratch
            got = lvb200.modularity_noalloc(n, d_off.data_ptr(), d_col.data_ptr(),
                                            d_w.data_ptr(), d_part.data_ptr(),
                                            d_q.data_ptr())
            assert abs(got - want) < TOL
            assert abs(float(d_q.item()) - want) < TOL
    og = pyoracle.read_mtx(golden_mtx(name))
    assert abs(expected[-1] - pyoracle.modularity(og, parts[-1])) < TOL


def test_noalloc_rejects_oversized_and_invalid_input():
    import torch

    d_q = torch.zeros(1, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(4, dtype=torch.int64, device="cuda")
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200.modularity_noalloc(lvb200.NOALLOC_MAX_VERTICES + 1, dummy.data_ptr(),
                                  dummy.data_ptr(), dummy.data_ptr(),
                                  dummy.data_ptr(), d_q.data_ptr())
    assert ei.value.status == 7  # LV_ERR_LIMIT
    g, n, (d_off, d_col, d_w) = _device_csr(golden_mtx("two_cliques"))
    bad = torch.full((n,), n + 5, dtype=torch.int32, device="cuda")
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200.modularity_noalloc(n, d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr(),
                                  bad.data_ptr(), d_q.data_ptr())
    assert ei.value.status == 1  # LV_ERR_ARG
    # the entry point still works after a rejected call
    part = torch.zeros(n, dtype=torch.int32, device="cuda")
    q = lvb200.modularity_noalloc(n, d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr(),
                                  part.data_ptr(), d_q.data_ptr())
    assert abs(q - 0.0) < TOL


def test_noalloc_on_a_caller_stream_at_the_largest_size():
    """n exactly at the limit (the top of the scratch, next to its
    accumulators), run on a caller-created stream, twice in a row."""
    import torch

    n = lvb200.NOALLOC_MAX_VERTICES
    # ring of n vertices plus chords to v + 7: every row holds 4 entries
    src = np.arange(n, dtype=np.uint32)
    s = np.concatenate([src, src])
    d = np.concatenate([(src + 1) % n, (src + 7) % n]).astype(np.uint32)
    g = lvb200.Graph.from_edges(n, s, d, np.ones(len(s), dtype=np.float32))
    nn, off, col, w, _ = g.csr()
    assert nn == n
    part = (np.arange(n, dtype=np.uint32) // 64).astype(np.uint32)
    with lvb200.Engine(rule="py") as e:
        e.load(g)
        want = e.modularity(part)
    d_off = torch.from_numpy(off.view(np.int64)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_w = torch.from_numpy(w).cuda()
    d_part = torch.from_numpy(part.view(np.int32)).cuda()
    st = torch.cuda.Stream()
    d_q = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        got = lvb200.modularity_noalloc(n, d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr(),
                                        d_part.data_ptr(), d_q.data_ptr(),
                                        stream=st.cuda_stream)
        assert abs(got - want) < TOL
        assert abs(float(d_q.item()) - want) < TOL


def test_noalloc_null_columns_and_nan_on_invalid_ids():
    import torch

    g, n, (d_off, d_col, d_w) = _device_csr(golden_mtx("two_cliques"))
    part = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_q = torch.zeros(1, dtype=torch.float64, device="cuda")
    for cols, wts in ((0, d_w.data_ptr()), (d_col.data_ptr(), 0)):
        with pytest.raises(lvb200.LouvainError) as ei:
            lvb200.modularity_noalloc(n, d_off.data_ptr(), cols, wts, part.data_ptr(),
                                      d_q.data_ptr())
        assert ei.value.status == 1  # LV_ERR_ARG
    bad = torch.arange(n, dtype=torch.int32, device="cuda")
    bad[n // 2] = n  # one id out of range
    with pytest.raises(lvb200.LouvainError) as ei:
        lvb200.modularity_noalloc(n, d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr(),
                                  bad.data_ptr(), d_q.data_ptr())
    assert ei.value.status == 1
    assert np.isnan(float(d_q.item()))
