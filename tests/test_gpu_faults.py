"""Failure handling without any GPU fault.

The reference exits the process on any CUDA error (HANDLE_ERROR,
utils.cuh:95-100).  Here every failure is a status code and the engine stays
usable: a device allocation made to fail on the host side (the library's
fault-injection hook, the nth allocation after it is set) must surface as
LV_ERR_NOMEM from the entry point that needed it, and the same engine must
then run the same graph to the same result as a clean engine.  Nothing here
faults, traps or hangs the GPU: the failure is an error code returned by the
host-side allocation wrapper before any device memory is touched.
"""
import numpy as np
import pytest

import lvb200
from conftest import golden_mtx

pytestmark = pytest.mark.gpu

NOMEM = 4


def _same(a, b):
    assert np.array_equal(a.assignment, b.assignment)
    assert abs(a.modularity - b.modularity) < 1e-12
    assert [l["passes"] for l in a.levels] == [l["passes"] for l in b.levels]


@pytest.mark.parametrize("name", ["hub3000", "rmat11"])
def test_injected_allocation_failure_then_clean_run(name):
    """A fresh engine per position n (a warm engine reuses its buffers and
    allocates nothing), so every allocation of a whole run is reached."""
    g = lvb200.Graph.load_mtx(golden_mtx(name))
    with lvb200.Engine(rule="py") as e:
        ref = e.run(g, 1e-6)
    failed = 0
    try:
        for n in range(1, 200):
            with lvb200.Engine(rule="py") as e:
                lvb200.fail_device_alloc(n)
                try:
                    e.run(g, 1e-6)
                except lvb200.LouvainError as err:
                    assert err.status == NOMEM, str(err)
                    failed += 1
                lvb200.fail_device_alloc(0)
                _same(e.run(g, 1e-6), ref)  # the same engine, afterwards
            if failed < n:  # the run needed fewer than n allocations
                break
    finally:
        lvb200.fail_device_alloc(0)
    assert failed >= 20  # allocations of loading, level set-up and contraction


def test_injected_allocation_failure_in_batched_form():
    graphs = [lvb200.Graph.load_mtx(golden_mtx(n)) for n in ("rmat11", "planted_small",
                                                             "ring_of_cliques")]
    with lvb200.Engine(rule="py") as e:
        ref = e.batch_run(graphs, 1e-6)
    failed = 0
    try:
        for n in range(1, 200):
            with lvb200.Engine(rule="py") as e:
                lvb200.fail_device_alloc(n)
                try:
                    e.batch_run(graphs, 1e-6)
                except lvb200.LouvainError as err:
                    assert err.status == NOMEM, str(err)
                    failed += 1
                lvb200.fail_device_alloc(0)
                got = e.batch_run(graphs, 1e-6)
                for a, b in zip(got[0], ref[0]):
                    assert np.array_equal(a, b)
                assert np.allclose(got[1], ref[1], rtol=0, atol=1e-12)
            if failed < n:
                break
    finally:
        lvb200.fail_device_alloc(0)
    assert failed >= 20
