"""The allocation-free transition-table entry point, esl_table_build_static.

It exists for callers that cannot allocate device memory while they run: code
whose framework's caching allocator already holds the GPU's memory, loops that
cannot pay for the device-wide synchronisation of cudaFree, and services that
allocate only at start-up.  Its scratch is a static device array inside the
library.  This file checks, through the C ABI, that two calls in a row give
exactly the CSC table of the allocating entry point, esl_table_build, for
different networks (so stale scratch from the first call cannot leak into the
second).  It also checks that a call leaves the device's free memory unchanged,
and that sizes beyond the stated maximum are rejected.  The file is named so that
pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MiB = 1 << 20


@pytest.fixture(scope="module")
def env():
    import torch

    import paraexastolog_b200 as esl

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")
    ctx = esl.Context(0)
    return esl, ctx, torch


def _static_table(esl, torch, model, rates, capacity=None):
    """Calls esl_table_build_static; returns (status, nnz, indptr, rows, cols)."""
    dev = "cuda:0"
    N = 1 << model.n
    cap = capacity if capacity is not None else model.n * N
    indptr = torch.full((N + 1,), -1, dtype=torch.int32, device=dev)
    rows = torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev)
    cols = torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev)
    rates = np.ascontiguousarray(rates, np.float64)
    stream = torch.cuda.current_stream(0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    nnz = C.c_int64(-1)
    st = esl.lib().esl_table_build_static(model._h, rates.ctypes.data, C.c_void_p(stream.cuda_stream),
                                          indptr.data_ptr(), rows.data_ptr(), cols.data_ptr(), cap, C.byref(nnz))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    return st, nnz.value, indptr, rows, cols, free0 - free1


def _check_same_as_allocating(esl, ctx, torch, bnet, rates):
    model = esl.Model.parse(bnet)
    ref_indptr, ref_rows, ref_cols = esl.table(ctx, model, rates)
    st, nnz, indptr, rows, cols, grown = _static_table(esl, torch, model, rates)
    assert st == esl.ESL_OK, esl.lib().esl_last_error().decode()
    assert nnz == ref_rows.numel()
    assert torch.equal(indptr, ref_indptr)
    assert torch.equal(rows[:nnz], ref_rows)
    assert torch.equal(cols[:nnz], ref_cols)
    return grown


def test_two_calls_match_allocating_entry_point(env):
    esl, ctx, torch = env
    from paraexastolog_b200 import synth

    # call 1: the n=20 precision network (the maximum size), log-uniform rates
    big = synth.config_precision()
    _check_same_as_allocating(esl, ctx, torch, big.networks[0].bnet, big.rates[0][0])
    # call 2: a different, smaller network with zero rates (other edges, other counts)
    rng = np.random.default_rng(7)
    small = synth.random_table_network(rng, 12, [2, 3], 0.5)
    rates = synth.log_uniform_rates(rng, 12, 1)[0]
    rates[[1, 4, 9]] = 0.0
    grown = _check_same_as_allocating(esl, ctx, torch, small.bnet, rates)
    assert grown < MiB, f"free device memory fell by {grown} bytes during the call"
    # and the large one again: still exact, and still no device memory taken
    grown = _check_same_as_allocating(esl, ctx, torch, big.networks[0].bnet, big.rates[0][0])
    assert grown < MiB, f"free device memory fell by {grown} bytes during the call"


def test_rejects_sizes_beyond_the_limit(env):
    esl, ctx, torch = env
    from paraexastolog_b200 import synth

    rng = np.random.default_rng(3)
    n = 21  # one node above ESL_STATIC_TABLE_MAX_NODES
    net = synth.random_table_network(rng, n, [2], 0.5)
    model = esl.Model.parse(net.bnet)
    rates = np.ones(2 * n)
    nnz = C.c_int64(-1)
    dummy = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    st = esl.lib().esl_table_build_static(model._h, rates.ctypes.data, None, dummy.data_ptr(), dummy.data_ptr(),
                                          None, 0, C.byref(nnz))
    assert st == -7  # ESL_ERR_TOO_LARGE
    assert "at most 20 nodes" in esl.lib().esl_last_error().decode()


def test_rejects_too_small_row_capacity(env):
    esl, ctx, torch = env
    from paraexastolog_b200 import synth

    w = synth.config_small()
    model = esl.Model.parse(w.networks[0].bnet)
    _, ref_rows, _ = esl.table(ctx, model, w.rates[0][0])
    st, nnz, _, rows, _, _ = _static_table(esl, torch, model, w.rates[0][0], capacity=10)
    assert st == -7
    assert nnz == ref_rows.numel()
    assert torch.all(rows == -1)  # nothing written
