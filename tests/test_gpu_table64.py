"""Transition tables of 2^31 or more edges: esl_table_build64 (int64 column pointers).

The reference's index_t = int (cuda/src/types.h:6) cannot address them.  At n = 23 the
64-bit table equals the 32-bit one (esl_table_build) entry for entry.  At n = 28 (about
3.8e9 edges, 17 GB on the device) it is checked by properties: the pointers start at 0,
never decrease and end at the edge count that esl_table_nnz gives; the count exceeds
2^31 - 1; and the columns of 4,096 seeded random states equal their expected
destinations, rebuilt from the per-state flip masks (esl_flip_masks): bits cleared high
to low, then set low to high, the reference's ascending order within a column."""
import numpy as np
import pytest

from paraexastolog_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def esl():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import paraexastolog_b200 as E
    E.lib()
    return E


@pytest.fixture(scope="module")
def ctx(esl):
    return esl.Context(0)


def _expected_column(s, f):
    down = [s ^ (1 << i) for i in range(31, -1, -1) if (f >> i) & 1 and (s >> i) & 1]
    up = [s ^ (1 << i) for i in range(32) if (f >> i) & 1 and not (s >> i) & 1]
    return down + up


def test_table64_equals_table32_n23(esl, ctx):
    net = synth.nested_canalizing_network(np.random.default_rng(23), 23, 3)
    m = esl.Model.parse(net.bnet)
    rates = synth.log_uniform_rates(np.random.default_rng(1), 23, 1)[0]
    ip32, rows32, cols32 = esl.table(ctx, m, rates, with_cols=True)
    ip64, rows64, cols64 = esl.table64(ctx, m, rates, with_cols=True)
    assert ip64.dtype == torch.int64
    assert torch.equal(ip64, ip32.to(torch.int64))
    assert torch.equal(rows64, rows32)
    assert torch.equal(cols64, cols32)


def test_table64_above_2_31_edges_n28(esl, ctx):
    n = 28
    net = synth.random_table_network(np.random.default_rng(28), n, [3], 0.5)
    m = esl.Model.parse(net.bnet)
    rates = np.ones(2 * n)
    indptr, rows, _ = esl.table64(ctx, m, rates)
    nnz = rows.numel()
    assert nnz > 2**31 - 1
    assert int(indptr[0]) == 0 and int(indptr[-1]) == nnz
    assert bool((indptr[1:] >= indptr[:-1]).all())
    F, _ = esl.flip_masks(ctx, m, rates)
    rng = np.random.default_rng(7)
    sample = np.unique(np.concatenate([rng.integers(0, 1 << n, 4096), [0, (1 << n) - 1]]))
    idx = torch.as_tensor(sample, device=F.device)
    f = F.index_select(0, idx).cpu().numpy().astype(np.uint32)
    lo = indptr.index_select(0, idx).cpu().numpy()
    hi = indptr.index_select(0, idx + 1).cpu().numpy()
    deg = np.array([bin(int(x)).count("1") for x in f])
    assert np.array_equal(hi - lo, deg)
    rows_h = {}
    for s, a, b in zip(sample, lo, hi):
        rows_h[int(s)] = rows[int(a):int(b)].cpu().numpy().tolist()
    for s, fs in zip(sample, f):
        assert rows_h[int(s)] == _expected_column(int(s), int(fs)), int(s)
