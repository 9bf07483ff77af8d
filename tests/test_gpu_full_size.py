"""The drop-in and precision workloads at their full sizes.

n = 22 drop-in case (4,194,304 states, 535,520 SCCs, a 368,384-state transient SCC):
the integer stages are bit-exact against the oracle (flip masks; order, offsets,
levels and canonical labels), and the FP64 solve is checked through size-independent
properties instead of a full oracle solve:
  - the occupation z solves (Q - A) z = x0 on the transient states (relative L1 1e-8);
  - each terminal SCC's mass equals x0 on it plus the rate-weighted flux of z into it
    (1e-9 absolute per terminal);
  - x_inf is stationary inside each terminal SCC (balance residual 1e-10), is >= 0,
    sums to 1 (1e-12), is zero on transient states, and the marginals are its bit sums.
n = 20 precision case (the learned workload's network): the mixed method is within
L1 <= 1e-10 of the FP64 oracle, as the precision configuration asks.
"""
import numpy as np
import pytest

import oracle as O
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


def _edge_rates(n, F, r):
    """rate of edge v -> v ^ (1 << i) for every state and bit, 0 where there is none"""
    v = np.arange(F.size, dtype=np.int64)
    out = np.zeros((n, F.size))
    for i in range(n):
        has = ((F >> i) & 1).astype(bool)
        out[i] = np.where(has, r[2 * i + ((v >> i) & 1)], 0.0)
    return out


def test_n22_drop_in_full_size(esl, ctx):
    w = synth.config_scale()
    text, r, x0 = w.networks[0].bnet, w.rates[0][0], w.x0[0][0]
    n, N = 22, 1 << 22
    om = O.Model(text=text)
    m = esl.Model.parse(text)
    F_ref = om.flip_masks(r)
    F, _ = esl.flip_masks(ctx, m, r)
    assert np.array_equal(F.cpu().numpy().astype(np.uint32), F_ref)
    sym = om.analyse(r)
    net = esl.Net.build(ctx, m, r)
    order, offsets, levels, labels = [t.cpu().numpy() for t in net.export()]
    assert (net.n_sccs, net.T) == (sym.n_sccs, sym.T)
    assert np.array_equal(order, sym.order) and np.array_equal(offsets, sym.offsets)
    assert np.array_equal(levels, sym.levels) and np.array_equal(labels, sym.labels)

    occ = torch.empty((1, N), dtype=torch.float64, device="cuda")
    res = esl.solve_batch(ctx, net, r, x0, method=esl.METHOD_DIRECT, tol=1e-12, occupation=occ)
    assert res.report.converged == 1
    xi = res.x_inf[0, 0].cpu().numpy()
    mg = res.marginals[0, 0].cpu().numpy()
    z = occ[0].cpu().numpy()
    del occ, res
    term = np.full(N, -1)
    for t in range(sym.T):
        term[order[offsets[t]:offsets[t + 1]]] = t
    tr = term < 0
    v = np.arange(N, dtype=np.int64)
    E = _edge_rates(n, F_ref, r)
    q = E.sum(0)
    # (Q - A) z = x0 on transient states, and the flux of z into each terminal
    inflow_tr = np.zeros(N)
    for i in range(n):
        src = np.nonzero(tr & (E[i] > 0))[0]
        inflow_tr[src ^ (1 << i)] += E[i][src] * z[src]  # one source per target for a fixed bit
    res_tr = q * z - inflow_tr - x0
    assert np.abs(res_tr[tr]).sum() <= 1e-8 * np.abs(x0[tr]).sum()
    assert np.all(z[~tr] == 0.0)
    for t in range(sym.T):
        states = order[offsets[t]:offsets[t + 1]]
        want = x0[states].sum() + inflow_tr[states].sum()
        assert abs(xi[states].sum() - want) <= 1e-9
    # stationarity inside the terminal SCCs
    inflow_t = np.zeros(N)
    for i in range(n):
        src = np.nonzero(~tr & (E[i] > 0))[0]
        inflow_t[src ^ (1 << i)] += E[i][src] * xi[src]
    assert np.abs((q * xi - inflow_t)[~tr]).sum() <= 1e-10
    assert np.all(xi >= 0.0) and np.all(xi[tr] == 0.0)
    assert abs(xi.sum() - 1.0) <= 1e-12
    for i in range(n):
        assert abs(mg[i] - xi[((v >> i) & 1) == 1].sum()) <= 1e-12


def test_n20_precision_mixed_vs_oracle(esl, ctx):
    w = synth.config_precision(n_rate_sets=2)
    text, rates, x0 = w.networks[0].bnet, w.rates[0], w.x0[0][0]
    net = esl.Net.build(ctx, esl.Model.parse(text), rates[0])
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_MIXED, tol=1e-12)
    assert net.T >= 8
    sym = O.Model(text=text).analyse(rates[0])
    ref, _ = sym.solve_many(rates, np.stack([x0, x0]), threads=2)
    got = res.x_inf[:, 0].cpu().numpy()
    l1 = np.abs(got - ref.reshape(2, -1)).sum(1)
    assert l1.max() <= 1e-10, l1
