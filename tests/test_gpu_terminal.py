"""Terminal kernels of terminal SCCs above 128 states on the GPU.

For each such SCC C, the level sweep solves the rank-one deflated system
(-K_C + u 1^T) pi = u (u = out-rates / |C| on the odd-parity states) by FP64 BiCGStab on
its odd-row Schur complement.  This replaces the reference's minor-determinant
kernels (cuda/src/solver.cu:102-159).  The results are checked against:
- closed forms (the self-negating cube, whose kernel is a product of two-state chains);
- the FP64 oracle's kernels, at L1 <= 1e-10 per SCC and rate set;
- the generator residual |K pi|_1 / sum_v q_v pi_v <= 1e-12, on the two 262,144-state
  attractors (n = 18) of the many-network workload, where the pinned form of the
  previous solver missed its tolerance.
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


def _generator_residual(F, rates, pi):
    n = int(np.log2(F.size))
    s = np.arange(F.size, dtype=np.int64)
    F = F.astype(np.int64)
    Kpi = np.zeros(F.size)
    outflow = np.zeros(F.size)
    for b in range(n):
        src = s[((F >> b) & 1) == 1]
        up = ((src >> b) & 1) == 0
        flow = np.where(up, rates[2 * b], rates[2 * b + 1]) * pi[src]
        np.add.at(Kpi, src ^ (1 << b), flow)
        outflow[src] += flow
    Kpi -= outflow
    return np.abs(Kpi).sum() / outflow.sum()


@pytest.mark.parametrize("n", [9, 12])
def test_cube_closed_form_batch(esl, ctx, n):
    text = "targets, factors\n" + "".join(f"v{i}, !v{i}\n" for i in range(n))
    m = esl.Model.parse(text)
    rates = synth.log_uniform_rates(np.random.default_rng(40 + n), n, 4)
    net = esl.Net.build(ctx, m, rates[0])
    assert net.T == 1 and net.terminal_states == 1 << n
    x0 = np.full((1, 1 << n), 1.0 / (1 << n))
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT)
    assert res.report.converged == 1
    xi = res.x_inf.cpu().numpy()
    s = np.arange(1 << n)
    for b in range(rates.shape[0]):
        expect = np.ones(1 << n)
        for i in range(n):
            up, down = rates[b, 2 * i], rates[b, 2 * i + 1]
            expect *= np.where((s >> i) & 1, up / (up + down), down / (up + down))
        np.testing.assert_allclose(xi[b, 0], expect, atol=1e-13, rtol=1e-10)


@pytest.mark.parametrize("seed,n", [(5, 12), (3, 14), (2, 14)])
def test_precision_networks_vs_oracle(esl, ctx, seed, n):
    """Networks with several cyclic attractors of 240-2,048 states next to small ones."""
    net_g = synth.precision_network(seed=seed, n=n)
    rng = np.random.default_rng(seed)
    rates = synth.log_uniform_rates(rng, n, 3)
    om = O.Model(text=net_g.bnet)
    sym = om.analyse(rates[0])
    sizes = np.diff(sym.offsets[: sym.T + 1])
    assert sizes.max() > 128
    m = esl.Model.parse(net_g.bnet)
    net = esl.Net.build(ctx, m, rates[0])
    x0 = synth.dirichlet_subspace_x0(rng, n, rng.choice(n, 5, replace=False))
    for b in range(rates.shape[0]):
        res = esl.solve(ctx, net, rates[b], x0, want_R=True, method=esl.METHOD_DIRECT)
        R = res.R.cpu().numpy()
        oR = sym.terminal_kernels(rates[b])
        for t in range(sym.T):
            a, e = sym.offsets[t], sym.offsets[t + 1]
            assert np.abs(R[a:e] - oR[a:e]).sum() <= 1e-10, (b, t, e - a)
        ox, om_ = sym.solve(x0, rates[b])
        assert np.abs(res.x_inf.cpu().numpy() - ox).sum() <= 1e-9
        np.testing.assert_allclose(res.marginals.cpu().numpy(), om_, atol=1e-9, rtol=0)


@pytest.mark.parametrize("index", [10, 31])
def test_n18_attractors_of_the_many_network_workload(esl, ctx, index):
    """A single 262,144-state terminal SCC: kernel against the oracle and the generator."""
    w = synth.config_batch()
    net_g, rates = w.networks[index], w.rates[index][:3]
    m = esl.Model.parse(net_g.bnet)
    net = esl.Net.build(ctx, m, rates[0])
    assert net.T == 1 and net.terminal_states == 1 << 18
    om = O.Model(text=net_g.bnet)
    sym = om.analyse(rates[0])
    F = np.asarray(om.flip_masks(rates[0]))
    order = np.asarray(sym.order)
    x0 = w.x0[index][:1]
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT)
    assert res.report.converged == 1
    xi = res.x_inf.cpu().numpy()
    for b in range(rates.shape[0]):
        pi = xi[b, 0]
        # x_inf = pi times the terminal mass of x0, whose 2^18 terms alone sum to 1 only
        # within ~1e-12 in sequential FP64 (many equal terms round the same way)
        assert abs(pi.sum() - 1.0) <= 1e-11 and pi.min() >= -1e-15
        assert _generator_residual(F, rates[b], pi) <= 1e-12
        oR = np.empty(1 << 18)
        oR[order] = sym.terminal_kernels(rates[b])
        assert np.abs(pi - oR).sum() <= 1e-10
