"""Fallback and failure paths of the GPU solver, driven by iteration budgets.

No device fault is involved: the budgets of esl_solve_opts (Krylov iterations and
refinement steps of the level sweep) and of esl_ctx_set_budgets (graph fixpoint sweeps,
the block forward solve's Krylov budget, the dense-LU block cap) are set so low that
each path is taken, and every result is checked against the FP64 oracle:
- level sweep misses -> block forward solve (cuda/src/linear_system_solve.cu:249-325
  is the reference's block-triangular solve it follows);
- block solve misses -> dense FP64 LU of each SCC block of the level group (the
  reference's dense getrf of SCC blocks, linear_system_solve.cu:69-88);
- a block above the dense cap -> ESL_ERR_NOT_CONVERGED, and the context stays usable;
- graph fixpoint budget -> ESL_ERR_TIMEOUT, and the context stays usable.
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


def _case(n=13, seed=3, family="random"):
    """A network whose transient part has SCCs of 1,317-2,532 states (grid-wide Krylov
    groups of the level sweep, within the dense fallback's cap) and many small ones."""
    if family == "random":
        net_g = synth.random_table_network(np.random.default_rng(seed), n, [3], 0.5)
    else:
        net_g = synth.precision_network(seed=seed, n=n)
    rng = np.random.default_rng(60 + seed)
    rates = synth.log_uniform_rates(rng, n, 3)
    x0 = np.stack([synth.dirichlet_subspace_x0(rng, n, rng.choice(n, 5, replace=False)) for _ in range(2)])
    return net_g.bnet, rates, x0


def _check_vs_oracle(text, rates, x0, res):
    sym = O.Model(text=text).analyse(rates[0])
    xi = res.x_inf.cpu().numpy()
    mg = res.marginals.cpu().numpy()
    for b in range(rates.shape[0]):
        for q in range(x0.shape[0]):
            ox, om = sym.solve(x0[q], rates[b])
            assert np.abs(xi[b, q] - ox).sum() <= 1e-9, (b, q)
            np.testing.assert_allclose(mg[b, q], om, atol=1e-9, rtol=0)


def test_normal_solve_takes_no_fallback(esl):
    text, rates, x0 = _case()
    ctx = esl.Context(0)
    net = esl.Net.build(ctx, esl.Model.parse(text), rates[0])
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT)
    assert res.report.converged == 1
    assert res.report.fallback_systems == 0 and res.report.dense_lu_systems == 0
    _check_vs_oracle(text, rates, x0, res)


def test_sweep_miss_falls_back_to_block_solve(esl):
    text, rates, x0 = _case()
    ctx = esl.Context(0)
    net = esl.Net.build(ctx, esl.Model.parse(text), rates[0])
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT, max_iters=1, max_refine=1)
    assert res.report.converged == 1
    assert res.report.fallback_systems > 0, res.report.fallback_systems
    assert res.report.dense_lu_systems == 0, res.report.dense_lu_systems
    _check_vs_oracle(text, rates, x0, res)


def test_block_miss_falls_back_to_dense_lu(esl):
    text, rates, x0 = _case()
    ctx = esl.Context(0)
    ctx.set_budgets(block_iters=1)
    net = esl.Net.build(ctx, esl.Model.parse(text), rates[0])
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT, max_iters=1, max_refine=1)
    assert res.report.converged == 1
    assert res.report.fallback_systems > 0 and res.report.dense_lu_systems > 0
    _check_vs_oracle(text, rates, x0, res)


def test_block_above_dense_cap_is_not_converged(esl):
    text, rates, x0 = _case()
    ctx = esl.Context(0)
    m = esl.Model.parse(text)
    net = esl.Net.build(ctx, m, rates[0])
    ctx.set_budgets(block_iters=1, dense_max=1)
    with pytest.raises(esl.EslError) as e:
        esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT, max_iters=1, max_refine=1)
    assert e.value.code == -6  # ESL_ERR_NOT_CONVERGED
    # the context still works with the default budgets
    ctx.set_budgets()
    res = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT)
    assert res.report.converged == 1
    _check_vs_oracle(text, rates, x0, res)


def test_graph_budget_timeout(esl):
    text, rates, _ = _case(n=14, seed=3, family="precision")
    ctx = esl.Context(0)
    m = esl.Model.parse(text)
    ctx.set_budgets(graph_sweeps=1)
    with pytest.raises(esl.EslError) as e:
        esl.Net.build(ctx, m, rates[0])
    assert e.value.code == -5  # ESL_ERR_TIMEOUT
    ctx.set_budgets()
    net = esl.Net.build(ctx, m, rates[0])
    sym = O.Model(text=text).analyse(rates[0])
    order, offsets, levels, _ = net.export()
    assert np.array_equal(order.cpu().numpy(), sym.order)
    assert np.array_equal(offsets.cpu().numpy(), sym.offsets)
