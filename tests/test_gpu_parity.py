"""CUDA path vs the CPU FP64 oracle and the reference's known-answer tests.

Integer and graph stages must be bit-exact (table CSC, flip masks, SCC labels,
levels, reordered vertices, offsets); numeric results within L1 <= 1e-9 of the
oracle (tolerance stated per test) and within the reference's own tolerances of
its goldens (128 * FLT_EPSILON, or 1e-7 for the mammal case).
"""
import numpy as np
import pytest

import oracle as O
from paraexastolog_b200 import synth
from tests.helpers import FLT_EPS, nonzeros, reference_L_csr

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def esl():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import paraexastolog_b200 as E
    E.lib()  # fails loudly when the library is missing
    return E


@pytest.fixture(scope="module")
def ctx(esl):
    return esl.Context(0)


def _nets():
    out = []
    for seed in range(3):
        rng = np.random.default_rng(100 + seed)
        out.append((f"rand{seed}", synth.random_table_network(rng, 9 + seed, [1, 2, 3], 0.5).bnet))
    rng = np.random.default_rng(7)
    out.append(("canal12", synth.nested_canalizing_network(rng, 12, 3).bnet))
    out.append(("prec12", synth.precision_network(seed=5, n=12).bnet))
    for n in (1, 2, 3, 4, 5, 6):
        rng = np.random.default_rng(n)
        out.append((f"tiny{n}", synth.random_table_network(rng, n, [1, 2] if n > 1 else [1], 0.5).bnet))
    return out


def _rates(n, seed, zeros=0):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(0.1), np.log(10), 2 * n))
    if zeros:
        r[rng.choice(2 * n, size=min(zeros, 2 * n), replace=False)] = 0.0
    return r


def _models(goldens):
    return [(k, goldens["models"][k]) for k in ["toy.bnet", "toy2.bnet", "toy3.bnet", "krasmodel15vars.bnet",
                                                 "mammalian_cc.bnet"]] + _nets()


@pytest.mark.parametrize("zeros", [0, 3])
def test_table_bit_exact(esl, ctx, goldens, zeros):
    for name, text in _models(goldens):
        om = O.Model(text=text)
        m = esl.Model.parse(text)
        r = _rates(m.n, 1, zeros)
        ip, rows, cols = om.table(r)
        dip, drows, dcols = esl.table(ctx, m, r)
        assert np.array_equal(dip.cpu().numpy(), ip), name
        assert np.array_equal(drows.cpu().numpy(), rows), name
        assert np.array_equal(dcols.cpu().numpy(), cols), name
        F, G = esl.flip_masks(ctx, m, r)
        oF = om.flip_masks(r).astype(np.int64)
        assert np.array_equal(F.cpu().numpy().astype(np.int64) & 0xFFFFFFFF, oF), name
        s = np.arange(1 << m.n)
        oG = np.zeros_like(oF)
        for i in range(m.n):
            oG |= ((oF[s ^ (1 << i)] >> i) & 1) << i
        assert np.array_equal(G.cpu().numpy().astype(np.int64) & 0xFFFFFFFF, oG), name


def test_table_golden(esl, ctx, goldens):
    c = goldens["cases"]["trans_table.toy"]
    m = esl.Model.parse(goldens["models"][c["model"]])
    ip, rows, cols = esl.table(ctx, m, m.rates_uniform())
    assert ip.cpu().tolist() == c["indptr"]
    assert cols.cpu().tolist() == c["cols"]


@pytest.mark.parametrize("zeros", [0, 4])
def test_graph_bit_exact(esl, ctx, goldens, zeros):
    for name, text in _models(goldens):
        om = O.Model(text=text)
        m = esl.Model.parse(text)
        r = _rates(m.n, 2, zeros)
        sym = om.analyse(r)
        net = esl.Net.build(ctx, m, r)
        assert (net.n_sccs, net.T, net.terminal_states) == (sym.n_sccs, sym.T, int(sym.offsets[sym.T])), name
        order, offsets, levels, labels = net.export()
        assert np.array_equal(order.cpu().numpy(), sym.order), name
        assert np.array_equal(offsets.cpu().numpy(), sym.offsets), name
        assert np.array_equal(levels.cpu().numpy(), sym.levels), name
        assert np.array_equal(labels.cpu().numpy(), sym.labels), name
        # the same from the CSC table
        ip, rows, _ = esl.table(ctx, m, r, with_cols=False)
        net2 = esl.Net.from_csc(ctx, m.n, ip, rows)
        o2 = net2.export()
        assert np.array_equal(o2[0].cpu().numpy(), sym.order), name
        assert np.array_equal(o2[1].cpu().numpy(), sym.offsets), name


def test_graph_golden(esl, ctx, goldens):
    c = goldens["cases"]["trans_graph.toy"]
    m = esl.Model.parse(goldens["models"][c["model"]])
    net = esl.Net.build(ctx, m, m.rates_uniform())
    order, offsets, _, _ = net.export()
    assert order.cpu().tolist() == c["reordered_vertices"]
    assert offsets.cpu().tolist()[: net.T + 1] == c["terminal_offsets"]


def test_initial_state(esl, ctx, goldens):
    c = goldens["cases"]["initial_value.toy"]
    m = esl.Model.parse(goldens["models"][c["model"]])
    assert m.initial_state(ctx, c["fixed"], c["values"]).cpu().tolist() == c["state"]
    om = O.Model(text=goldens["models"]["krasmodel15vars.bnet"])
    km = esl.Model.parse(goldens["models"]["krasmodel15vars.bnet"])
    for p in (1.0, 0.7):
        a = km.initial_state(ctx, ["cc", "KRAS"], [1, 0], p).cpu().numpy()
        b = om.initial_state(["cc", "KRAS"], [1, 0], p)
        np.testing.assert_allclose(a, b, rtol=1e-15, atol=0)


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("name", ["solver.toy", "solver.toy2", "solver.toy3"])
def test_solver_toy_goldens(esl, ctx, goldens, name, method):
    c = goldens["cases"][name]
    m = esl.Model.parse(goldens["models"][c["model"]])
    r = m.rates_uniform()
    net = esl.Net.build(ctx, m, r)
    x0 = m.initial_state(ctx, c["fixed"], c["values"])
    res = esl.solve(ctx, net, r, x0, want_R=True, want_L=True, method=method)
    order, offsets, _, _ = net.export()
    order, offsets = order.cpu().numpy(), offsets.cpu().numpy()
    R = res.R.cpu().numpy()
    assert offsets[: net.T + 1].tolist() == c["term_indptr"]
    assert order[: net.terminal_states].tolist() == c["term_rows"]
    if c["term_data_each"] is not None:
        np.testing.assert_allclose(R, c["term_data_each"], atol=1e-12, rtol=0)
    indptr, cols, data = reference_L_csr(order, offsets, net.T, res.L.cpu().numpy())
    assert indptr == c["nonterm_indptr"]
    assert cols == c["nonterm_cols"]
    expect = c["nonterm_data"] if c["nonterm_data"] is not None else [c["nonterm_data_each"]] * len(data)
    np.testing.assert_allclose(data, expect, atol=1e-12, rtol=0)
    idx, val = nonzeros(res.x_inf.cpu().numpy())
    assert idx.tolist() == c["nonzero_indices"]
    np.testing.assert_allclose(val, c["nonzero_data_each"], atol=1e-12, rtol=0)


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("name", ["solver.kras", "solver.mammal", "rates.toy", "zero_rate.toy", "solver.cohen",
                                  "symbolic.cohen_rates"])
def test_solver_goldens(esl, ctx, goldens, name, method):
    c = goldens["cases"][name]
    m = esl.Model.parse(goldens["models"][c["model"]])
    r = m.rates_uniform(up=c.get("up"), down=c.get("down"))
    net = esl.Net.build(ctx, m, r)
    x0 = m.initial_state(ctx, c["fixed"], c["values"])
    res = esl.solve(ctx, net, r, x0, method=method, tol=1e-12)
    xi = res.x_inf.cpu().numpy()
    idx, val = nonzeros(xi)
    # the reference's FP32 goldens: indices exact, values within its tolerance
    big = idx[val > 1e-12]
    assert big.tolist() == c["nonzero_indices"]
    tol = 1e-7 if c["tolerance"] == "1e-7" else 128 * FLT_EPS
    np.testing.assert_allclose(xi[big], c["nonzero_data"], atol=tol, rtol=0)
    # and the FP64 oracle: L1 <= 1e-9
    om = O.Model(text=goldens["models"][c["model"]])
    ox, om_marg = om.analyse(r).solve(x0.cpu().numpy())
    assert np.abs(xi - ox).sum() <= 1e-9
    np.testing.assert_allclose(res.marginals.cpu().numpy(), om_marg, atol=1e-9, rtol=0)


@pytest.mark.parametrize("method", [0, 1, 2])
def test_random_networks_vs_oracle(esl, ctx, method):
    for name, text in _nets():
        om = O.Model(text=text)
        m = esl.Model.parse(text)
        for seed in range(2):
            r = _rates(m.n, 10 + seed, zeros=seed)
            rng = np.random.default_rng(seed)
            x0 = rng.dirichlet(np.ones(1 << m.n))
            ox, omarg = om.analyse(r).solve(x0)
            net = esl.Net.build(ctx, m, r)
            res = esl.solve(ctx, net, r, x0, method=method, tol=1e-10)
            xi = res.x_inf.cpu().numpy()
            l1 = np.abs(xi - ox).sum()
            assert l1 <= 1e-9, (name, seed, l1)
            assert abs(xi.sum() - 1.0) <= 1e-9
            np.testing.assert_allclose(res.marginals.cpu().numpy(), omarg, atol=1e-9, rtol=0)


def test_absorption_matrix_vs_oracle(esl, ctx):
    for name, text in _nets()[:5]:
        om = O.Model(text=text)
        m = esl.Model.parse(text)
        r = _rates(m.n, 3)
        sym = om.analyse(r)
        net = esl.Net.build(ctx, m, r)
        x0 = np.full(1 << m.n, 1.0 / (1 << m.n))
        res = esl.solve(ctx, net, r, x0, want_R=True, want_L=True)
        np.testing.assert_allclose(res.R.cpu().numpy(), sym.terminal_kernels(), atol=1e-12, rtol=0)
        np.testing.assert_allclose(res.L.cpu().numpy(), sym.absorption(), atol=1e-9, rtol=0)


def test_large_terminal_scc(esl, ctx):
    # every node negates itself: the whole cube is one terminal SCC and the kernel
    # is the product of per-node two-state chains
    n = 9
    text = "targets, factors\n" + "".join(f"v{i}, !v{i}\n" for i in range(n))
    m = esl.Model.parse(text)
    r = _rates(n, 4)
    net = esl.Net.build(ctx, m, r)
    assert net.T == 1 and net.terminal_states == 1 << n
    x0 = np.full(1 << n, 1.0 / (1 << n))
    res = esl.solve(ctx, net, r, x0, want_R=True)
    s = np.arange(1 << n)
    expect = np.ones(1 << n)
    for i in range(n):
        up, down = r[2 * i], r[2 * i + 1]
        expect *= np.where((s >> i) & 1, up / (up + down), down / (up + down))
    np.testing.assert_allclose(res.x_inf.cpu().numpy(), expect, atol=1e-12, rtol=0)


@pytest.mark.parametrize("method", [0, 1, 2])
def test_batch_vs_oracle(esl, ctx, method):
    w = synth.config_batch(seed=5, n_networks=3, n_rate_sets=4, n_x0=3, n_lo=9, n_hi=12)
    for net_g, rates, x0s in zip(w.networks, w.rates, w.x0):
        om = O.Model(text=net_g.bnet)
        m = esl.Model.parse(net_g.bnet)
        net = esl.Net.build(ctx, m, rates[0])
        res = esl.solve_batch(ctx, net, rates, x0s, method=method, tol=1e-10)
        xi = res.x_inf.cpu().numpy()
        mg = res.marginals.cpu().numpy()
        sym = om.analyse(rates[0])
        for b in range(rates.shape[0]):
            for k in range(x0s.shape[0]):
                ox, omarg = sym.solve(x0s[k], rates[b])
                assert np.abs(xi[b, k] - ox).sum() <= 1e-9
                np.testing.assert_allclose(mg[b, k], omarg, atol=1e-9, rtol=0)


def test_incompatible_zero_pattern_rejected(esl, ctx, goldens):
    m = esl.Model.parse(goldens["models"]["toy.bnet"])
    net = esl.Net.build(ctx, m, m.rates_uniform())
    bad = m.rates_uniform(down={"C": 0.0})
    assert not net.compatible(bad)
    with pytest.raises(esl.EslError):
        esl.solve(ctx, net, bad, np.full(8, 1 / 8))


def test_host_api_matches_device_api(esl, ctx):
    w = synth.config_small()
    m = esl.Model.parse(w.networks[0].bnet)
    xi, mg, rep = esl.solve_host(ctx, m, w.rates[0], w.x0[0])
    om = O.Model(text=w.networks[0].bnet)
    ox, omarg = om.analyse(w.rates[0][0]).solve(w.x0[0][0])
    assert np.abs(xi[0, 0] - ox).sum() <= 1e-9
    assert rep.converged == 1


@pytest.mark.parametrize("method", [0, 2])
def test_absorption_matrix_kras(esl, ctx, goldens, method):
    # 40 terminal SCCs; L is checked against the oracle's absorption probabilities
    text = goldens["models"]["krasmodel15vars.bnet"]
    m = esl.Model.parse(text)
    r = m.rates_uniform()
    net = esl.Net.build(ctx, m, r)
    x0 = m.initial_state(ctx)
    res = esl.solve(ctx, net, r, x0, want_L=True, method=method)
    Lo = O.Model(text=text).analyse(r).absorption(r)
    L = res.L.cpu().numpy()
    assert np.abs(L - Lo.reshape(L.shape)).max() <= 1e-9
    # the backward solve itself converged: kras's transient part is acyclic, where one of
    # the 40 backward systems breaks down with the shadow residual r0 = r and needs the
    # dense restart shadow
    assert res.report.absorption_by_sweep == 0


WIDE_AND_CONSTANT = ("targets, factors\nA, B & C & D & E & F & !G\nB, 1\nC, 0\nD, A | B\nE, !E\n"
                     "F, (A & !B) | (C & D) | (E & G)\nG, A\nH, true\nI, FALSE & H\n")


def test_constants_and_six_input_rules(esl, ctx):
    # rules over 6 inputs and constant rules (1, 0, true, FALSE)
    om = O.Model(text=WIDE_AND_CONSTANT)
    m = esl.Model.parse(WIDE_AND_CONSTANT)
    r = _rates(m.n, 8)
    ip, rows, cols = esl.table(ctx, m, r)
    rip, rrows, rcols = om.table(r)
    assert np.array_equal(ip.cpu().numpy(), rip) and np.array_equal(rows.cpu().numpy(), rrows)
    assert np.array_equal(cols.cpu().numpy(), rcols)
    net = esl.Net.build(ctx, m, r)
    x0 = np.full(1 << m.n, 1.0 / (1 << m.n))
    res = esl.solve(ctx, net, r, x0, method=esl.METHOD_DIRECT, tol=1e-12)
    ox, om_marg = om.analyse(r).solve(x0)
    assert np.abs(res.x_inf.cpu().numpy() - ox).sum() <= 1e-9


def test_zanudo_golden_n23(esl, ctx, goldens):
    # the reference's largest known-answer case: 23 nodes, 8,388,608 states
    c = goldens["cases"]["solver.zanudo"]
    m = esl.Model.parse(goldens["models"][c["model"]])
    assert m.n == 23
    r = m.rates_uniform()
    net = esl.Net.build(ctx, m, r)
    x0 = m.initial_state(ctx, c["fixed"], c["values"])
    res = esl.solve(ctx, net, r, x0, method=esl.METHOD_DIRECT, tol=1e-12)
    xi = res.x_inf.cpu().numpy()
    idx, val = nonzeros(xi)
    big = idx[val > 1e-12]
    assert big.tolist() == c["nonzero_indices"]
    np.testing.assert_allclose(xi[big], c["nonzero_data"], atol=128 * FLT_EPS, rtol=0)
    assert abs(xi.sum() - 1.0) <= 1e-12


def test_autotune_keeps_results(esl, ctx):
    # the autotuner changes only the tiling: results stay within the solver tolerance
    w = synth.config_precision(seed=3, n=14, n_rate_sets=96)
    text, rates, x0 = w.networks[0].bnet, w.rates[0], w.x0[0]
    net = esl.Net.build(ctx, esl.Model.parse(text), rates[0])
    before = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT, tol=1e-12).x_inf.cpu().numpy()
    pick = net.autotune(rates, x0, method=esl.METHOD_DIRECT, tol=1e-12)
    assert pick["tile_mb"] in (16, 48, 128) and pick["ms"] > 0
    after = esl.solve_batch(ctx, net, rates, x0, method=esl.METHOD_DIRECT, tol=1e-12).x_inf.cpu().numpy()
    assert np.abs(after - before).sum(-1).max() <= 1e-10


@pytest.mark.parametrize("name", ["rand0", "canal12", "prec12", "tiny3", "bench20"])
def test_device_plan_equals_host_plan(esl, ctx, name):
    """The level-sweep plan the solver builds on the device equals, part for part, the
    one the host reference builder makes from copies of the net's arrays."""
    if name == "bench20":
        text = synth.config_learned(n_rate_sets=1).networks[0].bnet
    else:
        text = dict(_nets())[name]
    m = esl.Model.parse(text)
    r = _rates(m.n, 9)
    net = esl.Net.build(ctx, m, r)
    dev = net.plan_checksums(host_builder=False)
    host = net.plan_checksums(host_builder=True)
    assert np.array_equal(dev, host), (dev, host)
