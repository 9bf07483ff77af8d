"""Pins the CPU FP64 oracle against the reference's own known-answer tests
(``cuda/test/test.cu``) and against its Python CPU path (``python/exastolog.py``)."""
import numpy as np
import pytest

import oracle as O
from tests.helpers import FLT_EPS, nonzeros, reference_L_csr


def _model(goldens, name):
    return O.Model(text=goldens["models"][name])


def test_table_toy(goldens):
    c = goldens["cases"]["trans_table.toy"]
    m = _model(goldens, c["model"])
    indptr, rows, cols = m.table(m.rates())
    assert indptr.tolist() == c["indptr"]
    assert cols.tolist() == c["cols"]
    # every destination differs from its source in exactly one bit
    x = rows ^ cols
    assert np.all(x > 0) and np.all((x & (x - 1)) == 0)


def test_graph_toy(goldens):
    c = goldens["cases"]["trans_graph.toy"]
    m = _model(goldens, c["model"])
    s = m.analyse(m.rates())
    assert s.order.tolist() == c["reordered_vertices"]
    assert s.offsets[: s.T + 1].tolist() == c["terminal_offsets"]


def test_initial_value_toy(goldens):
    c = goldens["cases"]["initial_value.toy"]
    m = _model(goldens, c["model"])
    assert m.initial_state(c["fixed"], c["values"]).tolist() == c["state"]


def test_initial_state_with_a_node_listed_twice(goldens):
    # the reference sums (1 << node) * value: A listed with 1 and with 0 is fixed to 1
    m = _model(goldens, "toy.bnet")
    a = m.names[0]
    once = m.initial_state([a], [1], p=0.8)
    assert np.array_equal(m.initial_state([a, a], [1, 0], p=0.8), once)
    assert np.array_equal(m.initial_state([a, a], [0, 1], p=0.8), once)
    assert abs(once.sum() - 1.0) < 1e-15 and np.all(np.isfinite(once))


@pytest.mark.parametrize("name", ["solver.toy", "solver.toy2", "solver.toy3"])
def test_solver_toys(goldens, name):
    c = goldens["cases"][name]
    m = _model(goldens, c["model"])
    r = m.rates()
    s = m.analyse(r)
    assert s.order.tolist() == c["reordered_vertices"]
    assert s.offsets[: s.T + 1].tolist() == c["terminal_offsets"]
    R = s.terminal_kernels()
    assert s.offsets[: s.T + 1].tolist() == c["term_indptr"]
    assert s.order[: s.offsets[s.T]].tolist() == c["term_rows"]
    if c["term_data_each"] is not None:
        np.testing.assert_allclose(R, c["term_data_each"], rtol=0, atol=1e-14)
    Lm = s.absorption()
    indptr, cols, data = reference_L_csr(s.order, s.offsets, s.T, Lm)
    assert indptr == c["nonterm_indptr"]
    assert cols == c["nonterm_cols"]
    if c["nonterm_data"] is not None:
        np.testing.assert_allclose(data, c["nonterm_data"], rtol=0, atol=1e-14)
    else:
        np.testing.assert_allclose(data, c["nonterm_data_each"], rtol=0, atol=1e-14)
    x0 = m.initial_state(c["fixed"], c["values"])
    for use_abs in (0, 1):
        xi, marg = s.solve(x0, use_absorption=use_abs)
        idx, val = nonzeros(xi)
        assert idx.tolist() == c["nonzero_indices"]
        np.testing.assert_allclose(val, c["nonzero_data_each"], rtol=0, atol=1e-14)
        bits = (np.arange(1 << m.n)[:, None] >> np.arange(m.n)) & 1
        np.testing.assert_allclose(marg, xi @ bits, atol=1e-15)


SLOW = {"solver.zanudo"}


@pytest.mark.parametrize("name", ["solver.kras", "solver.cohen", "solver.mammal", "rates.toy", "zero_rate.toy",
                                  "symbolic.cohen_rates", "solver.zanudo"])
def test_solver_goldens(goldens, name):
    c = goldens["cases"][name]
    m = _model(goldens, c["model"])
    r = m.rates(up=c.get("up"), down=c.get("down"))
    s = m.analyse(r)
    x0 = m.initial_state(c["fixed"], c["values"])
    xi, _ = s.solve(x0)
    idx, val = nonzeros(xi)
    tol = 1e-7 if c["tolerance"] == "1e-7" else 128 * FLT_EPS
    assert idx.tolist() == c["nonzero_indices"]
    np.testing.assert_allclose(val, c["nonzero_data"], rtol=0, atol=tol)
    assert abs(xi.sum() - 1.0) < 1e-12


def test_forward_and_backward_formulations_agree(goldens):
    m = _model(goldens, "mammalian_cc.bnet")
    rng = np.random.default_rng(7)
    r = np.exp(rng.uniform(np.log(0.1), np.log(10), 2 * m.n))
    s = m.analyse(r)
    x0 = rng.dirichlet(np.ones(1 << m.n))
    a, _ = s.solve(x0, use_absorption=False)
    b, _ = s.solve(x0, use_absorption=True)
    assert np.abs(a - b).sum() < 1e-12


def test_python_reference_fixtures(goldens):
    checked = 0
    for key, ref in goldens["python_ref"].items():
        if not ref["valid"]:
            continue
        text = goldens["models"].get(key) or goldens["generated_models"].get(key)
        m = O.Model(text=text)
        s = m.analyse(m.rates())
        xi, _ = s.solve(m.initial_state())
        idx, val = nonzeros(xi)
        assert idx.tolist() == ref["nonzero_indices"], key
        np.testing.assert_allclose(val, ref["nonzero_data"], rtol=0, atol=1e-10, err_msg=key)
        checked += 1
    assert checked >= 5


def test_uniformized_limits(goldens):
    """The oracle against the limit of the uniformized chain (uniform rates and x0),
    computed by repeated squaring with no SCC or solver logic, for every model the
    Python path was run on -- including the ones where that path is wrong."""
    checked = wrong_python = 0
    for key, lim in goldens["uniformized_limits"].items():
        text = goldens["models"].get(key) or goldens["generated_models"].get(key)
        m = O.Model(text=text)
        s = m.analyse(m.rates())
        xi, _ = s.solve(m.initial_state())
        exact = np.zeros(1 << m.n)
        exact[lim["nonzero_indices"]] = lim["nonzero_data"]
        assert np.abs(xi - exact).sum() <= 1e-10, key
        checked += 1
        wrong_python += not goldens["python_ref"][key]["valid"]
    assert checked >= 30 and wrong_python >= 10


def test_bnet_quirks():
    # header skipped only when it starts with "targets"; unterminated last line dropped
    m = O.Model(text="targets, factors\nA, A\nB, !A")
    assert m.names == ["A"]
    m = O.Model(text="A, A\nB, !A\n")
    assert m.names == ["A", "B"]
    # identifiers that are not nodes are dropped from their clause: B = A & X -> A
    m = O.Model(text="targets, factors\nA, A\nB, A & X\n")
    off, pos, neg = m.clauses()
    assert pos[off[1]:off[2]].tolist() == [1] and neg[off[1]:off[2]].tolist() == [0]
    # contradictory terms are removed before the drop: (A & X & !X) | B -> B
    m = O.Model(text="targets, factors\nA, (A & X & !X) | B\nB, B\n")
    off, pos, neg = m.clauses()
    assert pos[off[0]:off[1]].tolist() == [2]
    with pytest.raises(O.OracleError):
        O.Model(text="targets, factors\nA, (A & \nB, B\n")


def test_threaded_solve_many_equals_serial_solves():
    # the CPU baseline and several GPU tests use the oracle's threaded batch solve
    from paraexastolog_b200 import synth

    rng = np.random.default_rng(9)
    net = synth.random_table_network(rng, 10, [2, 3], 0.5)
    rates = synth.log_uniform_rates(rng, 10, 6)
    x0 = np.stack([synth.dirichlet_subspace_x0(rng, 10, rng.choice(10, 4, replace=False)) for _ in range(6)])
    s = O.Model(text=net.bnet).analyse(rates[0])
    many, marg = s.solve_many(rates, x0, threads=4)
    for k in range(6):
        one, om = s.solve(x0[k], rates[k])
        assert np.array_equal(many.reshape(6, -1)[k], one)
        assert np.array_equal(marg.reshape(6, -1)[k], om)
