"""CPU-side checks of the C-ABI library: it loads, exports every declared symbol,
and its host front end (bnet parsing, rate vectors) agrees with the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import paraexastolog_b200 as esl
from paraexastolog_b200 import synth


def test_library_exports_every_declared_symbol():
    L = esl.lib()
    names = esl.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


# entry point -> arguments of a call with NULL handles (C.c_double / c_float where the
# signature has a floating-point argument, so that the call matches the ABI)
_NULL_CALLS = {
    "esl_ctx_synchronize": (None,),
    "esl_model_parse": (None, None),
    "esl_model_load": (None, None),
    "esl_model_nodes": (None, None),
    "esl_model_node_index": (None, None, None),
    "esl_initial_state": (None, None, 0, None, None, 0, None, None, None),
    "esl_table_nnz": (None, None, None, None),
    "esl_table_build": (None, None, None, None, None, None),
    "esl_flip_masks": (None, None, None, None, None),
    "esl_net_build": (None, None, None, None),
    "esl_net_info": (None, None, None, None, None),
    "esl_net_export": (None, None, None, None, None, None),
    "esl_net_autotune": (None, None, 1, None, 1, None, None, None, None, None),
    "esl_net_compatible": (None, None, None),
    "esl_solve": (None, None, None, None, None, None, None, None, None, None),
    "esl_solve_batch": (None, None, 1, None, 1, None, None, None, None, None),
    "esl_solve_many": (None, 0, None, 0, None),
    "esl_mlp_create": (None, None, C.c_uint64(0), None),
    "esl_mlp_info": (None, None, None, None),
    "esl_mlp_targets": (None, None),
    "esl_mlp_reach": (None, None),
    "esl_mlp_get_params": (None, None),
    "esl_mlp_set_params": (None, None, C.c_float(0.0), C.c_float(1.0)),
    "esl_mlp_predict": (None, 1, None, None),
    "esl_ctx_set_profiling": (None, 1),
    "esl_ctx_profile": (None, None, None, None),
    "esl_ctx_profile_records": (None, 0, None, None, None),
    "esl_launch_count": (None,),
}


@pytest.mark.parametrize("name", sorted(_NULL_CALLS))
def test_null_handles_are_rejected(name):
    """Every entry point returns ESL_ERR_INVALID for NULL handles or outputs, before any
    device work (this container has no GPU), and sets a message."""
    f = getattr(esl.lib(), name)
    f.restype = C.c_int
    assert f(*_NULL_CALLS[name]) == -1
    msg = esl.lib().esl_last_error
    msg.restype = C.c_char_p
    assert msg()


@pytest.mark.parametrize("name", ["esl_ctx_destroy", "esl_model_free", "esl_net_free", "esl_mlp_free"])
def test_free_of_null_is_a_no_op(name):
    f = getattr(esl.lib(), name)
    f.restype = C.c_int
    assert f(None) == 0


def _truth(off, pos, neg, i, states):
    f = np.zeros(len(states), bool)
    for c in range(off[i], off[i + 1]):
        f |= ((states & pos[c]) == pos[c]) & ((states & neg[c]) == 0)
    return f


def _same_clauses(text):
    """Same node list and the same truth function of every rule (the clause lists
    may pick different never-true representatives for all-contradictory rules)."""
    a = esl.Model.parse(text)
    b = O.Model(text=text)
    assert a.names == b.names
    oa, pa, na = a.clauses()
    ob, pb, nb = b.clauses()
    states = np.arange(1 << a.n, dtype=np.int64) if a.n <= 16 else None
    for i in range(a.n):
        if states is not None:
            assert np.array_equal(_truth(oa, pa, na, i, states), _truth(ob, pb, nb, i, states)), a.names[i]
        else:
            ca = sorted(zip(pa[oa[i]:oa[i + 1]].tolist(), na[oa[i]:oa[i + 1]].tolist()))
            cb = sorted(zip(pb[ob[i]:ob[i + 1]].tolist(), nb[ob[i]:ob[i + 1]].tolist()))
            assert ca == cb, (a.names[i], ca, cb)


def test_parser_matches_oracle_on_reference_models(goldens):
    for name, text in goldens["models"].items():
        _same_clauses(text)


@pytest.mark.parametrize("seed", range(4))
def test_parser_matches_oracle_on_generated(seed):
    rng = np.random.default_rng(seed)
    _same_clauses(synth.random_table_network(rng, 8, [1, 2, 3, 4], 0.5).bnet)
    _same_clauses(synth.nested_canalizing_network(rng, 9, 3).bnet)


def test_parser_quirks():
    assert esl.Model.parse("targets, factors\nA, A\nB, !A").names == ["A"]
    assert esl.Model.parse("A, A\nB, !A\n").names == ["A", "B"]
    _same_clauses("targets, factors\nA, A\nB, A & X\n")
    _same_clauses("targets, factors\nA, (A & X & !X) | B\nB, B\n")
    _same_clauses("targets, factors\nA, !(A | !(B & (A | !B)))\nB, !!B\n")
    _same_clauses("targets,\tfactors\nA,\tA & !A\nB, B\n")
    with pytest.raises(esl.EslError):
        esl.Model.parse("targets, factors\nA, (A & \nB, B\n")
    with pytest.raises(esl.EslError):
        esl.Model.parse("targets, factors\nA, (X & !X) | (Y & !Y)\nB, B\n")


def test_rates_host_api(goldens):
    m = esl.Model.parse(goldens["models"]["toy.bnet"])
    r = m.rates_uniform(down={"C": 2.0})
    assert r.tolist() == [1, 1, 1, 2, 1, 1]
    with pytest.raises(esl.EslError):
        m.rates_uniform(up={"Z": 1.0})
    with pytest.raises(esl.EslError):
        m.rates_uniform(up={"A": -1.0})
    a = m.rates_normal(1.0, 0.5)
    b = m.rates_normal(1.0, 0.5)
    assert np.array_equal(a, b) and np.all(a >= 0)
    assert m.rates_normal(1.0, 0.5, up={"A": 7.0})[0] == 7.0


@pytest.mark.parametrize("mean,std,seed", [(1.0, 0.5, 0), (0.2, 1.0, 0), (3.0, 2.0, 12345)])
def test_rates_normal_matches_oracle(goldens, mean, std, seed):
    # the same engine, distribution, redraw rule and draw order as the reference's
    # generate_normal; (0.2, 1.0) redraws about 42% of the draws
    for name in ("toy.bnet", "krasmodel15vars.bnet", "mammalian_cc.bnet"):
        text = goldens["models"][name]
        m, om = esl.Model.parse(text), O.Model(text=text)
        assert m.rates_normal(mean, std, seed=seed).tolist() == om.rates_normal(mean, std, seed=seed).tolist()
        # explicit rates take no draw: the following nodes get the draws the reference gives them
        up, down = {om.names[0]: 7.0}, {om.names[-1]: 0.0, om.names[1]: 2.5}
        got = m.rates_normal(mean, std, seed=seed, up=up, down=down)
        assert got.tolist() == om.rates_normal(mean, std, seed=seed, up=up, down=down).tolist()
        assert got[0] == 7.0 and got[-1] == 0.0 and got[3] == 2.5 and np.all(got >= 0)


def test_rates_normal_gives_up_like_the_reference():
    m, om = esl.Model.parse("A, A\nB, B\n"), O.Model(text="A, A\nB, B\n")
    with pytest.raises(esl.EslError):
        m.rates_normal(-50.0, 1.0)
    with pytest.raises(O.OracleError):
        om.rates_normal(-50.0, 1.0)


def test_explicit_rate_lists_are_checked():
    """A count with a NULL name or value array, or a NULL name inside it, is an error
    rather than a dereference."""
    m = esl.Model.parse("A, A\nB, !A\n")
    out = np.zeros(4)
    f = esl.lib().esl_rates_uniform
    name = C.c_char_p(b"A")
    names = (C.c_char_p * 1)(name)
    vals = np.array([2.0])
    assert f(m._h, 1, None, vals.ctypes.data, 0, None, None, out.ctypes.data) == -1
    assert f(m._h, 1, names, None, 0, None, None, out.ctypes.data) == -1
    assert f(m._h, 0, None, None, -1, None, None, out.ctypes.data) == -1
    assert f(m._h, 1, (C.c_char_p * 1)(None), vals.ctypes.data, 0, None, None, out.ctypes.data) == -1
    assert f(m._h, 1, names, vals.ctypes.data, 0, None, None, out.ctypes.data) == 0
    assert out.tolist() == [2.0, 1.0, 1.0, 1.0]
    g = esl.lib().esl_rates_normal
    assert g(m._h, 1.0, 0.5, 0, 0, None, None, 1, None, vals.ctypes.data, out.ctypes.data) == -1


def test_long_chains_and_deep_nesting():
    """Chains of any length parse (they used to recurse once per operator and overflow
    the stack); parenthesis nesting beyond 512 levels is a parse error, not a crash."""
    k = 200_000
    for text in (" | ".join(["A"] * k), " & ".join(["A"] * k), "(" * 512 + "!!A" + ")" * 512):
        m = esl.Model.parse("targets, factors\nA, " + text + "\nB, A | B\n")
        off, pos, neg = m.clauses()
        assert off.tolist() == [0, 1, 3] and pos[0] == 1 and neg[0] == 0
    for depth in (513, k):
        with pytest.raises(esl.EslError, match="nested too deeply"):
            esl.Model.parse("targets, factors\nA, " + "(" * depth + "A" + ")" * depth + "\n")
    # the same rule written flat and as a long mixed chain gives the oracle's clauses
    _same_clauses("targets, factors\nA, " + " | ".join(f"(A & !B & C{i % 3})" for i in range(3000)) +
                  "\nB, B\nC0, A\nC1, B\nC2, C0\n")


def _random_rule(rng, depth=0):
    atoms = ["A", "B", "C", "D"] * 3 + ["X", "Y", "1", "0", "true", "n_1"]
    if depth > 3 or rng.random() < 0.3:
        return "!" * int(rng.integers(0, 3)) + atoms[rng.integers(len(atoms))]
    op = " & " if rng.random() < 0.5 else " | "
    body = op.join(_random_rule(rng, depth + 1) for _ in range(int(rng.integers(2, 4))))
    return "!" * int(rng.integers(0, 2)) + "(" + body + ")" if rng.random() < 0.7 else body


def test_parser_fuzz_against_oracle():
    """Random rules (nesting, negation chains, identifiers that are not nodes, constants,
    contradictions, uneven spacing): the library and the oracle either both reject a
    model or give every node the same truth function."""
    rng = np.random.default_rng(0)
    agree = rejected = 0
    for _ in range(300):
        text = "targets, factors\n" + "".join(
            f"{n},{' ' * int(rng.integers(0, 3))}{_random_rule(rng)}\n" for n in "ABCD")
        try:
            esl.Model.parse(text)
        except esl.EslError:
            with pytest.raises(O.OracleError):
                O.Model(text=text)
            rejected += 1
            continue
        _same_clauses(text)
        agree += 1
    assert agree >= 250 and rejected >= 1


def test_node_count_limits():
    """30 nodes (ESL_MAX_NODES) parse; 31 are ESL_ERR_TOO_LARGE; an empty model is a
    parse error.  Checked on the host, before any device work."""
    def model(n):
        return "targets, factors\n" + "".join(f"v{i}, !v{i}\n" for i in range(n))

    assert esl.Model.parse(model(30)).n == 30
    with pytest.raises(esl.EslError) as e:
        esl.Model.parse(model(31))
    assert e.value.code == -7 and "more than 30 nodes" in str(e.value)
    with pytest.raises(esl.EslError) as e:
        esl.Model.parse("targets, factors\n")
    assert e.value.code == -2
    # the allocation-free table build rejects more than 20 nodes before touching a device
    m = esl.Model.parse(model(21))
    nnz = C.c_int64(-1)
    st = esl.lib().esl_table_build_static(m._h, np.ones(42).ctypes.data, None, C.c_void_p(1), C.c_void_p(1),
                                          None, 0, C.byref(nnz))
    assert st == -7 and "at most 20 nodes" in esl.lib().esl_last_error().decode()


def test_batch_buffers_are_checked_before_the_library_sees_them():
    """The library reads and writes every batch buffer by the sizes the network implies:
    a short, mistyped or misplaced one is a ValueError in the binding, not an access past
    its end."""
    import torch

    n, N = 4, 16
    r, x = torch.ones(3, 2 * n, dtype=torch.float64), torch.full((2, N), 1.0 / N, dtype=torch.float64)
    assert esl._check_batch(n, r, x) == (3, 2)
    assert esl._check_batch(n, r, x, warm=torch.zeros(6, N, dtype=torch.float64),
                            occupation=torch.zeros(6 * N, dtype=torch.float64),
                            out=torch.zeros(3, 2, N, dtype=torch.float64)) == (3, 2)
    bad = [
        dict(rates=torch.ones(3, 2 * n + 1, dtype=torch.float64)),    # wrong rate width
        dict(x0=torch.ones(2, N - 1, dtype=torch.float64)),           # short x0 rows
        dict(x0=torch.ones(2, 2, N, dtype=torch.float64)),            # x0 not R x N
        dict(warm=torch.zeros(5, N, dtype=torch.float64)),            # one system short
        dict(occupation=torch.zeros(6, N, dtype=torch.float32)),      # float32: half the bytes
        dict(occupation=torch.zeros(N, 6, dtype=torch.float64).t()),  # not contiguous
        dict(out=torch.zeros(2, 3, N, dtype=torch.float64)),          # B and R swapped
        dict(warm=np.zeros((6, N))),                                  # not a tensor
    ]
    for kw in bad:
        args = dict(rates=r, x0=x)
        args.update(kw)
        with pytest.raises(ValueError):
            esl._check_batch(n, args.pop("rates"), args.pop("x0"), **args)
    # device buffers must be on the context's device: a host tensor's address is no
    # device address
    with pytest.raises(ValueError, match="cuda:0"):
        esl._check_batch(n, r, x, warm=torch.zeros(6, N, dtype=torch.float64), device=0)
