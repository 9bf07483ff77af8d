"""CPU checks of the MLP oracle (oracle/mlp.py) that the GPU gradient test relies on:
its gradient against central finite differences, BF16 rounding, and the feature and
reachability restatements on a small network."""
import numpy as np
import pytest

import oracle as O
from oracle import mlp as OM
from paraexastolog_b200 import synth


def _params(rng):
    p = np.zeros(OM.N_PARAMS)
    d = OM.unpack(p)
    d["W1"][:] = rng.normal(0, 0.3, d["W1"].shape)
    d["b1"][:] = rng.normal(0, 0.1, d["b1"].shape)
    d["W2"][:] = rng.normal(0, 0.2, d["W2"].shape)
    d["b2"][:] = rng.normal(0, 0.1, d["b2"].shape)
    d["w3"][:] = rng.normal(0, 0.2, d["w3"].shape)
    d["b3"][:] = 0.3
    return OM.pack(d)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    X = rng.normal(0, 1, (24, OM.N_IN))
    t = rng.normal(0, 1, 24)
    loss, g = OM.loss_grad(p, X, t, rnd=False)
    idx = np.concatenate([rng.choice(OM.N_PARAMS, 60, replace=False), [OM.N_PARAMS - 1]])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (OM.loss_grad(pp, X, t, rnd=False)[0] - OM.loss_grad(pm, X, t, rnd=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_round():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0, 1e-3], np.float32)
    r = OM.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie rounds to even
    assert r[2] == np.float32(1.0078125)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_features_and_reach_small_network():
    w = synth.config_precision(seed=3, n=14, n_rate_sets=4)
    m = O.Model(text=w.networks[0].bnet)
    rates = w.rates[0]
    sym = m.analyse(rates[0])
    F = m.flip_masks(rates[0])
    reach = OM.reach_bits(sym, F)
    T = sym.T
    term = np.full(sym.N, -1)
    for t in range(T):
        term[sym.order[sym.offsets[t]:sym.offsets[t + 1]]] = t
    # terminal states reach exactly themselves; every transient state reaches something
    assert np.all(reach[term >= 0] == (np.uint32(1) << term[term >= 0].astype(np.uint32)))
    assert np.all(reach[term < 0] != 0)
    # a transient state's set is the union over its successors outside its SCC
    rng = np.random.default_rng(1)
    for v in rng.choice(np.nonzero(term < 0)[0], 50, replace=False):
        u = [v ^ (1 << i) for i in range(14) if (F[v] >> i) & 1]
        want = np.bitwise_or.reduce([reach[x] for x in u] + [np.uint32(0)])
        assert reach[v] == want
    X = OM.features(14, T, F, reach, rates, [0, 3], [5, 77])
    assert X.shape == (2, OM.N_IN)
    assert set(np.unique(X[:, :14])) <= {-1.0, 1.0} and np.all(X[:, 14:20] == 0)
    assert np.allclose(X[1, 37:37 + 28], np.log(rates[3]))
    assert np.all(X[:, 37 + 28:] == 0)
