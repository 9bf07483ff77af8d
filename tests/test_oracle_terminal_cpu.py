"""The oracle against exact answers that need no solver.

- Terminal kernels of SCCs too large for its dense LU (more than 2,048 states), which
  it solves by BiCGStab on the rank-one deflated system (-K_C + u 1^T) pi = u: a closed
  form, and the generator residual on the largest attractor of the many-network
  workload (n = 18: all 262,144 states in one terminal SCC).
- The iterative transient path: a closed form from a symmetry of the chain.
- Per-node rates (some zero) and non-uniform x0 on small networks: the limit of the
  uniformized chain by repeated squaring."""
import numpy as np
import pytest

import oracle as O
from paraexastolog_b200 import synth


def _generator_residual(F, rates, pi):
    """|K pi|_1 / sum_v q_v pi_v for the generator K (K[dst, src] = rate, columns sum to 0)."""
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


def test_large_attractor_closed_form():
    # every node negates itself: the whole 4,096-state cube is one terminal SCC and its
    # kernel is the product of the per-node two-state chains
    n = 12
    m = O.Model(text="targets, factors\n" + "".join(f"v{i}, !v{i}\n" for i in range(n)))
    rates = synth.log_uniform_rates(np.random.default_rng(5), n, 1)[0]
    sym = m.analyse(rates)
    assert sym.T == 1 and sym.N == 1 << n
    pi = sym.terminal_kernels(rates)
    assert O.iterative_blocks() == 1  # the iterative path, not the dense LU
    s = np.arange(1 << n)
    expect = np.ones(1 << n)
    for i in range(n):
        up, down = rates[2 * i], rates[2 * i + 1]
        expect *= np.where((s >> i) & 1, up / (up + down), down / (up + down))
    order = np.asarray(sym.order)
    got = np.empty(1 << n)
    got[order] = pi
    np.testing.assert_allclose(got, expect, rtol=1e-11, atol=1e-15)


def test_largest_attractor_of_the_many_network_workload():
    w = synth.config_batch()
    net, rates = w.networks[10], w.rates[10][0]
    m = O.Model(text=net.bnet)
    sym = m.analyse(rates)
    assert sym.T == 1 and sym.N == 1 << 18 and sym.offsets[1] == sym.N
    pi = sym.terminal_kernels(rates)
    assert O.last_relres() <= 1e-13
    assert abs(pi.sum() - 1.0) <= 1e-12 and pi.min() >= 0.0
    full = np.empty(sym.N)
    full[np.asarray(sym.order)] = pi
    assert _generator_residual(np.asarray(m.flip_masks(rates)), rates, full) <= 1e-12


def test_large_transient_block_closed_form():
    # v0 latches on from the all-ones corner of the free nodes, v1 from the all-zeros
    # corner; the other nodes flip freely.  Terminal SCCs: (v0, v1) = (1, 0), (0, 1) and
    # (1, 1), each uniform over the 4,096 states of the free nodes; the 4,096-state block
    # (0, 0) is transient.  With equal rates, swapping v0 and v1 and complementing the
    # free nodes maps the chain to itself, so the block's mass splits evenly: from a
    # uniform x0, (1, 0) and (0, 1) end with 3/8 each and (1, 1) keeps its 1/4.
    n = 14
    free = range(2, n)
    text = ("targets, factors\n"
            f"v0, v0 | (!v1 & {' & '.join(f'v{i}' for i in free)})\n"
            f"v1, v1 | (!v0 & {' & '.join(f'!v{i}' for i in free)})\n" +
            "".join(f"v{i}, !v{i}\n" for i in free))
    m = O.Model(text=text)
    rates = m.rates()
    sym = m.analyse(rates)
    assert sym.T == 3 and sym.n_sccs == 4
    x, marg = sym.solve(m.initial_state(), rates)
    assert O.iterative_blocks() >= 1
    s = np.arange(1 << n)
    b0, b1 = s & 1, (s >> 1) & 1
    expect = np.where(b0 & ~b1 & 1, 0.375, 0.0) + np.where(~b0 & b1 & 1, 0.375, 0.0) + np.where(b0 & b1, 0.25, 0.0)
    expect /= 1 << (n - 2)
    assert np.abs(x - expect).sum() <= 1e-10
    np.testing.assert_allclose(marg[:2], [0.625, 0.625], rtol=0, atol=1e-11)
    np.testing.assert_allclose(marg[2:], 0.5, rtol=0, atol=1e-11)


def _limit_matrix(F, rates):
    """lim exp(K t) by repeated squaring of the uniformized chain (columns renormalised);
    uses the transition table only."""
    n = int(np.log2(F.size))
    N = F.size
    s = np.arange(N, dtype=np.int64)
    F = F.astype(np.int64)
    K = np.zeros((N, N))
    for b in range(n):
        src = s[((F >> b) & 1) == 1]
        rate = np.where(((src >> b) & 1) == 0, rates[2 * b], rates[2 * b + 1])
        K[src ^ (1 << b), src] += rate
        K[src, src] -= rate
    P = np.eye(N) + K / (1.5 * max(-K.diagonal().min(), 1e-300))
    for _ in range(80):
        P = P @ P
        P /= P.sum(0, keepdims=True)
    return P


def _limit(F, rates, x0):
    return _limit_matrix(F, rates) @ x0


def test_oracle_matches_the_uniformized_limit_with_rates():
    # per-node log-uniform rates, some of them zero, and Dirichlet x0 over a node subset:
    # the cases the reference's Python path cannot solve (it ignores rates)
    rng = np.random.default_rng(11)
    for _ in range(12):
        n = int(rng.integers(5, 9))
        net = synth.random_table_network(rng, n, [1, 2, 3], 0.5)
        rates = synth.log_uniform_rates(rng, n, 1)[0]
        rates[rng.choice(2 * n, 2, replace=False)] = 0.0
        x0 = synth.dirichlet_subspace_x0(rng, n, rng.choice(n, 3, replace=False))
        m = O.Model(text=net.bnet)
        x, _ = m.analyse(rates).solve(x0, rates)
        exact = _limit(np.asarray(m.flip_masks(rates)), rates, x0)
        assert np.abs(x - exact).sum() <= 1e-10


@pytest.mark.parametrize("family", ["nested_canalizing", "precision"])
def test_oracle_matches_the_uniformized_limit_on_workload_families(family):
    # the two other generators behind the workloads, at small n: nested-canalizing
    # rules (the drop-in workload) and Bernoulli(0.3) tables with self-holding source
    # nodes (the precision and learned workloads: several attractors, cyclic ones too)
    rng = np.random.default_rng(12 if family == "precision" else 13)
    for seed in range(8):
        n = int(rng.integers(6, 9))
        if family == "precision":
            net = synth.precision_network(seed, n)
        else:
            net = synth.nested_canalizing_network(rng, n, 3)
        rates = synth.log_uniform_rates(rng, n, 1)[0]
        x0 = synth.dirichlet_subspace_x0(rng, n, rng.choice(n, 3, replace=False))
        m = O.Model(text=net.bnet)
        x, _ = m.analyse(rates).solve(x0, rates)
        exact = _limit(np.asarray(m.flip_masks(rates)), rates, x0)
        assert np.abs(x - exact).sum() <= 1e-10, (family, seed)


def test_absorption_matrix_matches_the_limit_matrix():
    # L[t, s]: the probability of ending in terminal SCC t from state s, which is the
    # mass the limit matrix moves from s onto t's states (backward formulation)
    rng = np.random.default_rng(17)
    for _ in range(8):
        n = int(rng.integers(5, 9))
        net = synth.random_table_network(rng, n, [1, 2, 3], 0.5)
        rates = synth.log_uniform_rates(rng, n, 1)[0]
        m = O.Model(text=net.bnet)
        sym = m.analyse(rates)
        Lm = sym.absorption(rates)
        P = _limit_matrix(np.asarray(m.flip_masks(rates)), rates)
        order, offs = np.asarray(sym.order), np.asarray(sym.offsets)
        expect = np.stack([P[order[offs[t]:offs[t + 1]]].sum(0) for t in range(sym.T)])
        assert np.abs(Lm - expect).max() <= 1e-10
        np.testing.assert_allclose(Lm.sum(0), 1.0, rtol=0, atol=1e-11)
