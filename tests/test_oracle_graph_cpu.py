"""The oracle's table and graph stages against independent computations.  The table:
from the generator's truth tables, without the bnet text.  The graph: strongly connected
components from scipy (scipy.sparse.csgraph), terminal SCCs as the sinks of the
condensation, and levels by a longest-path recursion over the condensation (level 1 =
terminal, otherwise 1 + the largest level of a successor SCC).  The reference's own
known-answer tests pin these stages only on its toy models; this covers random
networks of the three families behind the workloads, with zero rates."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

import oracle as O
from paraexastolog_b200 import synth


def _independent(F):
    n = int(np.log2(F.size))
    N = F.size
    s = np.arange(N, dtype=np.int64)
    F = F.astype(np.int64)
    src, dst = [], []
    for b in range(n):
        v = s[((F >> b) & 1) == 1]
        src.append(v)
        dst.append(v ^ (1 << b))
    src, dst = np.concatenate(src), np.concatenate(dst)
    g = sp.csr_matrix((np.ones(src.size), (src, dst)), shape=(N, N))
    k, comp = connected_components(g, directed=True, connection="strong")
    # condensation edges and levels (longest path to a sink, sinks at 1)
    cs, cd = comp[src], comp[dst]
    cross = cs != cd
    succ = [[] for _ in range(k)]
    for a, b in set(zip(cs[cross].tolist(), cd[cross].tolist())):
        succ[a].append(b)
    level = np.zeros(k, np.int64)
    order = []
    state = np.zeros(k, np.int8)
    for root in range(k):  # iterative post-order DFS
        if state[root]:
            continue
        stack = [(root, 0)]
        state[root] = 1
        while stack:
            c, i = stack[-1]
            if i < len(succ[c]):
                stack[-1] = (c, i + 1)
                nxt = succ[c][i]
                if not state[nxt]:
                    state[nxt] = 1
                    stack.append((nxt, 0))
            else:
                stack.pop()
                level[c] = 1 + max((level[x] for x in succ[c]), default=0)
    return comp, level


@pytest.mark.parametrize("family", ["table", "nested_canalizing", "precision"])
def test_graph_stages_match_scipy(family):
    rng = np.random.default_rng({"table": 21, "nested_canalizing": 22, "precision": 23}[family])
    for seed in range(6):
        n = int(rng.integers(8, 13))
        if family == "table":
            net = synth.random_table_network(rng, n, [1, 2, 3], 0.5)
        elif family == "nested_canalizing":
            net = synth.nested_canalizing_network(rng, n, 3)
        else:
            net = synth.precision_network(seed, n)
        rates = synth.log_uniform_rates(rng, n, 1)[0]
        rates[rng.choice(2 * n, 2, replace=False)] = 0.0
        m = O.Model(text=net.bnet)
        sym = m.analyse(rates)
        comp, level = _independent(np.asarray(m.flip_masks(rates)))
        labels = np.asarray(sym.labels)
        # same partition: canonical label = smallest state of the SCC
        canon = np.full(comp.max() + 1, 1 << 30)
        np.minimum.at(canon, comp, np.arange(comp.size))
        assert np.array_equal(labels, canon[comp]), (family, seed)
        # order: every SCC contiguous, terminals first, then levels non-increasing
        order, offs = np.asarray(sym.order), np.asarray(sym.offsets)
        lev_at = np.asarray(sym.levels)[: sym.n_sccs]
        assert sym.n_sccs == comp.max() + 1
        for j in range(sym.n_sccs):
            members = order[offs[j]:offs[j + 1]]
            assert np.all(comp[members] == comp[members[0]])
            assert lev_at[j] == level[comp[members[0]]], (family, seed, j)
        assert np.all(lev_at[: sym.T] == 1) and np.all(lev_at[sym.T:] > 1)
        assert np.all(np.diff(lev_at[sym.T:]) <= 0)
        assert sym.T == int(np.sum(level == 1))


@pytest.mark.parametrize("family", ["table", "nested_canalizing", "precision"])
def test_table_matches_the_truth_tables(family):
    # the transition table from the generator's truth tables alone (no bnet text, no
    # DNF): node i flips in state s iff its rule disagrees with bit i and the rate of
    # that direction is not zero; the CSC lists each source's destinations ascending
    rng = np.random.default_rng({"table": 31, "nested_canalizing": 32, "precision": 33}[family])
    for seed in range(6):
        n = int(rng.integers(6, 12))
        if family == "table":
            net = synth.random_table_network(rng, n, [1, 2, 3, 4], 0.5)
        elif family == "nested_canalizing":
            net = synth.nested_canalizing_network(rng, n, 3)
        else:
            net = synth.precision_network(seed, n)
        rates = synth.log_uniform_rates(rng, n, 1)[0]
        rates[rng.choice(2 * n, 3, replace=False)] = 0.0
        N = 1 << n
        s = np.arange(N, dtype=np.int64)
        F = np.zeros(N, np.int64)
        for i in range(n):
            idx = np.zeros(N, np.int64)
            for j, inp in enumerate(net.inputs[i]):
                idx |= ((s >> inp) & 1) << j
            f = np.asarray(net.tables[i], bool)[idx]
            bit = ((s >> i) & 1).astype(bool)
            rate_ok = np.where(bit, rates[2 * i + 1] != 0.0, rates[2 * i] != 0.0)
            F |= ((f != bit) & rate_ok).astype(np.int64) << i
        m = O.Model(text=net.bnet)
        assert np.array_equal(np.asarray(m.flip_masks(rates)).astype(np.int64), F), (family, seed)
        indptr, rows, cols = m.table(rates)
        deg = np.array([bin(int(v)).count("1") for v in F])
        assert np.array_equal(np.diff(indptr), deg)
        expect_rows = np.concatenate([np.sort(v ^ (1 << np.nonzero((F[v] >> np.arange(n)) & 1)[0]))
                                      for v in range(N)])
        assert np.array_equal(rows, expect_rows) and np.array_equal(cols, np.repeat(np.arange(N), deg))
