"""Seeded synthetic workloads: random asynchronous Boolean networks written as bnet.

The reference ships no network generator and no public benchmark suite; its
models live in ``data/*.bnet``.  The workloads used by the tests and the
benchmark are therefore generated here, with fixed seeds, in the bnet dialect
that ``model_builder::construct_model`` reads (``cuda/src/model.cpp:80-125``):
a ``targets, factors`` header, then one ``name, expression`` line per node,
expressions over ``! & | ( )`` and identifiers, every line newline-terminated.

Each rule is written as the disjunction of the minterms of its truth table over
its inputs, so the transition function of node ``i`` is exactly the truth
table drawn here.  Node ``i`` is bit ``i`` of the state index (bnet line order,
``cuda/src/model.cpp:98-110``).

Workloads (sizes and distributions as stated for each function):

* ``config_small``      n=10, k=2 inputs, Bernoulli(0.5) tables, all rates 1.0,
                        uniform x0 (the CPU-runnable case).
* ``config_scale``      n=22, k=3 nested-canalizing rules, log-uniform rates in
                        [0.1, 10], x0 uniform over states with 4 nodes fixed.
* ``config_precision``  n=20, 3 self-holding source nodes, k~U{2,3,4},
                        Bernoulli(0.3) tables, log-uniform rates, x0 Dirichlet(1)
                        over the 2^8 assignments of 8 random nodes.
* ``config_batch``      48 networks, n~U{12..18}, k=3, Bernoulli(0.5) tables,
                        64 rate sets and 16 x0 (Dirichlet(1) over a random
                        6-node subspace) per network.
* ``config_learned``    the precision network with 4,096 rate sets
                        (3,584 train / 512 held out).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class Network:
    """A generated network: bnet text plus the truth tables it was written from."""

    names: List[str]
    inputs: List[List[int]]        # per node, its input node indices (table bit order)
    tables: List[np.ndarray]       # per node, bool array of length 2**len(inputs)
    bnet: str

    @property
    def n(self) -> int:
        return len(self.names)


def _literal(name: str, value: int) -> str:
    return name if value else "!" + name


def _rule_text(names: List[str], inputs: List[int], table: np.ndarray) -> str:
    """Minterm DNF of ``table``: entry ``m`` has input ``j`` equal to bit ``j`` of ``m``."""
    terms = []
    for m in range(len(table)):
        if table[m]:
            lits = [_literal(names[inp], (m >> j) & 1) for j, inp in enumerate(inputs)]
            terms.append("(" + " & ".join(lits) + ")")
    return " | ".join(terms)


def network_to_bnet(names: List[str], inputs: List[List[int]], tables: List[np.ndarray]) -> str:
    lines = ["targets, factors"]
    for i, name in enumerate(names):
        lines.append(f"{name}, {_rule_text(names, inputs[i], tables[i])}")
    return "\n".join(lines) + "\n"


def _names(n: int) -> List[str]:
    return [f"x{i:02d}" for i in range(n)]


def random_table_network(rng: np.random.Generator, n: int, k_choices, p_one: float,
                         sources: Optional[List[int]] = None) -> Network:
    """Each non-source node draws k from ``k_choices`` distinct inputs uniformly
    from all n nodes (itself included) and a Bernoulli(p_one) truth table;
    constant tables are redrawn.  A source node's rule is its own name, so it
    never flips."""
    names = _names(n)
    sources = set(sources or [])
    inputs, tables = [], []
    for i in range(n):
        if i in sources:
            inputs.append([i])
            tables.append(np.array([False, True]))
            continue
        k = int(rng.choice(k_choices))
        inp = [int(v) for v in rng.choice(n, size=k, replace=False)]
        while True:
            tab = rng.random(2 ** k) < p_one
            if tab.any() and not tab.all():
                break
        inputs.append(inp)
        tables.append(tab)
    return Network(names, inputs, tables, network_to_bnet(names, inputs, tables))


def nested_canalizing_network(rng: np.random.Generator, n: int, k: int) -> Network:
    """f = x_a1==c1 ? o1 : (x_a2==c2 ? o2 : ... (x_ak==ck ? ok : !ok)) with the
    canalizing values c and outputs o Bernoulli(0.5)."""
    names = _names(n)
    inputs, tables = [], []
    for _ in range(n):
        inp = [int(v) for v in rng.choice(n, size=k, replace=False)]
        canal = rng.integers(0, 2, size=k)
        outs = rng.integers(0, 2, size=k)
        tab = np.zeros(2 ** k, dtype=bool)
        for m in range(2 ** k):
            val = not outs[-1]
            for j in range(k):
                if ((m >> j) & 1) == canal[j]:
                    val = bool(outs[j])
                    break
            tab[m] = val
        inputs.append(inp)
        tables.append(tab)
    return Network(names, inputs, tables, network_to_bnet(names, inputs, tables))


def log_uniform_rates(rng: np.random.Generator, n: int, count: int, lo=0.1, hi=10.0) -> np.ndarray:
    """``count`` rate sets, each ``[up_0, down_0, ..., up_{n-1}, down_{n-1}]``
    (the layout of ``cuda/src/transition_rates.cpp:24-58``), log-uniform in [lo, hi]."""
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=(count, 2 * n)))


def fixed_nodes_x0(n: int, fixed_nodes, fixed_values) -> np.ndarray:
    """Uniform over the states whose ``fixed_nodes`` equal ``fixed_values``
    (``cuda/src/initial_state.cu:7-60`` with fixed_probability 1)."""
    s = np.arange(1 << n, dtype=np.int64)
    mask = np.ones(1 << n, dtype=bool)
    for node, val in zip(fixed_nodes, fixed_values):
        mask &= ((s >> node) & 1) == int(val)
    x0 = np.zeros(1 << n)
    x0[mask] = 1.0 / mask.sum()
    return x0


def dirichlet_subspace_x0(rng: np.random.Generator, n: int, nodes) -> np.ndarray:
    """Dirichlet(1) weights over the 2^len(nodes) assignments of ``nodes``,
    spread uniformly over the states of each assignment."""
    nodes = list(nodes)
    w = rng.dirichlet(np.ones(2 ** len(nodes)))
    s = np.arange(1 << n, dtype=np.int64)
    a = np.zeros(1 << n, dtype=np.int64)
    for j, node in enumerate(nodes):
        a |= ((s >> node) & 1) << j
    return w[a] / float(1 << (n - len(nodes)))


@dataclasses.dataclass
class Workload:
    name: str
    networks: List[Network]
    rates: List[np.ndarray]        # per network, (B, 2n) float64
    x0: List[np.ndarray]           # per network, (R, 2^n) float64
    notes: str = ""


def config_small(seed: int = 0) -> Workload:
    rng = np.random.default_rng(seed)
    net = random_table_network(rng, 10, [2], 0.5)
    rates = np.ones((1, 2 * net.n))
    x0 = np.full((1, 1 << net.n), 1.0 / (1 << net.n))
    return Workload("n10_k2_uniform", [net], [rates], [x0])


def config_scale(seed: int = 1) -> Workload:
    rng = np.random.default_rng(seed)
    n = 22
    net = nested_canalizing_network(rng, n, 3)
    rates = log_uniform_rates(rng, n, 1)
    nodes = rng.choice(n, size=4, replace=False)
    vals = rng.integers(0, 2, size=4)
    x0 = fixed_nodes_x0(n, nodes, vals)[None, :]
    return Workload("n22_k3_canalizing", [net], [rates], [x0])


def precision_network(seed: int = 2, n: int = 20) -> Network:
    rng = np.random.default_rng(seed)
    sources = sorted(int(v) for v in rng.choice(n, size=3, replace=False))
    return random_table_network(rng, n, [2, 3, 4], 0.3, sources=sources)


def config_precision(seed: int = 2, n: int = 20, n_rate_sets: int = 1) -> Workload:
    net = precision_network(seed, n)
    rng = np.random.default_rng(seed + 1000)
    rates = log_uniform_rates(rng, n, n_rate_sets)
    nodes = rng.choice(n, size=8, replace=False)
    x0 = dirichlet_subspace_x0(rng, n, nodes)[None, :]
    return Workload(f"n{n}_precision", [net], [rates], [x0])


def config_learned(seed: int = 2, n: int = 20, n_rate_sets: int = 4096, n_train: int = 3584) -> Workload:
    w = config_precision(seed, n, n_rate_sets)
    w.name = f"n{n}_learned_{n_rate_sets}"
    w.notes = f"train={n_train} heldout={n_rate_sets - n_train}"
    return w


def config_batch(seed: int = 3, n_networks: int = 48, n_rate_sets: int = 64, n_x0: int = 16,
                 n_lo: int = 12, n_hi: int = 18) -> Workload:
    rng = np.random.default_rng(seed)
    nets, rates, x0s = [], [], []
    for _ in range(n_networks):
        n = int(rng.integers(n_lo, n_hi + 1))
        net = random_table_network(rng, n, [3], 0.5)
        nets.append(net)
        rates.append(log_uniform_rates(rng, n, n_rate_sets))
        xs = [dirichlet_subspace_x0(rng, n, rng.choice(n, size=6, replace=False)) for _ in range(n_x0)]
        x0s.append(np.stack(xs))
    return Workload("batch48_n12_18", nets, rates, x0s)
