"""Regenerates tests/golden/reference_goldens.json from the reference checkout.

Run once where the reference is mounted (it is read only as text and, for the
Python CPU path, imported through a shim); the JSON it writes is committed so
the tests never need the reference at run time:

    python tests/golden/make_golden.py /path/to/paraExaStoLog

Contents:
* ``models``: the bnet texts of the reference's ``data/`` models used by its
  known-answer tests (``cuda/test/test.cu``).
* ``cases``: each known-answer test of ``cuda/test/test.cu`` -- model, rates,
  initial state and the expected arrays, parsed from the test source.
* ``python_ref``: x_inf produced by the reference's Python CPU implementation
  (``python/exastolog.py``) for uniform-rate networks: the small-database
  models, the seeded n=10 network and 24 seeded random networks (n = 6-10, terminal
  SCCs of at most 64 states), run through a shim because its optional
  dependencies (pyeda, sortednp, scikit-umfpack) are absent; models above 12
  nodes are skipped (its terminal kernels densify whole attractors).  The Python path
  ignores per-node rates (``exastolog.py:328-331``) and mis-places terminal
  kernels when a weak component holds a cyclic attractor followed by another
  attractor (``exastolog.py:365-375``).  A result is recorded ``"valid": true`` only
  if it sums to 1 and matches the uniformized limit below to L1 1e-9; the others
  (a run that raises included) are recorded with ``"valid": false`` and skipped.
* ``uniformized_limits``: for every model above, lim exp(K t) x0 (uniform rates and
  x0) by repeated squaring of the uniformized chain: an exact answer that depends on
  the transition table alone (``uniformized_limit``).
"""
from __future__ import annotations

import json
import os
import re
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _block(src: str, name: str) -> str:
    start = src.index(f"TEST({name})")
    nxt = src.find("\nTEST(", start + 1)
    return src[start: nxt if nxt >= 0 else len(src)]


def _ints(text: str):
    return [int(v) for v in re.findall(r"-?\d+", text)]


def _floats(text: str):
    return [float(v) for v in re.findall(r"-?\d+\.\d*(?:e[-+]?\d+)?|-?\d+e[-+]?\d+|-?\d+", text)]


def _elements(block: str, var: str):
    m = re.search(r"\b" + var + r",\s*::testing::ElementsAre\(([^)]*)\)", block)
    return m.group(1) if m else None


def _pointwise(block: str):
    m = re.search(r"Pointwise\(::testing::FloatNear\((.*?)\),\s*\{([^}]*)\}", block, re.S)
    return m.group(1), _floats(m.group(2))


def _initial(block: str):
    m = re.search(r"initial_state \w+\(\s*model\.nodes\s*(?:,\s*\{([^}]*)\}\s*,\s*\{([^}]*)\}\s*,\s*([\d.]+)f?)?\s*\)", block)
    if not m or m.group(1) is None:
        return [], []
    names = re.findall(r'"([^"]+)"', m.group(1))
    vals = [1 if v.strip() == "true" else 0 for v in m.group(2).split(",")]
    return names, vals


def _rates(block: str, which: str = "r"):
    m = re.search(which + r"\.generate_uniform\((.*?)\);", block, re.S)
    if not m:
        return {}, {}
    body = m.group(1)
    groups = re.findall(r"\{((?:\s*\{[^}]*\}\s*,?)*)\s*\}", body)
    def parse(g):
        return {k: float(v) for k, v in re.findall(r'\{\s*"([^"]+)"\s*,\s*([\d.]+)f?\s*\}', g)}
    up = parse(groups[0]) if len(groups) > 0 else {}
    down = parse(groups[1]) if len(groups) > 1 else {}
    return up, down


def parse_test_cu(ref: str):
    src = open(os.path.join(ref, "cuda/test/test.cu")).read()
    cases = {}

    b = _block(src, "trans_table, toy")
    cases["trans_table.toy"] = {"model": "toy.bnet", "indptr": _ints(_elements(b, "indptr")),
                                "cols": _ints(_elements(b, "indices")), "source": "cuda/test/test.cu:9-28"}
    b = _block(src, "trans_graph, toy")
    cases["trans_graph.toy"] = {"model": "toy.bnet", "reordered_vertices": _ints(_elements(b, "vertices")),
                                "terminal_offsets": _ints(_elements(b, "offsets")), "source": "cuda/test/test.cu:30-53"}
    b = _block(src, "initial_value, toy")
    names, vals = _initial(b)
    cases["initial_value.toy"] = {"model": "toy.bnet", "fixed": names, "values": vals,
                                  "state": _floats(_elements(b, "state")), "source": "cuda/test/test.cu:55-65"}

    for name, model, lines in [("toy", "toy.bnet", "67-130"), ("toy2", "toy2.bnet", "132-194"),
                               ("toy3", "toy3.bnet", "196-260")]:
        b = _block(src, f"solver, {name}")
        names, vals = _initial(b)
        case = {"model": model, "fixed": names, "values": vals, "source": f"cuda/test/test.cu:{lines}",
                "reordered_vertices": _ints(_elements(b, "vertices")),
                "terminal_offsets": _ints(_elements(b, "offsets")),
                "term_indptr": _ints(_elements(b, "term_indptr")),
                "term_rows": _ints(_elements(b, "term_rows")),
                "nonterm_indptr": _ints(_elements(b, "nonterm_indptr")),
                "nonterm_cols": _ints(_elements(b, "nonterm_cols")),
                "nonzero_indices": _ints(_elements(b, "nonzero_indices"))}
        td = _elements(b, "term_data")
        nd = _elements(b, "nonterm_data")
        fd = _elements(b, "nonzero_data")
        each = re.findall(r"ASSERT_THAT\((\w+), ::testing::Each\(::testing::Eq\(([^)]*)\)\)\)", b)
        eachd = {k: v for k, v in each}
        def ev(expr):
            expr = expr.replace("f", "")
            return float(eval(expr, {"__builtins__": {}}))  # e.g. "1.f / 6.f"
        case["term_data_each"] = ev(eachd["term_data"]) if "term_data" in eachd else None
        case["term_data"] = _floats(td) if td else None
        case["nonterm_data_each"] = ev(eachd["nonterm_data"]) if "nonterm_data" in eachd else None
        case["nonterm_data"] = _floats(nd) if nd else None
        case["nonzero_data_each"] = ev(eachd["nonzero_data"]) if "nonzero_data" in eachd else None
        case["nonzero_data"] = _floats(fd) if fd else None
        cases[f"solver.{name}"] = case

    for name, model, lines in [("kras", "krasmodel15vars.bnet", "262-305"), ("cohen", "EMT_cohen_ModNet.bnet", "307-352"),
                               ("zanudo", "zanudo_expanded.bnet", "354-397")]:
        b = _block(src, f"solver, {name}")
        names, vals = _initial(b)
        tol, probs = _pointwise(b)
        cases[f"solver.{name}"] = {"model": model, "fixed": names, "values": vals, "source": f"cuda/test/test.cu:{lines}",
                                   "nonzero_indices": _ints(_elements(b, "nonzero_indices")), "nonzero_data": probs,
                                   "tolerance": "128*FLT_EPSILON"}

    b = _block(src, "solver, mammal")
    names, vals = _initial(b)
    idx = _ints(b[b.index("expected_indices = {"):].split("{", 1)[1].split("}", 1)[0])
    probs = _floats(b[b.index("expected_probs = {"):].split("{", 1)[1].split("}", 1)[0])
    cases["solver.mammal"] = {"model": "mammalian_cc.bnet", "fixed": names, "values": vals,
                              "source": "cuda/test/test.cu:399-512", "nonzero_indices": idx, "nonzero_data": probs,
                              "tolerance": "1e-7"}

    for name, lines in [("rates, toy", "514-559"), ("zero_rate, toy", "927-969")]:
        b = _block(src, name)
        up, down = _rates(b)
        tol, probs = _pointwise(b)
        cases[name.replace(", ", ".")] = {"model": "toy.bnet", "fixed": [], "values": [], "up": up, "down": down,
                                          "source": f"cuda/test/test.cu:{lines}",
                                          "nonzero_indices": _ints(_elements(b, "nonzero_indices")),
                                          "nonzero_data": probs, "tolerance": "128*FLT_EPSILON"}

    b = _block(src, "symbolic_with_refactor, cohen")
    up, down = _rates(b, "r2")
    st = re.search(r"initial_state st\(\s*model\.nodes,\s*\{([^}]*)\}\s*,\s*\{([^}]*)\}", b)
    names = re.findall(r'"([^"]+)"', st.group(1))
    vals = [1 if v.strip() == "true" else 0 for v in st.group(2).split(",")]
    tol, probs = _pointwise(b)
    cases["symbolic.cohen_rates"] = {"model": "EMT_cohen_ModNet.bnet", "fixed": names, "values": vals, "up": up,
                                     "down": down, "source": "cuda/test/test.cu:860-925",
                                     "nonzero_indices": _ints(_elements(b, "nonzero_indices")),
                                     "nonzero_data": probs, "tolerance": "128*FLT_EPSILON"}
    return cases


def uniformized_limit(text: str) -> np.ndarray:
    """lim_{t->inf} exp(K t) x0 for the uniform x0 and uniform rates, by repeated
    squaring of the uniformized chain P = I + K / q (q above every exit rate, so P is
    aperiodic), columns renormalised after each squaring.  Dense, for small n only.
    It uses the transition table alone (the oracle's flip masks, which the reference's
    table goldens pin) and none of the SCC or solver logic, so it can judge a result of
    the Python path independently of the oracle's solve."""
    sys.path.insert(0, REPO)
    import oracle as O
    m = O.Model(text=text)
    r = m.rates()
    N = 1 << m.n
    F = np.asarray(m.flip_masks(r)).astype(np.int64)
    K = np.zeros((N, N))
    s = np.arange(N)
    for b in range(m.n):
        src = s[((F >> b) & 1) == 1]
        rate = np.where(((src >> b) & 1) == 0, r[2 * b], r[2 * b + 1])
        K[src ^ (1 << b), src] += rate
        K[src, src] -= rate
    P = np.eye(N) + K / (1.5 * max(-K.diagonal().min(), 1e-300))
    x0 = np.full(N, 1.0 / N)
    prev = None
    for _ in range(64):
        P = P @ P
        P /= P.sum(0, keepdims=True)
        x = P @ x0
        if prev is not None and np.abs(x - prev).sum() <= 1e-15:
            break
        prev = x
    return x


def python_reference(ref: str, models: dict, max_nodes: int = 12):
    """x_inf of the reference's Python path for uniform rates and uniform x0."""
    sys.modules.setdefault("pyeda", types.ModuleType("pyeda"))
    sys.modules.setdefault("pyeda.inter", types.ModuleType("pyeda.inter"))
    sn = types.ModuleType("sortednp")
    sn.DROP = 0
    sn.kway_merge = lambda *arrs, duplicates=None: np.unique(np.concatenate(arrs)).astype(int)
    sys.modules["sortednp"] = sn
    import scipy.sparse.linalg as spla
    spla.use_solver = lambda **kw: None
    _spsolve = spla.spsolve
    spla.spsolve = lambda A, b, use_umfpack=False, **kw: _spsolve(A, b, use_umfpack=False)
    sys.path.insert(0, os.path.join(ref, "python"))
    import exastolog as ex
    ex.USE_SYMPY = True
    import tempfile
    out = {}
    for key, text in models.items():
        with tempfile.NamedTemporaryFile("w", suffix=".bnet", delete=False) as f:
            f.write(text)
            path = f.name
        try:
            model = ex.Model(path)
            if len(model.model) > max_nodes:
                continue
            table = ex.TransitionTable(model)
            table.build_transition_table()
            init = ex.InitialState(model)
            graph = ex.TransitionGraph(table, init)
            graph.sort()
            sol = ex.Solution(graph, init, len(model.model.keys()))
            try:
                x = np.asarray(sol.compute_final_states(), dtype=float)
            except Exception as e:  # the Python path's own failure: recorded, not a golden
                out[key] = {"valid": False, "error": f"{type(e).__name__}: {e}",
                            "source": "python/exastolog.py (shimmed)"}
                continue
            nz = np.nonzero(x)[0]
            # valid only where it matches the uniformized limit (a sum of 1 is not
            # enough: the path can misplace mass and still sum to 1)
            l1 = float(np.abs(x - uniformized_limit(text)).sum())
            out[key] = {"nonzero_indices": nz.tolist(), "nonzero_data": x[nz].tolist(),
                        "valid": bool(abs(x.sum() - 1.0) < 1e-9 and l1 <= 1e-9), "l1_vs_uniformized_limit": l1,
                        "source": "python/exastolog.py (shimmed)"}
        finally:
            os.unlink(path)
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/paraExaStoLog")
    ref = sys.argv[1]
    data = os.path.join(ref, "data")
    names = ["toy.bnet", "toy2.bnet", "toy3.bnet", "krasmodel15vars.bnet", "mammalian_cc.bnet",
             "EMT_cohen_ModNet.bnet", "zanudo_expanded.bnet"]
    models = {nm: open(os.path.join(data, nm)).read() for nm in names}
    small = {}
    for nm in sorted(os.listdir(os.path.join(data, "database-small"))):
        small["database-small/" + nm] = open(os.path.join(data, "database-small", nm)).read()
    models.update(small)
    cases = parse_test_cu(ref)

    sys.path.insert(0, REPO)
    from paraexastolog_b200 import synth
    gen = {"synth.n10_k2_uniform": synth.config_small().networks[0].bnet}
    # seeded random uniform-rate networks whose terminal SCCs are small enough for the
    # Python path's O(s^4) cofactor kernels (at most 64 states)
    import oracle as O
    rng = np.random.default_rng(20)
    while len(gen) < 25:
        n = int(rng.integers(6, 11))
        text = synth.random_table_network(rng, n, [1, 2, 3], 0.5).bnet
        m = O.Model(text=text)
        sym = m.analyse(m.rates())
        if np.diff(sym.offsets[: sym.T + 1]).max() <= 64:
            gen[f"synth.random_{len(gen)}_n{n}"] = text
    pyref_models = dict(small)
    pyref_models.update(gen)
    pyref_models["toy.bnet"] = models["toy.bnet"]
    pyref_models["krasmodel15vars.bnet"] = models["krasmodel15vars.bnet"]
    pyref = python_reference(ref, pyref_models)

    # the uniformized limit of every model the Python path ran on: an exact answer for
    # uniform rates and x0 that does not depend on any solver, including where that
    # path is wrong
    limits = {}
    for key, text in pyref_models.items():
        if key not in pyref:
            continue
        x = uniformized_limit(text)
        nz = np.nonzero(x > 1e-15)[0]  # entries below count for nothing at the tests' 1e-10
        limits[key] = {"nonzero_indices": nz.tolist(), "nonzero_data": x[nz].tolist(),
                       "source": "uniformized chain, repeated squaring (make_golden.uniformized_limit)"}

    out = {"models": models, "generated_models": gen, "cases": cases, "python_ref": pyref,
           "uniformized_limits": limits}
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("cases:", len(cases), "python_ref:", {k: v["valid"] for k, v in pyref.items()})


if __name__ == "__main__":
    main()
