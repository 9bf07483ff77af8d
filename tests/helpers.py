"""Shared helpers for the tests (not product code)."""
import numpy as np

FLT_EPS = float(np.finfo(np.float32).eps)


def reference_L_csr(order, offsets, T, L_dense):
    """The reference's ``solution_nonterm`` layout (``cuda/src/solver.cu:205-300``):
    row t = the states of terminal SCC t (value 1) followed by the transient
    states with a nonzero absorption probability, in reordered position."""
    term_states = int(offsets[T])
    indptr, cols, data = [0], [], []
    for t in range(T):
        for p in range(offsets[t], offsets[t + 1]):
            cols.append(int(order[p])); data.append(1.0)
        for p in range(term_states, len(order)):
            v = L_dense[t, order[p]]
            if v != 0.0:
                cols.append(int(order[p])); data.append(float(v))
        indptr.append(len(cols))
    return indptr, cols, data


def nonzeros(x):
    idx = np.nonzero(x)[0]
    return idx, x[idx]
