"""ctypes binding of the CPU FP64 oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only to check or time against it.  The
oracle restates the reference's algorithm (see the header of
``esl_oracle.cpp`` for the file:line each part follows).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libesl_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp, cp, i32p, u32p, f64p = C.c_void_p, C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_uint32), C.POINTER(C.c_double)
    L.eo_last_error.restype = cp
    L.eo_last_relres.restype = C.c_double
    L.eo_iterative_blocks.restype = C.c_int
    L.eo_parse_bnet.restype = vp
    L.eo_parse_bnet.argtypes = [cp]
    L.eo_load_bnet.restype = vp
    L.eo_load_bnet.argtypes = [cp]
    L.eo_free_net.argtypes = [vp]
    L.eo_n.argtypes = [vp]
    L.eo_node_name.restype = cp
    L.eo_node_name.argtypes = [vp, C.c_int]
    L.eo_clauses.argtypes = [vp, i32p, u32p, u32p, C.c_int]
    L.eo_flip_masks.argtypes = [vp, f64p, u32p]
    L.eo_table.restype = C.c_int64
    L.eo_table.argtypes = [vp, f64p, i32p, i32p, i32p]
    L.eo_build.restype = vp
    L.eo_build.argtypes = [vp, f64p]
    L.eo_free_sym.argtypes = [vp]
    L.eo_n_sccs.argtypes = [vp]
    L.eo_n_terminals.argtypes = [vp]
    L.eo_graph.argtypes = [vp, i32p, i32p, i32p, i32p]
    L.eo_terminal_kernels.argtypes = [vp, f64p, f64p]
    L.eo_absorption.argtypes = [vp, f64p, f64p]
    L.eo_terminal_mass.argtypes = [vp, f64p, f64p, f64p]
    L.eo_solve.argtypes = [vp, f64p, f64p, f64p, f64p, C.c_int]
    L.eo_solve_many.argtypes = [vp, C.c_int, f64p, f64p, f64p, f64p, C.c_int]
    L.eo_initial_state.argtypes = [C.c_int, C.c_int, i32p, i32p, C.c_double, f64p]
    L.eo_rates_normal.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, f64p, f64p, f64p]
    _lib = L
    return L


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleError(RuntimeError):
    pass


class Model:
    """A parsed bnet model (``cuda/src/model.cpp:80-125`` semantics)."""

    def __init__(self, text: str | None = None, path: str | None = None):
        L = lib()
        h = L.eo_parse_bnet(text.encode()) if text is not None else L.eo_load_bnet(path.encode())
        if not h:
            raise OracleError(L.eo_last_error().decode())
        self._h = h
        self.n = L.eo_n(h)
        self.names = [L.eo_node_name(h, i).decode() for i in range(self.n)]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.eo_free_net(self._h)
            self._h = None

    def clauses(self):
        L = lib()
        total = L.eo_clauses(self._h, None, None, None, 0)
        off = np.zeros(self.n + 1, np.int32)
        pos = np.zeros(max(total, 1), np.uint32)
        neg = np.zeros(max(total, 1), np.uint32)
        L.eo_clauses(self._h, _p(off, C.c_int32), _p(pos, C.c_uint32), _p(neg, C.c_uint32), total)
        return off, pos[:total], neg[:total]

    def rates(self, up=None, down=None, default=1.0) -> np.ndarray:
        """``transition_rates::generate_uniform`` (``cuda/src/transition_rates.cpp:24-73``)."""
        r = np.full(2 * self.n, float(default))
        for name, v in (up or {}).items():
            r[2 * self.names.index(name)] = v
        for name, v in (down or {}).items():
            r[2 * self.names.index(name) + 1] = v
        return r

    def rates_normal(self, mean, std, seed=0, up=None, down=None) -> np.ndarray:
        """``transition_rates::generate_normal`` (``cuda/src/transition_rates.cpp:75-97``)."""
        up_set = np.full(self.n, -1.0)
        down_set = np.full(self.n, -1.0)
        for name, v in (up or {}).items():
            up_set[self.names.index(name)] = v
        for name, v in (down or {}).items():
            down_set[self.names.index(name)] = v
        r = np.zeros(2 * self.n)
        if lib().eo_rates_normal(self.n, float(mean), float(std), int(seed), _p(up_set, C.c_double),
                                 _p(down_set, C.c_double), _p(r, C.c_double)) != 0:
            raise OracleError(lib().eo_last_error().decode())
        return r

    def initial_state(self, fixed_names=(), fixed_values=(), p=1.0) -> np.ndarray:
        idx = np.array([self.names.index(f) for f in fixed_names], np.int32)
        vals = np.array([int(bool(v)) for v in fixed_values], np.int32)
        x0 = np.zeros(1 << self.n)
        lib().eo_initial_state(self.n, len(idx), _p(idx, C.c_int32), _p(vals, C.c_int32), float(p), _p(x0, C.c_double))
        return x0

    def flip_masks(self, rates) -> np.ndarray:
        rates = np.ascontiguousarray(rates, np.float64)
        F = np.zeros(1 << self.n, np.uint32)
        lib().eo_flip_masks(self._h, _p(rates, C.c_double), _p(F, C.c_uint32))
        return F

    def table(self, rates):
        """CSC by source: indptr[N+1], rows (destinations, ascending per column), cols (sources)."""
        rates = np.ascontiguousarray(rates, np.float64)
        L = lib()
        nnz = L.eo_table(self._h, _p(rates, C.c_double), None, None, None)
        indptr = np.zeros((1 << self.n) + 1, np.int32)
        rows = np.zeros(max(nnz, 1), np.int32)
        cols = np.zeros(max(nnz, 1), np.int32)
        L.eo_table(self._h, _p(rates, C.c_double), _p(indptr, C.c_int32), _p(rows, C.c_int32), _p(cols, C.c_int32))
        return indptr, rows[:nnz], cols[:nnz]

    def analyse(self, rates) -> "Symbolic":
        return Symbolic(self, rates)


class Symbolic:
    """SCC decomposition, levels and the reordered vertices for one zero-rate pattern."""

    def __init__(self, model: Model, rates):
        L = lib()
        self.model = model
        self.rates = np.ascontiguousarray(rates, np.float64)
        h = L.eo_build(model._h, _p(self.rates, C.c_double))
        if not h:
            raise OracleError(L.eo_last_error().decode())
        self._h = h
        self.n = model.n
        self.N = 1 << model.n
        self.n_sccs = L.eo_n_sccs(h)
        self.T = L.eo_n_terminals(h)
        self.order = np.zeros(self.N, np.int32)
        self.offsets = np.zeros(self.n_sccs + 1, np.int32)
        self.levels = np.zeros(self.n_sccs, np.int32)
        self.labels = np.zeros(self.N, np.int32)
        L.eo_graph(h, _p(self.order, C.c_int32), _p(self.offsets, C.c_int32), _p(self.levels, C.c_int32),
                   _p(self.labels, C.c_int32))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.eo_free_sym(self._h)
            self._h = None

    def _r(self, rates):
        r = self.rates if rates is None else np.ascontiguousarray(rates, np.float64)
        if not np.array_equal(r == 0, self.rates == 0):
            raise OracleError("rate set has a different zero pattern than the symbolic analysis")
        return r

    def terminal_kernels(self, rates=None) -> np.ndarray:
        r = self._r(rates)
        R = np.zeros(int(self.offsets[self.T]))
        if lib().eo_terminal_kernels(self._h, _p(r, C.c_double), _p(R, C.c_double)) != 0:
            raise OracleError(lib().eo_last_error().decode())
        return R

    def absorption(self, rates=None) -> np.ndarray:
        r = self._r(rates)
        Lm = np.zeros((self.T, self.N))
        if lib().eo_absorption(self._h, _p(r, C.c_double), _p(Lm, C.c_double)) != 0:
            raise OracleError(lib().eo_last_error().decode())
        return Lm

    def terminal_mass(self, x0, rates=None) -> np.ndarray:
        r = self._r(rates)
        x0 = np.ascontiguousarray(x0, np.float64)
        y = np.zeros(self.T)
        if lib().eo_terminal_mass(self._h, _p(r, C.c_double), _p(x0, C.c_double), _p(y, C.c_double)) != 0:
            raise OracleError(lib().eo_last_error().decode())
        return y

    def solve(self, x0, rates=None, use_absorption=False):
        r = self._r(rates)
        x0 = np.ascontiguousarray(x0, np.float64)
        xi = np.zeros(self.N)
        m = np.zeros(self.n)
        if lib().eo_solve(self._h, _p(r, C.c_double), _p(x0, C.c_double), _p(xi, C.c_double), _p(m, C.c_double),
                          int(use_absorption)) != 0:
            raise OracleError(lib().eo_last_error().decode())
        return xi, m

    def solve_many(self, rates, x0, threads=None):
        """One solve per row of ``rates`` (B x 2n) with the matching row of ``x0`` (B x N)."""
        rates = np.ascontiguousarray(rates, np.float64)
        x0 = np.ascontiguousarray(x0, np.float64)
        B = rates.shape[0]
        for b in range(B):
            self._r(rates[b])
        threads = threads or os.cpu_count() or 1
        xi = np.zeros((B, self.N))
        m = np.zeros((B, self.n))
        if lib().eo_solve_many(self._h, B, _p(rates, C.c_double), _p(x0, C.c_double), _p(xi, C.c_double),
                               _p(m, C.c_double), int(threads)) != 0:
            raise OracleError(lib().eo_last_error().decode())
        return xi, m


def last_relres() -> float:
    return lib().eo_last_relres()


def iterative_blocks() -> int:
    return lib().eo_iterative_blocks()
