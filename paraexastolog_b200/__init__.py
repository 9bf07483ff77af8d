"""ExaStoLog stationary distributions on B200: Python host binding of libesl_b200.so.

The library is the product: a C ABI (``include/esl_b200.h``) over hand-written
sm_100a CUDA kernels.  This module binds it with ctypes; torch is used only for
device memory and streams.  Importing it never falls back to another
implementation: if the library is missing, ``lib()`` raises.

Mirror of the reference's C++ API (``cuda/src/*.h``):
    model_builder().construct_model(path)  -> Model.load(path)
    transition_rates(model).generate_*      -> Model.rates_uniform / rates_normal
    initial_state(nodes, fixed, values, p)  -> Model.initial_state
    transition_table(...).construct_table   -> table()
    transition_graph(...).reorganize_vertices -> Net.build / Net.export
    solver(...).solve()                     -> solve(), solve_batch()
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libesl_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "esl_b200.h")

ESL_OK = 0
METHOD_FP64, METHOD_MIXED, METHOD_DIRECT = 0, 1, 2
ERRORS = {-1: "INVALID", -2: "PARSE", -3: "CUDA", -4: "NOMEM", -5: "TIMEOUT", -6: "NOT_CONVERGED", -7: "TOO_LARGE"}

_lib = None


class EslError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class SolveOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("tol", C.c_double), ("max_iters", C.c_int), ("max_refine", C.c_int),
                ("d_warm", C.c_void_p), ("d_occupation", C.c_void_p)]


class Report(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("relres", C.c_double), ("converged", C.c_int),
                ("fallback_systems", C.c_int), ("dense_lu_systems", C.c_int),
                ("absorption_by_sweep", C.c_int)]


class Job(C.Structure):
    _fields_ = [("net", C.c_void_p), ("B", C.c_int), ("d_rates", C.c_void_p), ("R", C.c_int), ("d_x0", C.c_void_p),
                ("d_x_inf", C.c_void_p), ("d_marginals", C.c_void_p), ("report", Report), ("status", C.c_int)]


def header_functions() -> list:
    """Names of the functions declared in include/esl_b200.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(esl_\w+)\s*\(", text, re.M)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m paraexastolog_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, cp, i32, u32, f64 = C.c_void_p, C.c_char_p, C.c_int32, C.c_uint32, C.c_double
    P = C.POINTER
    L.esl_last_error.restype = cp
    L.esl_ctx_create.argtypes = [C.c_int, vp, P(vp)]
    L.esl_ctx_destroy.argtypes = [vp]
    L.esl_ctx_synchronize.argtypes = [vp]
    L.esl_ctx_set_profiling.argtypes = [vp, C.c_int]
    L.esl_ctx_set_budgets.argtypes = [vp, C.c_int64, C.c_int, C.c_int]
    L.esl_launch_count.argtypes = [P(C.c_uint64)]
    L.esl_ctx_profile.argtypes = [vp, P(C.c_double), P(C.c_double), P(C.c_int)]
    L.esl_ctx_profile_records.argtypes = [vp, C.c_int, vp, vp, P(C.c_int)]
    L.esl_ctx_profile_entry.argtypes = [vp, C.c_int, P(cp), P(C.c_double), P(C.c_double)]
    L.esl_model_load.argtypes = [cp, P(vp)]
    L.esl_model_parse.argtypes = [cp, P(vp)]
    L.esl_model_free.argtypes = [vp]
    L.esl_model_nodes.argtypes = [vp, P(C.c_int)]
    L.esl_model_node_name.restype = cp
    L.esl_model_node_name.argtypes = [vp, C.c_int]
    L.esl_model_node_index.argtypes = [vp, cp, P(C.c_int)]
    L.esl_model_clauses.argtypes = [vp, vp, vp, vp, C.c_int, P(C.c_int)]
    L.esl_rates_uniform.argtypes = [vp, C.c_int, vp, vp, C.c_int, vp, vp, vp]
    L.esl_rates_normal.argtypes = [vp, f64, f64, C.c_uint64, C.c_int, vp, vp, C.c_int, vp, vp, vp]
    L.esl_initial_state.argtypes = [vp, vp, C.c_int, vp, vp, f64, vp]
    L.esl_table_nnz.argtypes = [vp, vp, vp, P(C.c_int64)]
    L.esl_table_build.argtypes = [vp, vp, vp, vp, vp, vp]
    L.esl_flip_masks.argtypes = [vp, vp, vp, vp, vp]
    L.esl_table_build64.argtypes = [vp, vp, vp, vp, vp, vp]
    L.esl_trim_cache.argtypes = []
    L.esl_table_build_static.argtypes = [vp, vp, vp, vp, vp, vp, C.c_int64, P(C.c_int64)]
    L.esl_net_build.argtypes = [vp, vp, vp, P(vp)]
    L.esl_net_from_csc.argtypes = [vp, C.c_int, vp, vp, P(vp)]
    L.esl_net_free.argtypes = [vp]
    L.esl_net_info.argtypes = [vp, P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_int)]
    L.esl_net_export.argtypes = [vp, vp, vp, vp, vp, vp]
    L.esl_net_compatible.argtypes = [vp, vp, P(C.c_int)]
    L.esl_net_plan_checksums.argtypes = [vp, vp, C.c_int, vp, C.c_int]
    L.esl_net_autotune.argtypes = [vp, vp, C.c_int, vp, C.c_int, vp, P(SolveOpts), P(C.c_int), P(C.c_int),
                                   P(C.c_double)]
    L.esl_solve.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, P(SolveOpts), P(Report)]
    L.esl_solve_batch.argtypes = [vp, vp, C.c_int, vp, C.c_int, vp, vp, vp, P(SolveOpts), P(Report)]
    L.esl_solve_host.argtypes = [vp, vp, C.c_int, vp, C.c_int, vp, vp, vp, P(SolveOpts), P(Report)]
    L.esl_solve_many.argtypes = [vp, C.c_int, P(Job), C.c_int, P(SolveOpts)]
    f32 = C.c_float
    L.esl_mlp_create.argtypes = [vp, vp, C.c_uint64, P(vp)]
    L.esl_mlp_free.argtypes = [vp]
    L.esl_mlp_info.argtypes = [vp, P(C.c_int), P(f32), P(f32)]
    L.esl_mlp_targets.argtypes = [vp, vp]
    L.esl_mlp_reach.argtypes = [vp, vp]
    L.esl_mlp_get_params.argtypes = [vp, vp]
    L.esl_mlp_set_params.argtypes = [vp, vp, f32, f32]
    L.esl_mlp_features.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.esl_mlp_loss_grad.argtypes = [vp, C.c_int, vp, vp, vp, vp, P(f32), vp]
    L.esl_mlp_forward.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.esl_mlp_train.argtypes = [vp, C.c_int, vp, vp, C.c_int, C.c_int, f32, P(f32)]
    L.esl_mlp_predict.argtypes = [vp, C.c_int, vp, vp]
    _lib = L
    return L


def trim_cache():
    """Return the library's cached device blocks to the driver."""
    check(lib().esl_trim_cache())


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    c = C.c_uint64()
    check(lib().esl_launch_count(C.byref(c)))
    return c.value


def check(code: int):
    if code != ESL_OK:
        raise EslError(code, lib().esl_last_error().decode(errors="replace"))


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    if t.numel() == 0:  # an empty view still points at its (non-empty) buffer
        return t.untyped_storage().data_ptr()
    return t.data_ptr()


def _strs(names: Sequence[str]):
    arr = (C.c_char_p * max(len(names), 1))(*[s.encode() for s in names])
    return arr


def _torch():
    import torch
    return torch


class Context:
    """Device, stream and scratch of the library (``cu_context`` in the reference)."""

    def __init__(self, device: int = 0, stream=None):
        torch = _torch()
        self.device = device
        torch.cuda.set_device(device)
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        # torch's default stream has handle 0, which the C ABI reads as "make a stream of
        # your own"; pass cudaStreamLegacy (0x1) instead so that library work stays ordered
        # with torch's work on that stream
        handle = self.stream.cuda_stream or 0x1
        h = C.c_void_p()
        check(lib().esl_ctx_create(device, C.c_void_p(handle), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().esl_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().esl_ctx_synchronize(self._h))

    def set_budgets(self, graph_sweeps: int = 0, block_iters: int = 0, dense_max: int = 0):
        """Budgets of the fallback paths (0 keeps a default): sweeps per graph fixpoint
        loop, Krylov iterations of the block forward solve, largest dense-LU block."""
        check(lib().esl_ctx_set_budgets(self._h, int(graph_sweeps), int(block_iters), int(dense_max)))

    def set_profiling(self, on: bool):
        """Record CUDA events around each reduced-operator application of the solver."""
        check(lib().esl_ctx_set_profiling(self._h, int(bool(on))))

    def profile(self):
        """(summed device ms, algorithmic bytes, launches) since profiling was switched on."""
        ms, by, n = C.c_double(), C.c_double(), C.c_int()
        check(lib().esl_ctx_profile(self._h, C.byref(ms), C.byref(by), C.byref(n)))
        return ms.value, by.value, n.value

    def profile_entries(self):
        """Every record since profiling was switched on: (kernel class, device ms,
        algorithmic bytes) tuples in launch order."""
        n = C.c_int()
        check(lib().esl_ctx_profile_records(self._h, 0, None, None, C.byref(n)))
        out = []
        name, ms, by = C.c_char_p(), C.c_double(), C.c_double()
        for i in range(n.value):
            check(lib().esl_ctx_profile_entry(self._h, i, C.byref(name), C.byref(ms), C.byref(by)))
            out.append((name.value.decode(), ms.value, by.value))
        return out

    def profile_records(self):
        """Per record: (device ms, algorithmic bytes) arrays."""
        n = C.c_int()
        check(lib().esl_ctx_profile_records(self._h, 0, None, None, C.byref(n)))
        ms = np.zeros(n.value)
        by = np.zeros(n.value)
        if n.value:
            check(lib().esl_ctx_profile_records(self._h, n.value, _ptr(ms), _ptr(by), C.byref(n)))
        return ms, by


class Model:
    """Parsed bnet model (``model_t``): node names and DNF clauses."""

    def __init__(self, handle):
        self._h = handle
        n = C.c_int()
        check(lib().esl_model_nodes(handle, C.byref(n)))
        self.n = n.value
        self.names = [lib().esl_model_node_name(handle, i).decode() for i in range(self.n)]

    @classmethod
    def parse(cls, text: str) -> "Model":
        h = C.c_void_p()
        check(lib().esl_model_parse(text.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path: str) -> "Model":
        h = C.c_void_p()
        check(lib().esl_model_load(path.encode(), C.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.esl_model_free(self._h)
            self._h = None

    def clauses(self):
        total = C.c_int()
        check(lib().esl_model_clauses(self._h, None, None, None, 0, C.byref(total)))
        off = np.zeros(self.n + 1, np.int32)
        pos = np.zeros(max(total.value, 1), np.uint32)
        neg = np.zeros(max(total.value, 1), np.uint32)
        check(lib().esl_model_clauses(self._h, _ptr(off), _ptr(pos), _ptr(neg), total.value, C.byref(total)))
        return off, pos[: total.value], neg[: total.value]

    def rates_uniform(self, up: Optional[Dict[str, float]] = None, down: Optional[Dict[str, float]] = None) -> np.ndarray:
        up, down = up or {}, down or {}
        out = np.zeros(2 * self.n)
        uv = np.array(list(up.values()), np.float64)
        dv = np.array(list(down.values()), np.float64)
        check(lib().esl_rates_uniform(self._h, len(up), _strs(list(up)), _ptr(uv), len(down), _strs(list(down)),
                                      _ptr(dv), _ptr(out)))
        return out

    def rates_normal(self, mean: float, std: float, seed: int = 0, up=None, down=None) -> np.ndarray:
        up, down = up or {}, down or {}
        out = np.zeros(2 * self.n)
        uv = np.array(list(up.values()), np.float64)
        dv = np.array(list(down.values()), np.float64)
        check(lib().esl_rates_normal(self._h, mean, std, seed, len(up), _strs(list(up)), _ptr(uv), len(down),
                                     _strs(list(down)), _ptr(dv), _ptr(out)))
        return out

    def initial_state(self, ctx: Context, fixed: Sequence[str] = (), values: Sequence[int] = (), p: float = 1.0):
        torch = _torch()
        x0 = torch.empty(1 << self.n, dtype=torch.float64, device=f"cuda:{ctx.device}")
        vals = np.array([int(bool(v)) for v in values], np.int32)
        check(lib().esl_initial_state(ctx._h, self._h, len(fixed), _strs(list(fixed)), _ptr(vals), float(p), _ptr(x0)))
        ctx.synchronize()
        return x0


def table(ctx: Context, model: Model, rates: np.ndarray, with_cols: bool = True):
    """CSC transition table (indptr, rows, cols) as int32 device tensors."""
    torch = _torch()
    rates = np.ascontiguousarray(rates, np.float64)
    nnz = C.c_int64()
    check(lib().esl_table_nnz(ctx._h, model._h, _ptr(rates), C.byref(nnz)))
    dev = f"cuda:{ctx.device}"
    indptr = torch.empty((1 << model.n) + 1, dtype=torch.int32, device=dev)
    rows = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
    cols = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev) if with_cols else None
    check(lib().esl_table_build(ctx._h, model._h, _ptr(rates), _ptr(indptr), _ptr(rows), _ptr(cols)))
    return indptr, rows[: nnz.value], (cols[: nnz.value] if with_cols else None)


def table64(ctx: Context, model: Model, rates: np.ndarray, with_cols: bool = False):
    """CSC transition table with int64 column pointers (tables of >= 2^31 edges):
    (indptr int64, rows int32, cols int32 or None) device tensors."""
    torch = _torch()
    rates = np.ascontiguousarray(rates, np.float64)
    nnz = C.c_int64()
    check(lib().esl_table_nnz(ctx._h, model._h, _ptr(rates), C.byref(nnz)))
    dev = f"cuda:{ctx.device}"
    indptr = torch.empty((1 << model.n) + 1, dtype=torch.int64, device=dev)
    rows = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
    cols = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev) if with_cols else None
    check(lib().esl_table_build64(ctx._h, model._h, _ptr(rates), _ptr(indptr), _ptr(rows), _ptr(cols)))
    return indptr, rows[: nnz.value], (cols[: nnz.value] if with_cols else None)


def flip_masks(ctx: Context, model: Model, rates: np.ndarray):
    torch = _torch()
    rates = np.ascontiguousarray(rates, np.float64)
    dev = f"cuda:{ctx.device}"
    F = torch.empty(1 << model.n, dtype=torch.int32, device=dev)
    G = torch.empty(1 << model.n, dtype=torch.int32, device=dev)
    check(lib().esl_flip_masks(ctx._h, model._h, _ptr(rates), _ptr(F), _ptr(G)))
    return F, G


class Net:
    """Device symbolic data of one (model, zero-rate pattern): masks, SCCs, order."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._h = handle
        n, s, t, ts = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().esl_net_info(handle, C.byref(n), C.byref(s), C.byref(t), C.byref(ts)))
        self.n, self.n_sccs, self.T, self.terminal_states = n.value, s.value, t.value, ts.value
        self.N = 1 << self.n

    @classmethod
    def build(cls, ctx: Context, model: Model, rates: np.ndarray) -> "Net":
        rates = np.ascontiguousarray(rates, np.float64)
        h = C.c_void_p()
        check(lib().esl_net_build(ctx._h, model._h, _ptr(rates), C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_csc(cls, ctx: Context, n: int, indptr, rows) -> "Net":
        h = C.c_void_p()
        check(lib().esl_net_from_csc(ctx._h, n, _ptr(indptr), _ptr(rows), C.byref(h)))
        return cls(ctx, h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.esl_net_free(self._h)
            self._h = None

    def export(self):
        torch = _torch()
        dev = f"cuda:{self.ctx.device}"
        order = torch.empty(self.N, dtype=torch.int32, device=dev)
        offsets = torch.empty(self.n_sccs + 1, dtype=torch.int32, device=dev)
        levels = torch.empty(max(self.n_sccs, 1), dtype=torch.int32, device=dev)
        labels = torch.empty(self.N, dtype=torch.int32, device=dev)
        check(lib().esl_net_export(self.ctx._h, self._h, _ptr(order), _ptr(offsets), _ptr(levels), _ptr(labels)))
        return order, offsets, levels[: self.n_sccs], labels

    def autotune(self, rates, x0, method: int = METHOD_DIRECT, tol: float = 1e-10) -> dict:
        """Time the batch solve under a few level-sweep tilings and keep the fastest."""
        torch = _torch()
        dev = f"cuda:{self.ctx.device}"
        r = torch.as_tensor(rates, dtype=torch.float64, device=dev).contiguous()
        x = torch.as_tensor(x0, dtype=torch.float64, device=dev).contiguous()
        r = r[None] if r.dim() == 1 else r
        x = x[None] if x.dim() == 1 else x
        mb, s2, ms = C.c_int(), C.c_int(), C.c_double()
        o = _opts(method, tol, 0, 0)
        check(lib().esl_net_autotune(self.ctx._h, self._h, r.shape[0], _ptr(r), x.shape[0], _ptr(x), C.byref(o),
                                     C.byref(mb), C.byref(s2), C.byref(ms)))
        return {"tile_mb": mb.value, "two_systems_per_thread": bool(s2.value), "ms": ms.value}

    def plan_checksums(self, host_builder: bool = False) -> np.ndarray:
        """Checksums of the 12 parts of the level-sweep plan, built afresh on the device
        or with the host reference builder (test hook)."""
        out = np.zeros(12, np.uint64)
        check(lib().esl_net_plan_checksums(self.ctx._h, self._h, int(bool(host_builder)), _ptr(out), 12))
        return out

    def compatible(self, rates: np.ndarray) -> bool:
        rates = np.ascontiguousarray(rates, np.float64)
        ok = C.c_int()
        check(lib().esl_net_compatible(self._h, _ptr(rates), C.byref(ok)))
        return bool(ok.value)


MLP_PARAMS = 26625


class Mlp:
    """Learned warm start of one network's transient solve (``esl_mlp_*``): a 3-layer
    MLP (77 -> 128 -> 128 -> 1) predicting the log occupation of the states whose warm
    start the level sweep's grid-wide Krylov groups read.  Keeps ``net`` alive."""

    def __init__(self, ctx: Context, net: Net, seed: int = 0):
        self.ctx, self.net = ctx, net
        h = C.c_void_p()
        check(lib().esl_mlp_create(ctx._h, net._h, seed, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.esl_mlp_free(self._h)
            self._h = None

    def info(self):
        nt, mu, sg = C.c_int(), C.c_float(), C.c_float()
        check(lib().esl_mlp_info(self._h, C.byref(nt), C.byref(mu), C.byref(sg)))
        return nt.value, mu.value, sg.value

    @property
    def n_targets(self) -> int:
        return self.info()[0]

    def _dev(self):
        return f"cuda:{self.ctx.device}"

    def targets(self):
        torch = _torch()
        t = torch.empty(max(self.n_targets, 1), dtype=torch.int32, device=self._dev())
        check(lib().esl_mlp_targets(self._h, _ptr(t)))
        self.ctx.synchronize()
        return t[: self.n_targets]

    def reach(self):
        torch = _torch()
        t = torch.empty(self.net.N, dtype=torch.int32, device=self._dev())
        check(lib().esl_mlp_reach(self._h, _ptr(t)))
        self.ctx.synchronize()
        return t

    def get_params(self) -> np.ndarray:
        p = np.zeros(MLP_PARAMS, np.float32)
        check(lib().esl_mlp_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, params: np.ndarray, mu: float, sigma: float):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == MLP_PARAMS
        check(lib().esl_mlp_set_params(self._h, _ptr(p), float(mu), float(sigma)))

    def _samples(self, rates, ks, vs):
        """Device copies of a sample list.  The library reads the rate-set and state
        indices on the device without bounds checks, so they are checked here."""
        torch = _torch()
        dev = self._dev()
        rates = torch.as_tensor(rates, dtype=torch.float64, device=dev).contiguous()
        ks = torch.as_tensor(ks, dtype=torch.int32, device=dev).contiguous()
        vs = torch.as_tensor(vs, dtype=torch.int32, device=dev).contiguous()
        if ks.numel() != vs.numel():
            raise ValueError(f"{ks.numel()} rate-set indices but {vs.numel()} states")
        sets = rates.numel() // (2 * self.net.n)
        if ks.numel():
            if int(ks.min()) < 0 or int(ks.max()) >= sets:
                raise ValueError(f"rate-set index outside [0, {sets})")
            if int(vs.min()) < 0 or int(vs.max()) >= self.net.N:
                raise ValueError(f"state outside [0, {self.net.N})")
        return rates, ks, vs

    def features(self, rates, ks, vs):
        torch = _torch()
        rates, ks, vs = self._samples(rates, ks, vs)
        x = torch.empty((ks.numel(), 80), dtype=torch.float32, device=self._dev())
        check(lib().esl_mlp_features(self._h, ks.numel(), _ptr(rates), _ptr(ks), _ptr(vs), _ptr(x)))
        self.ctx.synchronize()
        return x

    def loss_grad(self, rates, ks, vs, targets, grad: bool = True):
        torch = _torch()
        rates, ks, vs = self._samples(rates, ks, vs)
        t = torch.as_tensor(targets, dtype=torch.float32, device=self._dev()).contiguous()
        loss = C.c_float()
        g = np.zeros(MLP_PARAMS, np.float32) if grad else None
        check(lib().esl_mlp_loss_grad(self._h, ks.numel(), _ptr(rates), _ptr(ks), _ptr(vs), _ptr(t),
                                      C.byref(loss), _ptr(g)))
        return loss.value, g

    def forward(self, rates, ks, vs):
        torch = _torch()
        rates, ks, vs = self._samples(rates, ks, vs)
        y = torch.empty(ks.numel(), dtype=torch.float32, device=self._dev())
        check(lib().esl_mlp_forward(self._h, ks.numel(), _ptr(rates), _ptr(ks), _ptr(vs), _ptr(y)))
        self.ctx.synchronize()
        return y

    def train(self, rates, occupation, steps: int = 1000, batch: int = 16384, lr: float = 1e-3) -> float:
        """Adam steps on random (rate set, target state) pairs; ``occupation`` is the
        B x N output of solve_batch(..., occupation=...) for the B rate sets."""
        torch = _torch()
        rates = torch.as_tensor(rates, dtype=torch.float64, device=self._dev()).contiguous()
        loss = C.c_float()
        check(lib().esl_mlp_train(self._h, rates.shape[0], _ptr(rates), _ptr(occupation), steps, batch, lr,
                                  C.byref(loss)))
        return loss.value

    def predict(self, rates, out=None):
        """Warm start (B x N, float64, device): predicted occupation on the targets, 0 elsewhere."""
        torch = _torch()
        rates = torch.as_tensor(rates, dtype=torch.float64, device=self._dev()).contiguous()
        if rates.dim() == 1:
            rates = rates[None]
        B = rates.shape[0]
        w = out if out is not None else torch.empty((B, self.net.N), dtype=torch.float64, device=self._dev())
        check(lib().esl_mlp_predict(self._h, B, _ptr(rates), _ptr(w)))
        return w


@dataclass
class SolveResult:
    x_inf: object
    marginals: object
    R: object = None
    L: object = None
    report: Optional[Report] = None
    status: int = 0


def _check_batch(n: int, rates, x0, warm=None, occupation=None, out=None, device=None):
    """(B, R) of a batch of B rate sets (B x 2n) and R initial distributions (R x 2^n),
    or ValueError.  The library reads and writes every buffer by the sizes the network
    implies, so a short or mistyped one would be read or written past its end; the
    device buffers must also live on the context's device (``device``, if given)."""
    N = 1 << n
    if rates.dim() != 2 or rates.shape[1] != 2 * n or rates.shape[0] < 1:
        raise ValueError(f"rates must be B x {2 * n} (B >= 1), got {tuple(rates.shape)}")
    if x0.dim() != 2 or x0.shape[1] != N or x0.shape[0] < 1:
        raise ValueError(f"x0 must be R x {N} (R >= 1), got {tuple(x0.shape)}")
    B, R = rates.shape[0], x0.shape[0]
    for name, t, shape in (("warm", warm, None), ("occupation", occupation, None), ("out", out, (B, R, N))):
        if t is None:
            continue
        import torch
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float64 tensor")
        if shape is not None and tuple(t.shape) != shape:
            raise ValueError(f"{name} must be {shape}, got {tuple(t.shape)}")
        if t.numel() != B * R * N:
            raise ValueError(f"{name} must hold {B} x {R} x {N} values, got {t.numel()}")
        if device is not None and (not t.is_cuda or t.device.index != device):
            raise ValueError(f"{name} must be on cuda:{device}")
    return B, R


def _opts(method: int, tol: float, max_iters: int, max_refine: int, warm=None, occupation=None) -> SolveOpts:
    return SolveOpts(method, tol, max_iters, max_refine, _ptr(warm), _ptr(occupation))


def solve(ctx: Context, net: Net, rates, x0, want_R: bool = False, want_L: bool = False,
          method: int = METHOD_FP64, tol: float = 1e-10, max_iters: int = 0, max_refine: int = 0) -> SolveResult:
    """One (rate set, x0): x_inf, marginals and optionally R (terminal kernels in
    reordered position) and the dense absorption matrix L (T x N)."""
    torch = _torch()
    dev = f"cuda:{ctx.device}"
    rates = torch.as_tensor(np.ascontiguousarray(rates, np.float64) if isinstance(rates, np.ndarray) else rates,
                            dtype=torch.float64, device=dev).contiguous()
    x0 = torch.as_tensor(x0, dtype=torch.float64, device=dev).contiguous()
    _check_batch(net.n, rates.reshape(1, -1), x0.reshape(1, -1))
    xi = torch.empty(net.N, dtype=torch.float64, device=dev)
    mg = torch.empty(net.n, dtype=torch.float64, device=dev)
    Rv = torch.empty(max(net.terminal_states, 1), dtype=torch.float64, device=dev) if want_R else None
    Lm = torch.empty((net.T, net.N), dtype=torch.float64, device=dev) if want_L else None
    rep = Report()
    o = _opts(method, tol, max_iters, max_refine)
    torch.cuda.current_stream(ctx.device).synchronize()
    check(lib().esl_solve(ctx._h, net._h, _ptr(rates), _ptr(x0), _ptr(xi), _ptr(mg), _ptr(Rv), _ptr(Lm),
                          C.byref(o), C.byref(rep)))
    return SolveResult(xi, mg, Rv[: net.terminal_states] if want_R else None, Lm, rep)


def solve_batch(ctx: Context, net: Net, rates, x0, method: int = METHOD_FP64, tol: float = 1e-10,
                max_iters: int = 0, max_refine: int = 0, warm=None, out=None, marginals: bool = True,
                occupation=None) -> SolveResult:
    """B rate sets (B x 2n) x R initial distributions (R x N) -> x_inf (B x R x N).
    ``warm``: optional (B*R) x N device warm start of the occupation; ``occupation``:
    optional (B*R) x N device output of the expected occupation of transient states."""
    torch = _torch()
    dev = f"cuda:{ctx.device}"
    rates = torch.as_tensor(rates, dtype=torch.float64, device=dev).contiguous()
    x0 = torch.as_tensor(x0, dtype=torch.float64, device=dev).contiguous()
    if rates.dim() == 1:
        rates = rates[None]
    if x0.dim() == 1:
        x0 = x0[None]
    B, R = _check_batch(net.n, rates, x0, warm, occupation, out, ctx.device)
    xi = out if out is not None else torch.empty((B, R, net.N), dtype=torch.float64, device=dev)
    mg = torch.empty((B, R, net.n), dtype=torch.float64, device=dev) if marginals else None
    rep = Report()
    o = _opts(method, tol, max_iters, max_refine, warm, occupation)
    check(lib().esl_solve_batch(ctx._h, net._h, B, _ptr(rates), R, _ptr(x0), _ptr(xi), _ptr(mg), C.byref(o),
                                C.byref(rep)))
    return SolveResult(xi, mg, report=rep)


def solve_many(ctxs: Sequence[Context], jobs, method: int = METHOD_DIRECT, tol: float = 1e-10,
               max_iters: int = 0, max_refine: int = 0, raise_on_error: bool = True):
    """Many (net, rates B x 2n, x0 R x N) jobs in one call, run concurrently over the
    contexts (give each its own stream); returns one SolveResult per job (with its
    status; the first failure raises unless raise_on_error is False)."""
    torch = _torch()
    keep, arr = [], (Job * max(1, len(jobs)))()
    results = []
    for i, (net, rates, x0) in enumerate(jobs):
        dev = f"cuda:{net.ctx.device}"
        r = torch.as_tensor(rates, dtype=torch.float64, device=dev).contiguous()
        x = torch.as_tensor(x0, dtype=torch.float64, device=dev).contiguous()
        r = r[None] if r.dim() == 1 else r
        x = x[None] if x.dim() == 1 else x
        B, R = _check_batch(net.n, r, x)
        xi = torch.empty((B, R, net.N), dtype=torch.float64, device=dev)
        mg = torch.empty((B, R, net.n), dtype=torch.float64, device=dev)
        keep += [r, x]
        arr[i] = Job(net._h.value if hasattr(net._h, "value") else net._h, B, _ptr(r), R, _ptr(x), _ptr(xi), _ptr(mg),
                     Report(), 0)
        results.append(SolveResult(xi, mg))
    handles = (C.c_void_p * len(ctxs))(*[c._h.value if hasattr(c._h, "value") else c._h for c in ctxs])
    torch.cuda.synchronize()
    o = _opts(method, tol, max_iters, max_refine)
    rc = lib().esl_solve_many(C.cast(handles, C.c_void_p), len(ctxs), arr, len(jobs), C.byref(o))
    for i, res in enumerate(results):
        res.report = arr[i].report
        res.status = arr[i].status
    if raise_on_error:
        check(rc)
    return results


def solve_host(ctx: Context, model: Model, rates: np.ndarray, x0: np.ndarray, method: int = METHOD_FP64,
               tol: float = 1e-10):
    """Host arrays in, host arrays out (builds its own symbolic data)."""
    rates = np.ascontiguousarray(np.atleast_2d(rates), np.float64)
    x0 = np.ascontiguousarray(np.atleast_2d(x0), np.float64)
    torch = _torch()
    B, R = _check_batch(model.n, torch.from_numpy(rates), torch.from_numpy(x0))
    N = 1 << model.n
    xi = np.zeros((B, R, N))
    mg = np.zeros((B, R, model.n))
    rep = Report()
    o = _opts(method, tol, 0, 0)
    check(lib().esl_solve_host(ctx._h, model._h, B, _ptr(rates), R, _ptr(x0), _ptr(xi), _ptr(mg), C.byref(o),
                               C.byref(rep)))
    return xi, mg, rep
