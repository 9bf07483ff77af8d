"""CPU restatement of the learned warm start's network (test infrastructure only).

The reference has no learned component, so nothing here follows a reference file; this
module is the checker for the library's MLP kernels (``esl_mlp_*``): the same features,
the same BF16 rounding of the weights, and the forward pass and gradient of the mean
squared error in float64.  Only tests and the smoke check import it.

Feature row of (state v, rate set k), 77 entries:
    [0, 20)   node bits of v as +-1 (0 past n)
    [20]      log of v's outgoing rate sum under k
    [21, 37)  +-1 for "v reaches terminal SCC t" (t < 16; 0 past T)
    [37, 77)  log of the 2n rates of k (0 past 2n and for a zero rate)
Parameters (flat): W1[128][77], b1[128], W2[128][128], b2[128], w3[128], b3.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 77, 128
SIZES = [("W1", (N_H, N_IN)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)), ("w3", (N_H,)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)
WEIGHTS = ("W1", "W2", "w3")


def bf16_round(x) -> np.ndarray:
    """Round float32 values to the nearest BF16 value (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(params):
    p = np.asarray(params)
    out, o = {}, 0
    for name, shape in SIZES:
        c = int(np.prod(shape))
        out[name] = p[o:o + c].reshape(shape)
        o += c
    return out


def pack(d) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SIZES])


def reach_bits(sym, F) -> np.ndarray:
    """Bit t of reach[v]: state v reaches terminal SCC t (t < 16).  Terminal SCCs reach
    themselves; a transient SCC reaches the union of what its out-of-SCC successors reach
    (successor SCCs come later in the order, which lists terminals first and then the
    transient SCCs by decreasing level)."""
    order, off, labels, T = sym.order, sym.offsets, sym.labels, sym.T
    N = order.size
    reach = np.zeros(N, np.uint32)
    for t in range(min(T, 16)):
        reach[order[off[t]:off[t + 1]]] = np.uint32(1 << t)
    n = int(N).bit_length() - 1
    for c in range(sym.n_sccs - 1, T - 1, -1):
        vs = order[off[c]:off[c + 1]]
        r = np.uint32(0)
        for i in range(n):
            out = (F[vs] >> i) & 1
            us = vs[out == 1] ^ (1 << i)
            ext = us[labels[us] != labels[vs[out == 1]]]
            if ext.size:
                r |= np.bitwise_or.reduce(reach[ext])
        reach[vs] = r
    return reach


def features(n: int, T: int, F, reach, rates, ks, vs) -> np.ndarray:
    rates = np.asarray(rates, np.float64).reshape(-1, 2 * n)
    ks = np.asarray(ks, np.int64)
    vs = np.asarray(vs, np.int64)
    S = ks.size
    X = np.zeros((S, N_IN))
    for i in range(n):
        X[:, i] = np.where((vs >> i) & 1, 1.0, -1.0)
    for s in range(S):
        v, r = int(vs[s]), rates[ks[s]]
        f = int(F[v])
        q = sum(r[2 * i + ((v >> i) & 1)] for i in range(n) if (f >> i) & 1)
        X[s, 20] = np.log(q) if q > 0 else 0.0
    for t in range(min(T, 16)):
        X[:, 21 + t] = np.where((np.asarray(reach)[vs] >> t) & 1, 1.0, -1.0)
    lr = np.where(rates > 0, np.log(np.where(rates > 0, rates, 1.0)), 0.0)
    X[:, 37:37 + 2 * n] = lr[ks]
    return X


def quantized(params, rnd: bool = True) -> dict:
    """Parameters as float64 arrays, weights rounded to BF16 as the kernels use them
    (rnd=False keeps them exact, for finite-difference checks of the gradient)."""
    if not rnd:
        return {k: np.asarray(v, np.float64) for k, v in unpack(np.asarray(params, np.float64)).items()}
    d = {k: np.asarray(v, np.float64) for k, v in unpack(np.asarray(params, np.float32)).items()}
    for w in WEIGHTS:
        d[w] = bf16_round(d[w].astype(np.float32)).astype(np.float64)
    return d


def forward(params, X, rnd: bool = True):
    d = quantized(params, rnd)
    z1 = X @ d["W1"].T + d["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ d["W2"].T + d["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ d["w3"] + d["b3"][0]
    return y, (d, h1, h2)


def loss_grad(params, X, t, rnd: bool = True):
    """Mean squared error over the samples and its gradient with respect to the
    (BF16-rounded) weights and the biases, flat in the parameter layout."""
    y, (d, h1, h2) = forward(params, X, rnd)
    S = X.shape[0]
    r = y - np.asarray(t, np.float64)
    loss = float(np.sum(r * r) / S)
    dy = 2.0 * r / S
    g = {"w3": h2.T @ dy, "b3": np.array([dy.sum()])}
    dz2 = np.outer(dy, d["w3"]) * (h2 > 0)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ d["W2"]) * (h1 > 0)
    g["W1"] = dz1.T @ X
    g["b1"] = dz1.sum(0)
    return loss, pack(g)
