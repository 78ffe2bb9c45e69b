"""CPU oracle of the autotuner's MLP (TEST INFRASTRUCTURE ONLY).

FP64 numpy restatement of mgxbench_b200/csrc/mlp.cu: the same parameter layout
(W1[64][6] | b1[64] | W2[64][64] | b2[64] | W3[2][64] | b3[2]), tanh hidden layers, loss
sum_o w_o (out_o - y_o)^2 / batch.  Gradients come from central finite differences, so the
GPU's hand-written backward kernel is checked against the definition of the derivative, not
against a second hand-written backward pass.
"""
from __future__ import annotations

import numpy as np

NI, NH, NO = 6, 64, 2
SIZES = [("W1", NH * NI), ("b1", NH), ("W2", NH * NH), ("b2", NH), ("W3", NO * NH), ("b3", NO)]
NPARAM = sum(s for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, size in SIZES:
        out[name] = p[o:o + size]
        o += size
    out["W1"] = out["W1"].reshape(NH, NI)
    out["W2"] = out["W2"].reshape(NH, NH)
    out["W3"] = out["W3"].reshape(NO, NH)
    return out


def forward(p, X):
    q = unpack(np.asarray(p, np.float64))
    h1 = np.tanh(X @ q["W1"].T + q["b1"])
    h2 = np.tanh(h1 @ q["W2"].T + q["b2"])
    return h2 @ q["W3"].T + q["b3"]


def loss(p, X, Y, w):
    d = forward(p, X) - Y
    return float(np.sum(w * d * d) / X.shape[0])


def fd_gradient(p, X, Y, w, h=1e-6, idx=None):
    """Central differences of `loss` with respect to the parameters listed in idx (all if None)."""
    p = np.asarray(p, np.float64).copy()
    idx = range(p.size) if idx is None else idx
    g = {}
    for i in idx:
        old = p[i]
        p[i] = old + h
        lp = loss(p, X, Y, w)
        p[i] = old - h
        lm = loss(p, X, Y, w)
        p[i] = old
        g[i] = (lp - lm) / (2 * h)
    return g
