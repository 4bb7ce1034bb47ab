"""Test infrastructure only: float64 restatement of the learned prefilter.

The product computes these on the GPU (mnhn-tree-tools_b200/csrc/mlp_kernels.cu
and prefilter.cu); this module is the checker the tests compare it against.
The prefilter has no counterpart in the reference; its k-mer features follow
kmers.c:157-241 (the oracle's orc_kmer_counts restates them).

Network: x (L1-normalised 5-mer counts) * 32 -> Linear(1024, 512) -> GELU ->
Linear(512, 256) -> GELU -> Linear(256, 128) = embedding e.  Loss over pairs
(a, b) with exact distance d: mean over pairs of (||e_a - e_b|| - t)^2 with
t = d / (4 * max(len_a, len_b)).  GELU is the exact erf form.

With emulate_bf16 the GEMM operands are rounded to bfloat16 (round to nearest
even) where the GPU stores them in bf16 (weights, inputs, activations and the
back-propagated gradients), and everything else is float64.
"""
from __future__ import annotations

import math

import numpy as np

D0, D1, D2, D3 = 1024, 512, 256, 128
IN_SCALE = 32.0
SIZES = [("W1", (D1, D0)), ("b1", (D1,)), ("W2", (D2, D1)), ("b2", (D2,)), ("W3", (D3, D2)), ("b3", (D3,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)

_erf = np.vectorize(math.erf)


def unpack(params: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def features(counts: np.ndarray) -> np.ndarray:
    """L1-normalised rows (zero rows stay zero)."""
    c = np.asarray(counts, dtype=np.float64)
    s = c.sum(axis=1, keepdims=True)
    return np.divide(c, s, out=np.zeros_like(c), where=s > 0)


def forward(X: np.ndarray, params: np.ndarray, emulate_bf16: bool = True):
    p = unpack(params)
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    Xs = r(X * IN_SCALE)
    Z1 = Xs @ r(p["W1"]).T + p["b1"]
    A1 = r(gelu(Z1))
    Z2 = A1 @ r(p["W2"]).T + p["b2"]
    A2 = r(gelu(Z2))
    E = A2 @ r(p["W3"]).T + p["b3"]
    return dict(Xs=Xs, Z1=Z1, A1=A1, Z2=Z2, A2=A2, E=E)


def loss_grad(X: np.ndarray, a, b, dist, lens, params: np.ndarray, emulate_bf16: bool = True):
    """X: per-sequence features [n x 1024]; returns (loss, flat gradient)."""
    a = np.asarray(a)
    b = np.asarray(b)
    P = len(a)
    rows = np.empty(2 * P, dtype=np.int64)
    rows[0::2] = a
    rows[1::2] = b
    f = forward(X[rows], params, emulate_bf16)
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    p = unpack(params)
    E = f["E"]
    diff = E[0::2] - E[1::2]
    de = np.sqrt((diff ** 2).sum(axis=1))
    lens = np.asarray(lens, dtype=np.float64)
    mx = np.maximum(lens[a], lens[b])
    t = np.where(mx > 0, np.asarray(dist, dtype=np.float64) / (4.0 * np.maximum(mx, 1)), 0.0)
    res = de - t
    loss = float((res ** 2).mean())
    c = np.where(de > 1e-20, 2.0 * res / (P * np.maximum(de, 1e-300)), 0.0)
    dEa = c[:, None] * diff
    dE = np.empty_like(E)
    dE[0::2] = dEa
    dE[1::2] = -dEa
    dE = r(dE)
    g = {}
    g["W3"] = dE.T @ f["A2"]
    g["b3"] = np.zeros(D3)
    dZ2 = (dE @ r(p["W3"])) * gelu_grad(f["Z2"])
    g["b2"] = dZ2.sum(axis=0)
    dZ2 = r(dZ2)
    g["W2"] = dZ2.T @ f["A1"]
    dZ1 = (dZ2 @ r(p["W2"])) * gelu_grad(f["Z1"])
    g["b1"] = dZ1.sum(axis=0)
    dZ1 = r(dZ1)
    g["W1"] = dZ1.T @ f["Xs"]
    return loss, pack(g)
