"""CPU oracle of the warm-start MLP (test infrastructure only).

The MLP has no counterpart in the reference; this is a numpy restatement of
the network the CUDA kernels in tlfea_b200/csrc/mlp.cu implement:
dims[0] -> ... -> dims[L], exact-erf GELU between layers, mean-squared-error
loss, AdamW.  With ``bf16=True`` every operand of a matrix product is rounded to
BF16 (round to nearest even) exactly where the GPU rounds it -- layer inputs,
weights, output gradients -- and products accumulate in float64, so the only
remaining differences from the GPU are FP32 accumulation order and the GPU's
FP32 GELU.  With ``bf16=False`` it is the plain float64 network, whose analytic
gradient the CPU tests pin against central finite differences.

Only tests/, smoke() and bench.py's CPU legs use this module.
"""
from __future__ import annotations

import math

import numpy as np

_ERF = np.vectorize(math.erf)


def bf16_round(a) -> np.ndarray:
    """float -> nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _ERF(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _ERF(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unflatten(flat, dims):
    """Flat layout of the C ABI: per layer W [dims[l+1] x dims[l]] row-major, then b."""
    Ws, bs, o = [], [], 0
    for l in range(len(dims) - 1):
        n, k = dims[l + 1], dims[l]
        Ws.append(np.asarray(flat[o:o + n * k], dtype=np.float64).reshape(n, k))
        o += n * k
        bs.append(np.asarray(flat[o:o + n], dtype=np.float64))
        o += n
    return Ws, bs


def flatten(Ws, bs):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in zip(Ws, bs)])


class MLP:
    def __init__(self, dims, flat_params, bf16=True):
        self.dims = list(dims)
        self.Ws, self.bs = unflatten(flat_params, dims)
        self.bf16 = bf16

    def _r(self, a):
        return bf16_round(a) if self.bf16 else np.asarray(a, dtype=np.float64)

    def forward(self, X):
        H = self._r(X)
        Hs, Zs = [], []
        for l, (W, b) in enumerate(zip(self.Ws, self.bs)):
            Hs.append(H)
            Z = H @ self._r(W).T + b
            Zs.append(Z)
            if l + 1 < len(self.Ws):
                H = self._r(gelu(Z))
        return Zs[-1], Hs, Zs

    def loss_grad(self, X, T):
        """Mean squared error over all outputs and its parameter gradient (flat)."""
        Y, Hs, Zs = self.forward(X)
        B, N = Y.shape
        E = Y - np.asarray(T, dtype=np.float64)
        loss = float(np.sum(E * E) / (B * N))
        dZ = 2.0 * E / (B * N)
        gWs, gbs = [None] * len(self.Ws), [None] * len(self.Ws)
        for l in range(len(self.Ws) - 1, -1, -1):
            dZr = self._r(dZ)
            gWs[l] = dZr.T @ Hs[l]
            gbs[l] = dZ.sum(0)
            if l == 0:
                break
            dH = dZr @ self._r(self.Ws[l])
            dZ = dH * gelu_grad(Zs[l - 1])
        return loss, flatten(gWs, gbs)


def adamw(flat, grad, m, v, step, lr, b1, b2, eps, wd, dims):
    """One AdamW step (weights decayed, biases not), as k_mlp_adamw does."""
    flat, m, v = flat.copy(), m.copy(), v.copy()
    c1, c2 = 1.0 - b1 ** step, 1.0 - b2 ** step
    m[:] = b1 * m + (1 - b1) * grad
    v[:] = b2 * v + (1 - b2) * grad * grad
    decay = np.zeros_like(flat)
    o = 0
    for l in range(len(dims) - 1):
        n, k = dims[l + 1], dims[l]
        decay[o:o + n * k] = wd
        o += n * k + n
    flat -= lr * (decay * flat + (m / c1) / (np.sqrt(v / c2) + eps))
    return flat, m, v
