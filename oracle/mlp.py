"""CPU oracle of the energy surrogate network (test infrastructure only).

FP64 restatement of the library's MLP (64 -> H -> H -> H -> 1, SiLU, learned 32-wide
embedding in input columns 7..38) with its forward pass, mean-squared-error backward pass and
Adam step. With `bf16=True` the values the GPU stores in BF16 are rounded the same way
(round to nearest even of the FP32 value): the input rows, W1..W3, the activations A1..A3 and
the back-propagated pre-activation gradients D1..D3; everything else (biases, w4, the output,
the loss, products' accumulation) stays wide, as the GPU keeps it in FP32. With `bf16=False`
it is the exact FP64 network, used to check the analytic gradient by finite differences.

The network has no counterpart in the reference code; its parameter layout is the one
gd_mlp_get_params returns: W1 [64][H], b1 [H], W2 [H][H], b2, W3 [H][H], b3, w4 [H], b4 (+3
padding), embedding [n_emb][32].
"""
from __future__ import annotations

import numpy as np

IN = 64
EMB = 32
EMB_OFF = 7


def layout(hidden: int, n_emb: int):
    o = {}
    off = 0
    for name, size in (("w1", IN * hidden), ("b1", hidden), ("w2", hidden * hidden),
                       ("b2", hidden), ("w3", hidden * hidden), ("b3", hidden), ("w4", hidden),
                       ("b4", 4), ("emb", n_emb * EMB)):
        o[name] = (off, size)
        off += size
    o["total"] = off
    return o


def bf16(a):
    """Round FP32 values to BF16 (nearest, ties to even) and return them as float64."""
    f = np.ascontiguousarray(np.asarray(a, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


class MlpOracle:
    def __init__(self, theta: np.ndarray, hidden: int, n_emb: int, bf16_mode: bool = True):
        self.H, self.n_emb, self.bf = hidden, n_emb, bf16_mode
        self.L = layout(hidden, n_emb)
        assert theta.size == self.L["total"]
        self.theta = np.asarray(theta, np.float64).copy()

    def _p(self, name, shape=None):
        off, size = self.L[name]
        v = self.theta[off:off + size]
        return v.reshape(shape) if shape else v

    def _r(self, a):
        return bf16(a) if self.bf else a

    def rows(self, x, conf=None):
        x = np.asarray(x, np.float64).reshape(-1, IN).copy()
        if conf is not None and self.n_emb:
            emb = self._p("emb", (self.n_emb, EMB))
            for r, c in enumerate(conf):
                if c >= 0:
                    x[r, EMB_OFF:EMB_OFF + EMB] = emb[c]
        return self._r(x)

    def forward(self, x, conf=None, keep=False):
        H = self.H
        X = self.rows(x, conf)
        W1 = self._r(self._p("w1", (IN, H)))
        W2 = self._r(self._p("w2", (H, H)))
        W3 = self._r(self._p("w3", (H, H)))
        Z1 = X @ W1 + self._p("b1")
        A1 = self._r(_silu(Z1))
        Z2 = A1 @ W2 + self._p("b2")
        A2 = self._r(_silu(Z2))
        Z3 = A2 @ W3 + self._p("b3")
        A3 = self._r(_silu(Z3))
        y = A3 @ self._p("w4") + self._p("b4")[0]
        if keep:
            self._cache = (X, W1, W2, W3, Z1, A1, Z2, A2, Z3, A3)
        return y

    def loss(self, x, t, conf=None):
        y = self.forward(x, conf)
        return float(np.mean((y - np.asarray(t, np.float64)) ** 2))

    def backward(self, x, t, conf=None):
        """Loss and gradient (flat, in the parameter layout)."""
        y = self.forward(x, conf, keep=True)
        X, W1, W2, W3, Z1, A1, Z2, A2, Z3, A3 = self._cache
        t = np.asarray(t, np.float64)
        n = y.shape[0]
        g = np.zeros(self.L["total"])

        def put(name, v):
            off, size = self.L[name]
            g[off:off + v.size] += v.ravel()

        dy = 2.0 * (y - t) / n
        put("w4", A3.T @ dy)
        put("b4", np.array([dy.sum()]))
        D3 = self._r(np.outer(dy, self._p("w4")) * _silu_grad(Z3))
        put("w3", A2.T @ D3)
        put("b3", D3.sum(0))
        D2 = self._r((D3 @ W3.T) * _silu_grad(Z2))
        put("w2", A1.T @ D2)
        put("b2", D2.sum(0))
        D1 = self._r((D2 @ W2.T) * _silu_grad(Z1))
        put("w1", X.T @ D1)
        put("b1", D1.sum(0))
        if self.n_emb and conf is not None:
            dX = D1 @ W1.T
            off, _ = self.L["emb"]
            for r, c in enumerate(conf):
                if c >= 0:
                    g[off + c * EMB: off + (c + 1) * EMB] += dX[r, EMB_OFF:EMB_OFF + EMB]
        return float(np.mean((y - t) ** 2)), g

    @staticmethod
    def adam(theta, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
        """One Adam step (Kingma & Ba, 2015) in place; t is the 1-based step count."""
        m[:] = b1 * m + (1 - b1) * g
        v[:] = b2 * v + (1 - b2) * g * g
        theta -= lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
