"""CPU oracle of the surrogate network (test infrastructure only): a numpy
restatement of the spectral neural operator of the library's surrogate
(forward, mean-squared-error loss and hand-derived backward), in float64.

With bf16=True every matrix product rounds both operands to BF16 (round to
nearest even) first, as the GPU's tensor-core GEMM does; the sums stay in
float64.  The network has no counterpart in the reference, so there is no
reference file to cite; its own pin is the finite-difference check of the
backward pass in tests/test_surrogate_oracle.py.
"""
from __future__ import annotations

import math

import numpy as np

WIDTH, MODES, LAYERS, HIDDEN, N_IN, N_OUT = 64, 8, 4, 128, 6, 8


def bf16_round(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64).reshape(np.shape(x))


def axis_basis(n, modes=MODES):
    x = (np.arange(n) + 0.5) / n
    rows = [np.cos(2 * math.pi * k * x) for k in range(modes)]
    rows += [np.sin(2 * math.pi * k * x) for k in range(1, modes + 1)]
    return np.array(rows)


def bases(H, W, modes=MODES):
    bz, by = axis_basis(H, modes), axis_basis(W, modes)
    prod = np.einsum("ah,bw->abhw", bz, by).reshape(len(bz) * len(by), H * W)
    return prod / (H * W), prod.T.copy()


def gelu(x):
    c = math.sqrt(2 / math.pi)
    t = np.tanh(c * (x + 0.044715 * x ** 3))
    return 0.5 * x * (1 + t)


def gelu_grad(x):
    c = math.sqrt(2 / math.pi)
    t = np.tanh(c * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * c * (1 + 3 * 0.044715 * x * x)


class Oracle:
    def __init__(self, H, W, bf16=False):
        self.H, self.W, self.P = H, W, H * W
        self.F, self.G = bases(H, W)
        self.r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))

    def mm(self, a, b):
        """a @ b with both operands rounded as the GPU GEMM rounds them."""
        return np.matmul(self.r(a), self.r(b))

    def forward(self, p, x):
        """x: B x P x 6.  Returns the output (B x P x 8) and the saved values."""
        mm = self.mm
        s = {"x": x}
        z = mm(x, p["W_in"]) + p["b_in"]
        h = z
        s["h"] = [h]
        s["z"] = []
        s["V"] = []
        for l in range(LAYERS):
            V = np.stack([mm(self.F, hb) for hb in h])                   # B x Q x C
            U = np.einsum("bqc,qcd->bqd", self.r(V), self.r(p[f"R{l}"]))
            S = np.stack([mm(self.G, ub) for ub in U])                   # B x P x C
            z = mm(h, p[f"W{l}"]) + S + p[f"b{l}"]
            h = gelu(z) if l < LAYERS - 1 else z
            s["V"].append(V)
            s["z"].append(z)
            s["h"].append(h)
        zp = mm(h, p["W_p1"]) + p["b_p1"]
        y1 = gelu(zp)
        out = mm(y1, p["W_p2"]) + p["b_p2"]
        s["zp"], s["y1"] = zp, y1
        return out, s

    @staticmethod
    def loss(out, target):
        return float(np.mean((out - target) ** 2))

    def backward(self, p, s, out, target):
        mm, r = self.mm, self.r
        g = {}
        n = out.size
        go = 2.0 * (out - target) / n
        y1 = s["y1"]
        g["W_p2"] = np.einsum("bpi,bpo->io", r(y1), r(go))
        g["b_p2"] = go.sum((0, 1))
        gzp = mm(go, p["W_p2"].T) * gelu_grad(s["zp"])
        h = s["h"][LAYERS]
        g["W_p1"] = np.einsum("bpi,bpo->io", r(h), r(gzp))
        g["b_p1"] = gzp.sum((0, 1))
        gh = mm(gzp, p["W_p1"].T)
        for l in reversed(range(LAYERS)):
            z, hin, V = s["z"][l], s["h"][l], s["V"][l]
            gz = gh * gelu_grad(z) if l < LAYERS - 1 else gh
            g[f"W{l}"] = np.einsum("bpi,bpo->io", r(hin), r(gz))
            g[f"b{l}"] = gz.sum((0, 1))
            gU = np.stack([mm(self.G.T, gb) for gb in gz])              # B x Q x C
            g[f"R{l}"] = np.einsum("bqi,bqo->qio", r(V), r(gU))
            gV = np.einsum("bqo,qio->bqi", r(gU), r(p[f"R{l}"]))
            gh = mm(gz, p[f"W{l}"].T) + np.stack([mm(self.F.T, gb) for gb in gV])
        g["W_in"] = np.einsum("bpi,bpo->io", r(s["x"]), r(gh))
        g["b_in"] = gh.sum((0, 1))
        return g
