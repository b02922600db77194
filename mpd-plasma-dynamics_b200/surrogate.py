"""Learned warm start: a spectral neural operator that predicts the steady
state of the channel from its parameters, trained and run on the GPU with the
library's own kernels (tcgen05 BF16 GEMMs with FP32 accumulation, FP32
element-wise kernels, Adam).  torch only allocates device memory and supplies
the stream; every arithmetic operation is a kernel of libmpd_b200.so.

Network (grid H x W = L x (M+1) points, P = H W, width C = 64):
  input   per point: the 4 parameters (amp, beta, v_z, a; scaled to [-1, 1],
          beta in log space) broadcast over the grid, and r, z
  lift    h = x W_in + b_in
  4 x     h <- act(h W_l + b_l + G (R_l . (F h)))
          F: projection on 8 Fourier modes per axis (cos 2 pi k x, k = 0..7,
          sin 2 pi k x, k = 1..8) -> Q = 16 x 16 coefficients per channel;
          R_l: one C x C channel mix per coefficient; G: synthesis back to the
          grid; act = GELU (none after the last layer)
  project y = GELU(h W_p1 + b_p1) W_p2 + b_p2: the 8 fields rho, v_z, v_r,
          v_phi, e, H_z, H_r, H_phi, each normalised by its training mean/std
Loss: mean squared error of the normalised fields.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np

from . import _native as N
from . import nn

FIELDS = ("rho", "v_z", "v_r", "v_phi", "e", "H_z", "H_r", "H_phi")
N_IN, N_OUT = 6, 8
WIDTH, MODES, LAYERS, HIDDEN = 64, 8, 4, 128
PARAM_RANGES = ((0.5, 2.0), (math.log(0.05), math.log(1.0)), (0.05, 0.3), (0.0, 0.2))


def axis_basis(n: int, modes: int = MODES) -> np.ndarray:
    """(2 modes) x n: cos(2 pi k x), k < modes, then sin(2 pi k x), k = 1..modes,
    at cell centres x = (i + 1/2) / n."""
    x = (np.arange(n) + 0.5) / n
    cos = [np.cos(2 * np.pi * k * x) for k in range(modes)]
    sin = [np.sin(2 * np.pi * k * x) for k in range(1, modes + 1)]
    return np.array(cos + sin)


def bases(H: int, W: int, modes: int = MODES):
    """Forward projection F (Q x P, the grid average of each basis product)
    and synthesis G (P x Q), Q = (2 modes)^2, P = H W, point index h W + w."""
    bz, by = axis_basis(H, modes), axis_basis(W, modes)
    prod = np.einsum("ah,bw->abhw", bz, by).reshape(bz.shape[0] * by.shape[0], H * W)
    return prod / (H * W), np.ascontiguousarray(prod.T)


def param_vector(amp, beta, vz, a) -> np.ndarray:
    raw = (amp, math.log(beta), vz, a)
    return np.array([2 * (v - lo) / (hi - lo) - 1 for v, (lo, hi) in zip(raw, PARAM_RANGES)])


def features(pv: np.ndarray, r: np.ndarray, z: np.ndarray) -> np.ndarray:
    """P x 6 input of one solve: pv broadcast, r (H x W) and z (H) scaled."""
    H, W = r.shape
    x = np.empty((H, W, N_IN))
    x[..., :4] = pv
    x[..., 4] = 2 * (r - 0.5) / 0.6
    x[..., 5] = (2 * z - 1)[:, None]
    return x.reshape(H * W, N_IN)


def param_shapes(width=WIDTH, modes=MODES, layers=LAYERS, hidden=HIDDEN):
    q = (2 * modes) ** 2
    shapes = [("W_in", (N_IN, width)), ("b_in", (width,))]
    for l in range(layers):
        shapes += [(f"W{l}", (width, width)), (f"b{l}", (width,)), (f"R{l}", (q, width, width))]
    shapes += [("W_p1", (width, hidden)), ("b_p1", (hidden,)), ("W_p2", (hidden, N_OUT)),
               ("b_p2", (N_OUT,))]
    return shapes


def init_params(seed: int = 0, **kw) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    out = {}
    for name, shape in param_shapes(**kw):
        if name.startswith("b"):
            out[name] = np.zeros(shape)
        elif name.startswith("R"):
            out[name] = rng.standard_normal(shape) * (0.5 / math.sqrt(shape[1]))
        else:
            out[name] = rng.standard_normal(shape) / math.sqrt(shape[0])
    return out


@dataclasses.dataclass
class Normalizer:
    """Per-field affine normalisation of the targets.  A field that is the
    same constant in every training state (v_phi, H_z, H_r of the channel
    are identically zero) is not learned: decode returns the constant
    exactly, so a warm start keeps it exact (the per-field relative residual
    would otherwise see the network's tiny output there as a large change)."""
    mean: np.ndarray   # per field
    std: np.ndarray
    const: np.ndarray  # per field: True if constant in the training data

    @classmethod
    def fit(cls, fields: np.ndarray) -> "Normalizer":
        f = fields.reshape(-1, N_OUT)
        mean, std = f.mean(0, dtype=np.float64), f.std(0, dtype=np.float64)
        const = std <= 1e-12 * np.maximum(1.0, np.abs(mean))
        return cls(mean, np.where(const, 1.0, std), const)

    def encode(self, f):
        return np.where(self.const, 0.0, (f - self.mean) / self.std)

    def decode(self, f):
        return np.where(self.const, self.mean, f * self.std + self.mean)


class SpectralOperator:
    """The network on one grid shape, with its device buffers for a batch of
    `batch` samples.  forward / backward / adam_step run on the current torch
    stream."""

    def __init__(self, H: int, W: int, batch: int, params: dict | None = None, seed: int = 0):
        import torch
        self.torch = torch
        self.H, self.W, self.P, self.B = H, W, H * W, batch
        self.Q = (2 * MODES) ** 2
        self.shapes = param_shapes()
        sizes = [int(np.prod(s)) for _, s in self.shapes]
        self.nparam = sum(sizes)
        dev = torch.device("cuda")
        f32 = dict(device=dev, dtype=torch.float32)
        self.flat = torch.zeros(self.nparam, **f32)
        self.grad = torch.zeros(self.nparam, **f32)
        self.m = torch.zeros(self.nparam, **f32)
        self.v = torch.zeros(self.nparam, **f32)
        self.p, self.g = {}, {}
        off = 0
        for (name, shape), n in zip(self.shapes, sizes):
            self.p[name] = self.flat[off:off + n].view(shape)
            self.g[name] = self.grad[off:off + n].view(shape)
            off += n
        self.set_params(params if params is not None else init_params(seed))
        Fq, G = bases(H, W)
        self.F = torch.from_numpy(Fq.astype(np.float32)).to(dev)
        self.G = torch.from_numpy(G.astype(np.float32)).to(dev)
        rows = batch * self.P
        self.x = torch.zeros(rows, N_IN, **f32)
        self.z = [torch.zeros(rows, WIDTH, **f32) for _ in range(LAYERS + 1)]
        self.h = [torch.zeros(rows, WIDTH, **f32) for _ in range(LAYERS + 1)]
        self.V = [torch.zeros(batch, self.Q, WIDTH, **f32) for _ in range(LAYERS)]
        self.U = torch.zeros(batch, self.Q, WIDTH, **f32)
        self.zp = torch.zeros(rows, HIDDEN, **f32)
        self.y1 = torch.zeros(rows, HIDDEN, **f32)
        self.out = torch.zeros(rows, N_OUT, **f32)
        self.zo = torch.zeros(rows, N_OUT, **f32)
        # backward scratch
        self.g_a = torch.zeros(rows, max(WIDTH, HIDDEN), **f32)
        self.g_b = torch.zeros(rows, max(WIDTH, HIDDEN), **f32)
        self.g_out = torch.zeros(rows, N_OUT, **f32)
        self.gh = [torch.zeros(rows, WIDTH, **f32) for _ in range(2)]
        self.gz = torch.zeros(rows, WIDTH, **f32)
        self.gU = torch.zeros(batch, self.Q, WIDTH, **f32)
        self.gV = torch.zeros(batch, self.Q, WIDTH, **f32)
        self.parts = torch.zeros(batch * max(WIDTH, HIDDEN) * max(WIDTH, HIDDEN), **f32)
        self.partial = torch.zeros(148 * 32, device=dev, dtype=torch.float64)
        self.colwork = torch.zeros(128 * max(WIDTH, HIDDEN), **f32)
        # split-K partial sums of the long-K products (grid sums, weight gradients)
        self.work = torch.zeros(16 * batch * self.Q * WIDTH, **f32)
        self.loss = torch.zeros(1, device=dev, dtype=torch.float64)
        self.target = torch.zeros(rows, N_OUT, **f32)   # the captured iteration's targets
        self.graph = None
        self.step = 0
        self.lib = N.load()

    # ---------------------------------------------------------------- params
    def set_params(self, params: dict):
        for name, _ in self.shapes:
            self.p[name].copy_(self.torch.from_numpy(np.asarray(params[name], dtype=np.float32)))

    def get_params(self) -> dict[str, np.ndarray]:
        return {k: v.detach().cpu().numpy().astype(np.float64) for k, v in self.p.items()}

    def grads(self) -> dict[str, np.ndarray]:
        return {k: v.detach().cpu().numpy().astype(np.float64) for k, v in self.g.items()}

    # ----------------------------------------------------------------- calls
    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _chk(self, rc):
        N.check(rc, self.lib)

    def _linear(self, x, k_in, Wt, n_out, out, beta=0.0):
        """out[rows, n_out] (+)= x[rows, k_in] @ Wt[k_in, n_out]."""
        rows = x.shape[0]
        nn.gemm(x, Wt, out, rows, n_out, k_in, 1, sa=(x.stride(0), 1, 0), sb=(1, n_out, 0),
                sc=(out.stride(0), 1, 0), beta=beta)

    def _bias_act(self, z, b, out, act):
        self._chk(self.lib.mpd_nn_bias_act(C.c_void_p(z.data_ptr()), C.c_void_p(b.data_ptr()),
                                           C.c_void_p(out.data_ptr()), z.shape[0], z.shape[1],
                                           int(act), self._s()))

    def _wgrad(self, a, k_in, gz, n_out, dst):
        """dst[k_in, n_out] = sum over rows of a[:, :k_in]^T gz, split by sample."""
        B, P = self.B, self.P
        parts = self.parts[:B * k_in * n_out]
        nn.gemm(a, gz, parts, k_in, n_out, P, B, sa=(1, a.stride(0), P * a.stride(0)),
                sb=(1, gz.stride(0), P * gz.stride(0)), sc=(n_out, 1, k_in * n_out),
                work=self.work)
        self._chk(self.lib.mpd_nn_sum_parts(C.c_void_p(parts.data_ptr()), B, k_in * n_out,
                                            C.c_void_p(dst.data_ptr()), 0, self._s()))

    def _colsum(self, x, dst):
        self._chk(self.lib.mpd_nn_colsum(C.c_void_p(x.data_ptr()), x.shape[0], x.shape[1],
                                         C.c_void_p(dst.data_ptr()),
                                         C.c_void_p(self.colwork.data_ptr()), self._s()))

    # --------------------------------------------------------------- forward
    def load_inputs(self, x: np.ndarray):
        """x: B x P x 6 features."""
        self.x.copy_(self.torch.from_numpy(x.reshape(-1, N_IN).astype(np.float32)))

    def forward(self):
        B, P, Q, Cw = self.B, self.P, self.Q, WIDTH
        p = self.p
        self._linear(self.x, N_IN, p["W_in"], Cw, self.z[0])
        self._bias_act(self.z[0], p["b_in"], self.h[0], act=False)
        for l in range(LAYERS):
            h, z = self.h[l], self.z[l + 1]
            self._linear(h, Cw, p[f"W{l}"], Cw, z)
            # V[b] = F h[b]  (Q x C)
            nn.gemm(self.F, h, self.V[l], Q, Cw, P, B, sa=(P, 1, 0), sb=(1, Cw, P * Cw),
                    sc=(Cw, 1, Q * Cw), work=self.work)
            # U[b, q] = V[b, q] R[q]   (batched over q)
            nn.gemm(self.V[l], p[f"R{l}"], self.U, B, Cw, Cw, Q, sa=(Q * Cw, 1, Cw),
                    sb=(1, Cw, Cw * Cw), sc=(Q * Cw, 1, Cw))
            # z[b] += G U[b]
            nn.gemm(self.G, self.U, z, P, Cw, Q, B, sa=(Q, 1, 0), sb=(1, Cw, Q * Cw),
                    sc=(Cw, 1, P * Cw), beta=1.0)
            self._bias_act(z, p[f"b{l}"], self.h[l + 1], act=l < LAYERS - 1)
        self._linear(self.h[LAYERS], Cw, p["W_p1"], HIDDEN, self.zp)
        self._bias_act(self.zp, p["b_p1"], self.y1, act=True)
        self._linear(self.y1, HIDDEN, p["W_p2"], N_OUT, self.zo)
        self._bias_act(self.zo, p["b_p2"], self.out, act=False)
        return self.out

    def loss_and_grad(self, target) -> None:
        """Mean squared error against target (rows x 8, device); its gradient
        into g_out.  The loss stays on the device (self.loss)."""
        self._chk(self.lib.mpd_nn_mse(C.c_void_p(self.out.data_ptr()), C.c_void_p(target.data_ptr()),
                                      self.out.numel(), C.c_void_p(self.g_out.data_ptr()),
                                      C.c_void_p(self.partial.data_ptr()),
                                      C.c_void_p(self.loss.data_ptr()), self._s()))

    # -------------------------------------------------------------- backward
    def backward(self):
        B, P, Q, Cw = self.B, self.P, self.Q, WIDTH
        p, g = self.p, self.g
        rows = B * P
        # projection
        self._wgrad(self.y1, HIDDEN, self.g_out, N_OUT, g["W_p2"])
        self._colsum(self.g_out, g["b_p2"])
        gy1 = self.g_a[:, :HIDDEN]
        nn.gemm(self.g_out, p["W_p2"], gy1, rows, HIDDEN, N_OUT, 1, sa=(N_OUT, 1, 0),
                sb=(N_OUT, 1, 0), sc=(self.g_a.stride(0), 1, 0))
        gzp = self.g_b[:, :HIDDEN]
        self._chk(self.lib.mpd_nn_act_bwd(C.c_void_p(gy1.data_ptr()), C.c_void_p(self.zp.data_ptr()),
                                          C.c_void_p(gzp.data_ptr()), rows * HIDDEN, self._s()))
        self._wgrad(self.h[LAYERS], Cw, gzp, HIDDEN, g["W_p1"])
        self._colsum(gzp, g["b_p1"])
        gh = self.gh[0]
        nn.gemm(gzp, p["W_p1"], gh, rows, Cw, HIDDEN, 1, sa=(HIDDEN, 1, 0), sb=(HIDDEN, 1, 0),
                sc=(Cw, 1, 0))
        for l in reversed(range(LAYERS)):
            z, h = self.z[l + 1], self.h[l]
            if l < LAYERS - 1:
                gz = self.gz
                self._chk(self.lib.mpd_nn_act_bwd(C.c_void_p(gh.data_ptr()), C.c_void_p(z.data_ptr()),
                                                  C.c_void_p(gz.data_ptr()), rows * Cw, self._s()))
            else:
                gz = gh
            self._wgrad(h, Cw, gz, Cw, g[f"W{l}"])
            self._colsum(gz, g[f"b{l}"])
            # gU[b] = G^T gz[b]
            nn.gemm(self.G, gz, self.gU, Q, Cw, P, B, sa=(1, Q, 0), sb=(1, Cw, P * Cw),
                    sc=(Cw, 1, Q * Cw), work=self.work)
            # dR[q] = sum_b V[b, q]^T gU[b, q]
            nn.gemm(self.V[l], self.gU, g[f"R{l}"], Cw, Cw, B, Q, sa=(1, Q * Cw, Cw),
                    sb=(1, Q * Cw, Cw), sc=(Cw, 1, Cw * Cw))
            # gV[b, q] = gU[b, q] R[q]^T
            nn.gemm(self.gU, p[f"R{l}"], self.gV, B, Cw, Cw, Q, sa=(Q * Cw, 1, Cw),
                    sb=(Cw, 1, Cw * Cw), sc=(Q * Cw, 1, Cw))
            # gh = gz W^T + F^T gV
            gh_new = self.gh[1] if gh is self.gh[0] else self.gh[0]
            nn.gemm(gz, p[f"W{l}"], gh_new, rows, Cw, Cw, 1, sa=(Cw, 1, 0), sb=(Cw, 1, 0),
                    sc=(Cw, 1, 0))
            nn.gemm(self.F, self.gV, gh_new, P, Cw, Q, B, sa=(1, P, 0), sb=(1, Cw, Q * Cw),
                    sc=(Cw, 1, P * Cw), beta=1.0)
            gh = gh_new
        # lift (the input needs no gradient)
        self._wgrad(self.x, N_IN, gh, Cw, g["W_in"])
        self._colsum(gh, g["b_in"])

    # ------------------------------------------------------ captured iteration
    def capture(self) -> None:
        """Record forward, loss (against self.target) and backward of one
        training iteration as a CUDA graph: ~100 kernel launches replayed as
        one.  Inputs and targets are read from self.x and self.target, so a
        step only refills those buffers; Adam stays outside the graph (its
        bias correction takes the step count as an argument)."""
        torch = self.torch
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):  # one eager pass first (one-time set-up of the launches)
            self.forward()
            self.loss_and_grad(self.target)
            self.backward()
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.forward()
            self.loss_and_grad(self.target)
            self.backward()
        self.graph = g

    def train_step(self, lr=1e-3) -> None:
        """One training iteration on self.x / self.target: the captured graph
        when there is one, else the same calls eagerly; then Adam."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self.forward()
            self.loss_and_grad(self.target)
            self.backward()
        self.adam_step(lr=lr)

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        self._chk(self.lib.mpd_nn_adam(C.c_void_p(self.flat.data_ptr()), C.c_void_p(self.grad.data_ptr()),
                                       C.c_void_p(self.m.data_ptr()), C.c_void_p(self.v.data_ptr()),
                                       self.nparam, float(lr), float(b1), float(b2), float(eps),
                                       self.step, self._s()))

    def wait(self):
        nn.wait_status()
