"""MLP emulator of the pixel likelihood: -2 Delta lnL(theta) from five parameters.

Network 5 -> 256 -> 256 -> 256 -> 1 with SiLU activations, BF16 weight
matrices and FP32 accumulation; FP32 master parameters and Adam moments.
Every forward, backward and optimiser operation is a kernel of
``csrc/mlp.cu``; one training step (forward, loss, backward, Adam) is
captured once in a CUDA graph and replayed.

Inputs are the parameters mapped from their prior box to [-1, 1]; the
target is standardised, t = (-2 lnL - mu) / sigma, so the network works on
O(1) numbers and lnL~ = -(mu + sigma y) / 2.

No counterpart in the reference: the emulator is trained on evaluations
of the exact likelihood (``Engine.lnl``) and serves as the first stage of
the delayed-acceptance sampler in :mod:`cosmoforge_b200.sampler`.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import check, lib, stream

SIZES = (5, 256, 256, 256, 1)
F32 = torch.float32


def param_layout(sizes=SIZES):
    """[(w_off, b_off, n_in, n_out)] of the flat parameter vector (W row-major out x in, then b)."""
    out, off = [], 0
    for n_in, n_out in zip(sizes[:-1], sizes[1:]):
        out.append((off, off + n_in * n_out, n_in, n_out))
        off += n_in * n_out + n_out
    return out, off


class MLPEmulator:
    def __init__(self, lo, hi, sizes=SIZES, seed: int = 0, device=None):
        self.dev = torch.device(device or "cuda")
        self.lib = lib()
        self.sizes = tuple(sizes)
        self.layout, self.n_params = param_layout(self.sizes)
        self.lo = torch.as_tensor(np.asarray(lo, np.float64), device=self.dev)
        self.hi = torch.as_tensor(np.asarray(hi, np.float64), device=self.dev)
        g = np.random.default_rng(seed)
        p = np.zeros(self.n_params, np.float32)
        for w_off, b_off, n_in, n_out in self.layout:
            bound = math.sqrt(6.0 / n_in) if n_out > 1 else math.sqrt(1.0 / n_in)
            p[w_off:b_off] = g.uniform(-bound, bound, n_in * n_out)
        self.p = torch.from_numpy(p).to(self.dev)
        self.p16 = torch.empty(self.n_params, dtype=torch.bfloat16, device=self.dev)
        check(self.lib.cf_to_bf16(self.n_params, self.p.data_ptr(), self.p16.data_ptr(), stream()), "cf_to_bf16")
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.loss = torch.zeros(1, dtype=F32, device=self.dev)
        self.mu, self.sigma = 0.0, 1.0
        self._bufs = {}
        self._graph = None

    # -- buffers -----------------------------------------------------------
    def _buffers(self, M):
        if M not in self._bufs:
            w = max(self.sizes[1:])
            self._bufs[M] = dict(
                X=torch.zeros((M, self.sizes[0]), dtype=F32, device=self.dev),
                Z=[torch.empty((M, n), dtype=F32, device=self.dev) for n in self.sizes[1:]],
                A=[torch.empty((M, n), dtype=F32, device=self.dev) for n in self.sizes[1:]],
                dZ=torch.empty((M, w), dtype=F32, device=self.dev),
                dZ2=torch.empty((M, w), dtype=F32, device=self.dev),
                t=torch.zeros(M, dtype=F32, device=self.dev),
                w=torch.ones(M, dtype=F32, device=self.dev),
            )
        return self._bufs[M]

    def _wptr(self, k, t=None):
        """Address of layer k's weight matrix in t (default: the BF16 working copy)."""
        t = self.p16 if t is None else t
        return t.data_ptr() + self.layout[k][0] * t.element_size()

    def _bptr(self, k, t=None):
        """Address of layer k's bias in t (default: the FP32 master vector)."""
        t = self.p if t is None else t
        return t.data_ptr() + self.layout[k][1] * t.element_size()

    # -- kernels -----------------------------------------------------------
    def _forward(self, buf, M):
        A = buf["X"]
        nl = len(self.layout)
        for k, (_, _, n_in, n_out) in enumerate(self.layout):
            act = 1 if k < nl - 1 else 0
            check(self.lib.cf_mlp_dense_fwd(M, n_out, n_in, A.data_ptr(), n_in, self._wptr(k), self._bptr(k), act,
                                            buf["Z"][k].data_ptr(), buf["A"][k].data_ptr(), n_out, stream()),
                  "cf_mlp_dense_fwd")
            A = buf["A"][k]
        return buf["A"][-1]

    def _backward(self, buf, M):
        """Gradients into self.g from dY in buf['dZ'][:, :1]."""
        nl = len(self.layout)
        dZ, spare = buf["dZ"], buf["dZ2"]
        for k in range(nl - 1, -1, -1):
            _, _, n_in, n_out = self.layout[k]
            Aprev = buf["X"] if k == 0 else buf["A"][k - 1]
            check(self.lib.cf_mlp_dense_bwd_weight(M, n_out, n_in, dZ.data_ptr(), Aprev.data_ptr(), n_in,
                                                   self._wptr(k, self.g),
                                                   self._bptr(k, self.g), stream()), "cf_mlp_dense_bwd_weight")
            if k > 0:
                check(self.lib.cf_mlp_dense_bwd_data(M, n_out, n_in, dZ.data_ptr(), self._wptr(k),
                                                     buf["Z"][k - 1].data_ptr(), spare.data_ptr(), stream()),
                      "cf_mlp_dense_bwd_data")
                dZ, spare = spare, dZ

    def loss_and_grad(self, X, t, w=None):
        """(loss, flat gradient) for inputs X (M x 5, already in [-1, 1]) and standardised targets t."""
        M = X.shape[0]
        buf = self._buffers(M)
        buf["X"].copy_(X)
        buf["t"].copy_(t)
        y = self._forward(buf, M)
        check(self.lib.cf_mlp_mse(M, y.data_ptr(), buf["t"].data_ptr(), None if w is None else w.data_ptr(),
                                  buf["dZ"].data_ptr(), self.loss.data_ptr(), stream()), "cf_mlp_mse")
        self._backward(buf, M)
        return float(self.loss.item()), self.g.clone()

    def _train_step(self, buf, M, lr, b1, b2, eps):
        y = self._forward(buf, M)
        check(self.lib.cf_mlp_mse(M, y.data_ptr(), buf["t"].data_ptr(), buf["w"].data_ptr(), buf["dZ"].data_ptr(),
                                  self.loss.data_ptr(), stream()), "cf_mlp_mse")
        self._backward(buf, M)
        check(self.lib.cf_mlp_adam(self.n_params, self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                                   self.v.data_ptr(), lr, b1, b2, eps, self.step.data_ptr(), self.p16.data_ptr(),
                                   stream()), "cf_mlp_adam")

    # -- public ------------------------------------------------------------
    def normalise(self, theta):
        th = torch.as_tensor(theta, dtype=torch.float64, device=self.dev)
        return (2.0 * (th - self.lo) / (self.hi - self.lo) - 1.0).to(F32)

    def fit(self, theta, m2lnl, steps: int = 3000, batch: int = 1024, lr: float = 1e-3, seed: int = 0,
            graph: bool = True, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        """Train on exact evaluations: theta (P x 5), m2lnl = -2 lnL (P,).  Returns the loss history."""
        th = torch.as_tensor(theta, dtype=torch.float64, device=self.dev)
        y = torch.as_tensor(m2lnl, dtype=torch.float64, device=self.dev)
        self.mu = float(y.mean())
        self.sigma = float(y.std()) or 1.0
        X_all = self.normalise(th)
        t_all = ((y - self.mu) / self.sigma).to(F32)
        P = th.shape[0]
        buf = self._buffers(batch)
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        perm = torch.randperm(P, device=self.dev, generator=gen)
        per_epoch = max(P // batch, 1)
        hist = []
        g = None
        for it in range(steps):
            k = it % per_epoch
            if k == 0 and it > 0:
                perm = torch.randperm(P, device=self.dev, generator=gen)
            idx = perm[k * batch:(k + 1) * batch]
            buf["X"].copy_(X_all[idx])
            buf["t"].copy_(t_all[idx])
            if g is not None:
                g.replay()
            else:
                # the first step runs eagerly (loads every kernel), later ones replay one capture
                self._train_step(buf, batch, lr, b1, b2, eps)
                if graph:
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        self._train_step(buf, batch, lr, b1, b2, eps)
            if it % 100 == 0 or it == steps - 1:
                hist.append((it, float(self.loss.item())))
        self._graph = g
        return hist

    def predict_std(self, X):
        """Standardised output y for normalised inputs X (M x 5, FP32 on the device)."""
        M = X.shape[0]
        buf = self._buffers(M)
        buf["X"].copy_(X)
        return self._forward(buf, M)[:, 0]

    def predict_m2lnl(self, theta):
        """Emulated -2 lnL at parameter points theta (M x 5)."""
        y = self.predict_std(self.normalise(theta))
        return self.mu + self.sigma * y.double()
