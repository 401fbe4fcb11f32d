"""Surrogate network: (parameters, stimulus protocol) -> trace feature vector.

A 4-layer MLP (in -> 512 -> 512 -> 512 -> out, GELU in its tanh form) whose
forward and backward products all run on the project's tcgen05 BF16 GEMM
(ngpu_gemm_bf16_tn, FP32 accumulation in tensor memory) with fused
epilogues:
  forward   Z = H W^T + b, H' = gelu(Z)      (epilogue 1: Z fp32, H' bf16 and
                                              its transpose for the weight
                                              gradients)
  output    Y = H W^T + b                    (epilogue 2)
  backward  dZ = (dZ_next W) * gelu'(Z)      (epilogue 3, bf16 + transpose)
            dW = dZ^T H                      (epilogue 0, K = the batch)
PyTorch holds the buffers and does the elementwise optimizer step (Adam on
FP32 master weights) and the bias sums; it does no matrix products.

Shapes are padded for the tensor cores: the input width to a multiple of 64,
the output to 32, the batch to a multiple of 128 (padding rows carry zero
loss gradient).  Inputs and targets are standardised with statistics fixed
at the first fit.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _ffi

EPI_STORE, EPI_BIAS_GELU, EPI_BIAS, EPI_GELU_GRAD, EPI_SPLIT = 0, 1, 2, 3, 4


def _pad(n: int, m: int) -> int:
    return (n + m - 1) // m * m


class SurrogateMLP:
    def __init__(self, n_in: int, n_out: int, width: int = 512, seed: int = 0, lr: float = 1e-3):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda")
        self.n_in, self.n_out, self.width = n_in, n_out, width
        # 256-wide tiles where the width allows: measured on B200 at batch 8192 x width 512,
        # 0.020 ms per hidden-layer forward GEMM against 0.024 with 128-wide tiles
        self.bn_hidden = 256 if width % 256 == 0 else 128
        self.k_in = _pad(n_in, 64)
        self.n_out_p = _pad(max(n_out, 16), 32)
        dims = [(width, self.k_in), (width, width), (width, width), (self.n_out_p, width)]
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W, self.b = [], []
        for k, (n, kk) in enumerate(dims):
            fan_in = n_in if k == 0 else width
            w = torch.randn(n, kk, generator=g) / math.sqrt(fan_in)
            if k == 0:
                w[:, n_in:] = 0.0
            if k == 3:
                w[n_out:, :] = 0.0
            self.W.append(w.to(self.dev).float().contiguous())
            self.b.append(torch.zeros(n, device=self.dev))
        self.m = [torch.zeros_like(w) for w in self.W] + [torch.zeros_like(b) for b in self.b]
        self.v = [torch.zeros_like(t) for t in self.m]
        self.step_n = 0
        self.lr = lr
        self.x_mu = self.x_sd = self.y_mu = self.y_sd = None
        self._refresh()

    # -------------------------------------------------------------- plumbing
    def _refresh(self):
        """bf16 copies of the weights, row-major [N][K] and transposed [K][N]
        (the backward data GEMM reads W through its transpose); the output
        layer's transpose is padded to K = 64."""
        t = self.torch
        self.Wb = [w.to(t.bfloat16).contiguous() for w in self.W]
        self.Wtb = []
        for k, w in enumerate(self.W):
            wt = w.t().contiguous()
            if k == 3:
                wt = t.nn.functional.pad(wt, (0, 64 - self.n_out_p))
            self.Wtb.append(wt.to(t.bfloat16).contiguous())

    def _gemm(self, A, B, M, N, K, epi, bn, out_f32=None, out_b=None, out_bt=None, ldo=None, ldt=None,
              bias=None, zin=None):
        p = lambda x: None if x is None else C.c_void_p(x.data_ptr())
        st = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        _ffi.check("ngpu_gemm_bf16_tn", _ffi.lib().ngpu_gemm_bf16_tn(
            p(A), p(B), M, N, K, A.shape[1], B.shape[1], epi, bn, p(out_f32), p(out_b), p(out_bt),
            ldo if ldo is not None else N, ldt if ldt is not None else M, p(bias), p(zin), st))

    def _prep_x(self, X):
        t = self.torch
        X = t.as_tensor(X, dtype=t.float32, device=self.dev)
        M = X.shape[0]
        Mp = _pad(M, 128)
        xn = (X - self.x_mu) / self.x_sd if self.x_mu is not None else X
        xb = t.zeros(Mp, self.k_in, device=self.dev, dtype=t.bfloat16)
        xb[:M, :self.n_in] = xn.to(t.bfloat16)
        return xb, M, Mp

    def _forward(self, xb, Mp):
        t = self.torch
        W = self.width
        acts = {"H0": xb, "H0t": xb.t().contiguous()}
        h = xb
        for k in range(3):
            z = t.empty(Mp, W, device=self.dev)
            hb = t.empty(Mp, W, device=self.dev, dtype=t.bfloat16)
            hbt = t.empty(W, Mp, device=self.dev, dtype=t.bfloat16)
            self._gemm(h, self.Wb[k], Mp, W, h.shape[1], EPI_BIAS_GELU, self.bn_hidden, z, hb, hbt, W, Mp,
                       bias=self.b[k])
            acts[f"Z{k + 1}"], acts[f"H{k + 1}"], acts[f"H{k + 1}t"] = z, hb, hbt
            h = hb
        y = t.empty(Mp, self.n_out_p, device=self.dev)
        self._gemm(h, self.Wb[3], Mp, self.n_out_p, W, EPI_BIAS, 32, y, bias=self.b[3])
        return y, acts

    # ------------------------------------------------------------------- API
    def fit_stats(self, X, Y):
        t = self.torch
        X = t.as_tensor(X, dtype=t.float32, device=self.dev)
        Y = t.as_tensor(Y, dtype=t.float32, device=self.dev)
        self.x_mu, self.x_sd = X.mean(0), X.std(0).clamp(min=1e-6)
        self.y_mu, self.y_sd = Y.mean(0), Y.std(0).clamp(min=1e-6)

    def predict(self, X):
        """Features (original units) for inputs X [M, n_in]."""
        xb, M, Mp = self._prep_x(X)
        y, _ = self._forward(xb, Mp)
        out = y[:M, :self.n_out]
        return out * self.y_sd + self.y_mu if self.y_mu is not None else out

    def loss_and_grads(self, X, Y, weight=None):
        """Mean squared error on standardised targets and the gradients of
        every weight and bias (lists in layer order)."""
        t = self.torch
        xb, M, Mp = self._prep_x(X)
        Yt = t.as_tensor(Y, dtype=t.float32, device=self.dev)
        yn = (Yt - self.y_mu) / self.y_sd if self.y_mu is not None else Yt
        y, a = self._forward(xb, Mp)
        diff = y[:M, :self.n_out] - yn
        if weight is not None:
            diff = diff * t.as_tensor(weight, dtype=t.float32, device=self.dev)[:, None]
        count = M * self.n_out
        loss = (diff * diff).sum() / count
        dy = t.zeros(Mp, 64, device=self.dev)
        dy[:M, :self.n_out] = 2.0 * diff / count
        dyb = dy.to(t.bfloat16).contiguous()
        dybt = dyb[:, :self.n_out_p].t().contiguous()          # [n_out_p][Mp]
        W = self.width
        gW, gb = [None] * 4, [None] * 4
        # output layer: dW4^T[W][n_out_p] = H3^T . dY  (A = H3^T [W][Mp], B = dY^T [n_out_p][Mp])
        g4t = t.empty(W, self.n_out_p, device=self.dev)
        self._gemm(a["H3t"], dybt, W, self.n_out_p, Mp, EPI_SPLIT, 32, g4t)
        gW[3] = g4t.t().contiguous()
        gb[3] = dy[:, :self.n_out_p].sum(0)
        dz = dyb
        wt = self.Wtb[3]
        for k in (2, 1, 0):                      # layer k+1 (1-based)
            dzb = t.empty(Mp, W, device=self.dev, dtype=t.bfloat16)
            dzbt = t.empty(W, Mp, device=self.dev, dtype=t.bfloat16)
            self._gemm(dz, wt, Mp, W, dz.shape[1], EPI_GELU_GRAD, self.bn_hidden, None, dzb, dzbt, W, Mp,
                       zin=a[f"Z{k + 1}"])
            kin = self.k_in if k == 0 else W
            g = t.empty(W, kin, device=self.dev)
            self._gemm(dzbt, a[f"H{k}t"], W, kin, Mp, EPI_SPLIT, 64 if kin == 64 else 128, g)
            gW[k], gb[k] = g, dzb.float().sum(0)
            dz, wt = dzb, self.Wtb[k]
        return loss, gW, gb

    def adam_step(self, gW, gb, lr=None, b1=0.9, b2=0.999, eps=1e-8):
        t = self.torch
        lr = self.lr if lr is None else lr
        self.step_n += 1
        params = self.W + self.b
        grads = gW + gb
        c1, c2 = 1 - b1 ** self.step_n, 1 - b2 ** self.step_n
        for p, g, m, v in zip(params, grads, self.m, self.v):
            m.mul_(b1).add_(g, alpha=1 - b1)
            v.mul_(b2).addcmul_(g, g, value=1 - b2)
            p.addcdiv_(m / c1, (v / c2).sqrt_().add_(eps), value=-lr)
        self.W[0][:, self.n_in:] = 0.0
        self.W[3][self.n_out:, :] = 0.0
        self.b[3][self.n_out:] = 0.0
        self._refresh()

    def train(self, X, Y, epochs: int = 10, batch: int = 4096, lr: float | None = None, seed: int = 0,
              X_val=None, Y_val=None) -> list[float]:
        """Minibatch Adam; returns the mean training loss per epoch (and sets
        self.val_loss when a validation set is given)."""
        t = self.torch
        X = t.as_tensor(X, dtype=t.float32, device=self.dev)
        Y = t.as_tensor(Y, dtype=t.float32, device=self.dev)
        if self.x_mu is None:
            self.fit_stats(X, Y)
        g = t.Generator(device="cpu").manual_seed(seed)
        hist = []
        for ep in range(epochs):
            perm = t.randperm(X.shape[0], generator=g).to(self.dev)
            tot, nb = 0.0, 0
            for i in range(0, X.shape[0], batch):
                idx = perm[i:i + batch]
                loss, gW, gb = self.loss_and_grads(X[idx], Y[idx])
                self.adam_step(gW, gb, lr)
                tot += float(loss)
                nb += 1
            hist.append(tot / max(nb, 1))
        if X_val is not None:
            self.val_loss = float(self.loss_and_grads(X_val, Y_val)[0])
        return hist
