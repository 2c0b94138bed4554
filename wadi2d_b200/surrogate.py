"""The storm-sweep surrogate: a small fully connected network, 16 -> 256 -> 256 -> 256 -> 16 with ReLU between, that
maps a storm's descriptors to the peak flow and time to peak at the design points. It is trained and run on the
device by this package's own kernels: every product on the tensor cores (w2b_mma_gemm: BF16 operands, FP32
accumulation), the activations and their gradients, transposes, the loss gradient, bias sums and Adam element-wise.

Numbers: FP32 master weights, BF16 copies for the products; activations stored in BF16 between layers, the
pre-activations in FP32; gradients w.r.t. pre-activations rounded to BF16 before their products; bias gradients and
Adam in FP32. Inputs and targets are standardised by the caller's statistics (``Scaler``).
"""

from __future__ import annotations

import gc
from dataclasses import dataclass

import numpy as np

from wadi2d_b200 import _lib

DIMS = (16, 256, 256, 256, 16)


def _pad16(n: int) -> int:
    return (n + 15) // 16 * 16


@dataclass
class Scaler:
    """Per-column standardisation: (x - mean) / std."""

    mean: np.ndarray
    std: np.ndarray

    @classmethod
    def fit(cls, x: np.ndarray) -> Scaler:
        x = np.asarray(x, np.float64)
        return cls(x.mean(0), np.where(x.std(0) > 1e-12, x.std(0), 1.0))

    def to(self, x):
        return (np.asarray(x, np.float64) - self.mean) / self.std

    def back(self, z):
        return np.asarray(z, np.float64) * self.std + self.mean


class Network:
    """The network's weights on the device and its forward pass, gradients and Adam steps."""

    def __init__(self, dims=DIMS, seed: int = 0, device="cuda", lr: float = 1e-3) -> None:
        import torch

        self.torch = torch
        self.dims = tuple(int(d) for d in dims)
        for d in self.dims[1:]:
            if d % 16 or not 16 <= d <= 256:
                raise ValueError("layer widths must be multiples of 16 between 16 and 256")
        if self.dims[0] % 16:
            raise ValueError("the input width must be a multiple of 16")
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        dev = self.device
        self.W, self.b, self.Wb, self.Wt = [], [], [], []
        self.mW, self.vW, self.mb, self.vb = [], [], [], []
        for fan_in, fan_out in zip(self.dims[:-1], self.dims[1:], strict=True):
            w = rng.standard_normal((fan_out, fan_in)) * np.sqrt(2.0 / fan_in)  # He initialisation
            self.W.append(torch.as_tensor(w, dtype=torch.float32, device=dev))
            self.b.append(torch.zeros(fan_out, dtype=torch.float32, device=dev))
            self.Wb.append(torch.empty((fan_out, fan_in), dtype=torch.bfloat16, device=dev))
            self.Wt.append(torch.empty((fan_in, fan_out), dtype=torch.bfloat16, device=dev))
            for lst, shape in ((self.mW, (fan_out, fan_in)), (self.vW, (fan_out, fan_in)), (self.mb, (fan_out,)),
                               (self.vb, (fan_out,))):  # fmt: skip
                lst.append(torch.zeros(shape, dtype=torch.float32, device=dev))
        for i in range(len(self.W)):
            self._sync(i)
        self.lr = lr
        self.t = 0
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.partial = torch.zeros(64, dtype=torch.float64, device=dev)

    # ------------------------------------------------------------------ plumbing

    def _s(self) -> int:
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def _sync(self, i: int) -> None:
        """The BF16 copy of layer i's weights and its transpose."""
        W = self.W[i]
        _lib.call("w2b_bf16_act", W.data_ptr(), W.numel(), 0, self.Wb[i].data_ptr(), self._s())
        out, inp = W.shape
        _lib.call("w2b_transpose_bf16", self.Wb[i].data_ptr(), out, inp, out, self.Wt[i].data_ptr(), self._s())

    def _gemm(self, a, b, m: int, n: int, k: int, bias=None):
        c = self.torch.empty((m, n), dtype=self.torch.float32, device=self.device)
        _lib.call("w2b_mma_gemm", a.data_ptr(), b.data_ptr(), m, n, k, None if bias is None else bias.data_ptr(),
                  c.data_ptr(), self.status.data_ptr(), self._s())  # fmt: skip
        return c

    def _bf16(self, z, relu: bool):
        out = self.torch.empty(z.shape, dtype=self.torch.bfloat16, device=self.device)
        _lib.call("w2b_bf16_act", z.data_ptr(), z.numel(), int(relu), out.data_ptr(), self._s())
        return out

    def _t(self, x, rows: int, cols: int):
        out = self.torch.empty((cols, rows), dtype=self.torch.bfloat16, device=self.device)
        _lib.call("w2b_transpose_bf16", x.data_ptr(), rows, cols, rows, out.data_ptr(), self._s())
        return out

    def _input(self, x):
        """Standardised inputs (host array, or FP32 on the device) padded to 16 rows and cast to BF16."""
        torch = self.torch
        if not (isinstance(x, torch.Tensor) and x.is_cuda):
            x = torch.as_tensor(np.asarray(x, np.float32), device=self.device)
        n = x.shape[0]
        npad = _pad16(max(n, 1))
        xp = torch.zeros((npad, self.dims[0]), dtype=torch.float32, device=self.device)
        xp[:n] = x
        return n, npad, self._bf16(xp, False)

    # ------------------------------------------------------------------ passes

    def forward(self, x, keep: bool = False):
        """Outputs (n x dims[-1], FP32 on the device) of standardised inputs x; with ``keep``, also the layers'
        inputs (BF16) and pre-activations (FP32) for the backward pass."""
        n, npad, h = self._input(x)
        hs, zs = [h], []
        L = len(self.W)
        for i in range(L):
            out, inp = self.W[i].shape
            z = self._gemm(h, self.Wb[i], npad, out, inp, self.b[i])
            zs.append(z)
            if i < L - 1:
                h = self._bf16(z, True)
                hs.append(h)
        if keep:
            return zs[-1][:n], (n, npad, hs, zs)
        return zs[-1][:n]

    def gradients(self, x, t):
        """Mean-square error of the standardised targets t and the gradients of the weights and biases (FP32)."""
        torch = self.torch
        y, (n, npad, hs, zs) = self.forward(x, keep=True)
        tt = torch.zeros((npad, self.dims[-1]), dtype=torch.float32, device=self.device)
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            t = torch.as_tensor(np.asarray(t, np.float32), device=self.device)
        tt[:n] = t
        yp = zs[-1]
        nout = self.dims[-1]
        dz = torch.empty((npad, nout), dtype=torch.bfloat16, device=self.device)
        scale = 2.0 / (n * nout)
        _lib.call("w2b_mse_grad", yp.data_ptr(), tt.data_ptr(), n, npad, nout, float(scale), dz.data_ptr(),
                  self.partial.data_ptr(), self._s())  # fmt: skip
        loss = self.partial.sum() / (n * nout)
        gW, gb = [None] * len(self.W), [None] * len(self.W)
        for i in range(len(self.W) - 1, -1, -1):
            out, inp = self.W[i].shape
            dzt = self._t(dz, npad, out)  # out x npad
            ht = self._t(hs[i], npad, inp)  # inp x npad
            gW[i] = self._gemm(dzt, ht, out, inp, npad)
            gb[i] = torch.empty(out, dtype=torch.float32, device=self.device)
            _lib.call("w2b_colsum_bf16", dz.data_ptr(), npad, out, gb[i].data_ptr(), self._s())
            if i > 0:
                g = self._gemm(dz, self.Wt[i], npad, inp, out)  # npad x inp
                dz = torch.empty((npad, inp), dtype=torch.bfloat16, device=self.device)
                _lib.call("w2b_relu_back", g.data_ptr(), zs[i - 1].data_ptr(), g.numel(), dz.data_ptr(), self._s())
        return loss, gW, gb

    def _lr(self, t: int, b1: float = 0.9, b2: float = 0.999) -> float:
        """Adam's bias-corrected step size at step t."""
        return float(self.lr * np.sqrt(1.0 - b2**t) / (1.0 - b1**t))

    def _adam(self, gW, gb, lr_t: float = 0.0, table=None, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        """Adam on every layer with step size lr_t, or (table) lr_table[*step] read on the device."""
        for i in range(len(self.W)):
            for w, g, m, v in ((self.W[i], gW[i], self.mW[i], self.vW[i]), (self.b[i], gb[i], self.mb[i], self.vb[i])):
                if table is None:
                    _lib.call("w2b_adam", w.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), w.numel(), lr_t, b1,
                              b2, eps, None, self._s())  # fmt: skip
                else:
                    _lib.call("w2b_adam_table", w.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), w.numel(),
                              table[0].data_ptr(), table[1].data_ptr(), b1, b2, eps, None, self._s())  # fmt: skip
            self._sync(i)

    def _check(self) -> None:
        if int(self.status.item()) != 0:
            raise _lib.W2BError(int(self.status.item()), "w2b_mma_gemm")

    def step(self, x, t):
        """One Adam step on the batch (x, t); returns the loss before the step (a device scalar)."""
        loss, gW, gb = self.gradients(x, t)
        self.t += 1
        self._adam(gW, gb, self._lr(self.t))
        self._check()
        return loss

    def fit(self, x, t, iters: int = 2000, batch: int = 256, seed: int = 0, graph: bool = True) -> list[float]:
        """Adam over random batches of (x, t), standardised; returns the loss every 100 steps.

        With ``graph`` (the default) the batches are drawn up front (the same draws, in the same order, as one step
        at a time draws them), the training set goes to the device once, and one step (gather, forward, backward,
        Adam with the step's own size read on the device) is captured as a CUDA graph after a first step run eagerly,
        then replayed: the same kernels on the same data in the same order as stepping from the host, without a host
        round trip a step."""
        rng = np.random.default_rng(seed)
        x, t = np.asarray(x, np.float32), np.asarray(t, np.float32)
        bs = min(batch, x.shape[0])
        draws = [rng.choice(x.shape[0], size=bs, replace=False) for _ in range(iters)]
        if not graph or iters < 2:
            losses = []
            for it in range(iters):
                loss = self.step(x[draws[it]], t[draws[it]])
                if it % 100 == 0 or it == iters - 1:
                    losses.append(float(loss))
            return losses
        torch, dev = self.torch, self.device
        X, T = torch.as_tensor(x, device=dev), torch.as_tensor(t, device=dev)
        idx = torch.as_tensor(np.stack(draws).astype(np.int64), device=dev)
        lr = torch.as_tensor(np.array([self._lr(self.t + s) for s in range(1, iters + 1)], np.float32), device=dev)
        k = torch.zeros(1, dtype=torch.int64, device=dev)
        loss_at = torch.zeros(iters, dtype=torch.float64, device=dev)

        def one() -> None:
            rows = idx.index_select(0, k).view(-1)
            loss, gW, gb = self.gradients(X.index_select(0, rows), T.index_select(0, rows))
            self._adam(gW, gb, table=(lr, k))
            loss_at.index_copy_(0, k, loss.view(1).to(torch.float64))
            k.add_(1)

        one()  # the first step, from the host: every kernel's first launch happens outside the capture
        # A finalizer that frees device memory (a solver backend dropped inside a reference cycle) must not run in the
        # capture, which that call would end: collect first and keep the collector off until the capture is over.
        # Thread-local capture: CUDA calls of other threads do not end it either.
        gc.collect()
        collecting = gc.isenabled()
        gc.disable()
        g = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(g, capture_error_mode="thread_local"):
                one()
        finally:
            if collecting:
                gc.enable()
        for _ in range(iters - 1):
            g.replay()
        self.t += iters
        self._check()
        del g
        out = loss_at.cpu().numpy()
        return [float(out[it]) for it in range(iters) if it % 100 == 0 or it == iters - 1]

    def predict(self, x) -> np.ndarray:
        return self.forward(x).cpu().numpy().astype(np.float64)

    def weights(self) -> list[tuple[np.ndarray, np.ndarray]]:
        return [(w.cpu().numpy().astype(np.float64), b.cpu().numpy().astype(np.float64)) for w, b in zip(self.W, self.b)]
