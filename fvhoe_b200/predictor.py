"""Learned troubled-cell predictor: training data, training and evaluation.

The network (100 -> 64 -> 64 -> 1, GELU) and its kernels live in libfvh.so
(fvh_mlp_* in include/fvh.h): the forward and backward passes run on the
tensor cores with BF16 operands and FP32 accumulation, Adam runs on the
device. This module holds the host side: a `TroubledCellPredictor` owning one
network, `collect_training_data` turning solver runs into (features,
a-posteriori flag) rows, and the miss / false-alarm evaluation.

The reference has no learned component; its troubled cells come only from
the a-posteriori check (fvhoe/solver.py:653-732). Attached to an EulerSolver
(`EulerSolver.set_predictor`), the network runs before the high-order fluxes
of each stage, faces next to predicted cells take the fallback flux in the
flux pass, and the a-posteriori check still runs on every cell and revises the
faces of the cells the network missed.
"""

import ctypes
import sys
from typing import Iterable, Optional, Tuple

import numpy as np

from . import _capi

__all__ = ["TroubledCellPredictor", "collect_training_data", "rates"]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(device):
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class TroubledCellPredictor:
    """One network on one CUDA device."""

    n_params = int(_capi.lib.fvh_mlp_param_count())

    def __init__(self, device: int = 0, seed: int = 0):
        import torch

        self.device = torch.device("cuda", device)
        handle = ctypes.c_void_p()
        st = _capi.lib.fvh_mlp_create(int(device), int(seed), ctypes.byref(handle))
        if st != _capi.OK:
            raise _capi.FvhError(st, (_capi.lib.fvh_mlp_last_error(None) or b"").decode())
        self._m = handle
        self.steps = 0

    def __del__(self):
        m = getattr(self, "_m", None)
        # at interpreter exit the CUDA runtime may already be torn down; the process frees everything
        if m and not sys.is_finalizing():
            _capi.lib.fvh_mlp_destroy(m)
            self._m = None

    def _check(self, st):
        if st != _capi.OK:
            raise _capi.FvhError(st, (_capi.lib.fvh_mlp_last_error(self._m) or b"").decode())

    # parameters ---------------------------------------------------------
    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        self._check(_capi.lib.fvh_mlp_get_params(self._m, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                 out.size))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        self._check(_capi.lib.fvh_mlp_set_params(self._m, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size))

    def save(self, path: str) -> None:
        np.savez(path, params=self.get_params())

    def load(self, path: str) -> None:
        with np.load(path) as d:
            self.set_params(d["params"])

    # kernels --------------------------------------------------------------
    def _rows(self, X, y=None):
        import torch

        if X.dtype != torch.bfloat16 or X.dim() != 2 or X.shape[1] != _capi.MLP_ROW or not X.is_contiguous():
            raise ValueError(f"X must be a contiguous (n, {_capi.MLP_ROW}) bfloat16 CUDA tensor")
        if y is not None and (y.dtype != torch.uint8 or y.shape != (X.shape[0],)):
            raise ValueError("y must be a uint8 CUDA tensor with one flag per row")
        return int(X.shape[0])

    def logits(self, X):
        import torch

        n = self._rows(X)
        out = torch.empty(n, dtype=torch.float32, device=X.device)
        self._check(_capi.lib.fvh_mlp_logits(self._m, _ptr(X), n, _ptr(out), _stream(X.device)))
        return out

    def gradients(self, X, y, pos_weight: float = 1.0) -> Tuple[np.ndarray, float]:
        import torch

        n = self._rows(X, y)
        g = torch.empty(self.n_params, dtype=torch.float32, device=X.device)
        loss = ctypes.c_float()
        self._check(_capi.lib.fvh_mlp_gradients(self._m, _ptr(X), _ptr(y), n, float(pos_weight), _ptr(g),
                                                ctypes.byref(loss), _stream(X.device)))
        return g.cpu().numpy(), float(loss.value)

    def train_step(self, X, y, lr: float, pos_weight: float = 1.0, want_loss: bool = False) -> Optional[float]:
        n = self._rows(X, y)
        loss = ctypes.c_float()
        self._check(_capi.lib.fvh_mlp_train_step(self._m, _ptr(X), _ptr(y), n, float(lr), float(pos_weight),
                                                 ctypes.byref(loss) if want_loss else None, _stream(X.device)))
        self.steps += 1
        return float(loss.value) if want_loss else None

    def fit(self, X, y, epochs: int = 2, batch: int = 65536, lr: float = 2e-3, pos_weight: Optional[float] = None,
            seed: int = 0, lr_decay: float = 0.5):
        """Mini-batch Adam over (X, y); returns the mean loss of each epoch.

        pos_weight defaults to the negative/positive ratio of y (at most 10)."""
        import torch

        n = self._rows(X, y)
        if pos_weight is None:
            pos = float(y.sum().item())
            pos_weight = float(min(10.0, max(1.0, (n - pos) / max(pos, 1.0))))
        gen = torch.Generator(device=X.device)
        gen.manual_seed(seed)
        history = []
        for e in range(epochs):
            perm = torch.randperm(n, device=X.device, generator=gen)
            losses = []
            for i, k in enumerate(range(0, n - batch + 1 if n >= batch else 1, batch)):
                idx = perm[k:k + batch]
                loss = self.train_step(X[idx].contiguous(), y[idx].contiguous(), lr, pos_weight,
                                       want_loss=(i % 16 == 0))
                if loss is not None:
                    losses.append(loss)
            history.append(float(np.mean(losses)) if losses else float("nan"))
            lr *= lr_decay
        self.pos_weight = pos_weight
        return history

    def evaluate(self, X, y, threshold: float = 0.5) -> dict:
        logit_thr = float(np.log(threshold / (1.0 - threshold)))
        pred = self.logits(X) > logit_thr
        return rates(pred, y.bool())

    def errors(self) -> int:
        """Tensor-core waits that reached their bound (0 when healthy)."""
        return int(_capi.lib.fvh_mlp_errors(self._m))


def rates(pred, truth) -> dict:
    """Miss rate (troubled cells not predicted / troubled) and false-alarm rate
    (predicted cells not troubled / untroubled) of boolean tensors or arrays."""
    pred = np.asarray(pred.cpu() if hasattr(pred, "cpu") else pred, dtype=bool).ravel()
    truth = np.asarray(truth.cpu() if hasattr(truth, "cpu") else truth, dtype=bool).ravel()
    t = int(truth.sum())
    f = int(truth.size - t)
    missed = int((truth & ~pred).sum())
    false_alarm = int((pred & ~truth).sum())
    return dict(cells=int(truth.size), troubled=t, predicted=int(pred.sum()), missed=missed,
                false_alarm=false_alarm, miss_rate=missed / t if t else 0.0,
                false_alarm_rate=false_alarm / f if f else 0.0)


def collect_training_data(solvers: Iterable, steps: int, every: int = 1, integrator: str = "ssprk3"):
    """(X, y) rows from solver runs: before every `every`-th step of each run,
    one right-hand-side evaluation of the current state yields the features
    and the a-posteriori flags of all cells. Solvers must run the fused 2D path
    with a-posteriori limiting and global NAD."""
    import torch

    xs, ys = [], []
    for s in solvers:
        ncell = int(np.prod(s.n))
        for k in range(steps):
            if k % every == 0:
                u = s.am("u")
                s.f(s.t, u)
                X = torch.empty((ncell, _capi.MLP_ROW), dtype=torch.bfloat16, device=u.device)
                y = torch.empty(ncell, dtype=torch.uint8, device=u.device)
                _capi.check(_capi.lib.fvh_mlp_features(s._handle, _ptr(X), _ptr(y), s._stream()), s._handle)
                xs.append(X)
                ys.append(y)
            getattr(s, integrator)(n=1)
    return torch.cat(xs), torch.cat(ys)
