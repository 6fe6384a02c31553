"""Array namespace of an initial-condition evaluation (host set-up code).

The library's initial conditions, `compute_conservatives` and `fv_average`
are written against `of(x)`: numpy for host arrays, and for torch tensors a
shim that gives torch the numpy names and conventions those functions use
(scalars promoted to float64, integer masks, value lookups from small host
tables). The same code then evaluates an initial condition on the host (the
reference's path, bit for bit) or on the device (`EulerSolver(ic_on_device=
True)`), where only the transcendental functions (sin, exp) may differ from
numpy's in the last unit of precision.
"""

import numpy as np


class _Numpy:
    pi = np.pi
    where = staticmethod(np.where)
    sin = staticmethod(np.sin)
    exp = staticmethod(np.exp)
    abs = staticmethod(np.abs)
    square = staticmethod(np.square)
    floor = staticmethod(np.floor)
    clip = staticmethod(np.clip)
    zeros_like = staticmethod(np.zeros_like)
    empty_like = staticmethod(np.empty_like)

    @staticmethod
    def div(a, b):
        return a / b

    @staticmethod
    def empty(shape, like):
        return np.empty(shape)

    @staticmethod
    def mask_like(x):
        """An all-true boolean mask of x's shape."""
        return np.ones_like(x, dtype=bool)

    @staticmethod
    def asint(x):
        return x.astype(int)

    @staticmethod
    def lookup(table, index, cache=None):
        """table[index] for a host table and an index array (or tuple of them);
        cache (a dict the caller owns) keeps device copies of the table."""
        return np.asarray(table)[index]

    @staticmethod
    def diff_mean(c, axis):
        return np.mean(np.diff(c, axis=axis))

    @staticmethod
    def asarray(a, like):
        return np.asarray(a, dtype=np.float64)


class _Torch:
    pi = np.pi

    def __init__(self):
        import torch

        self.torch = torch

    def _t(self, a, like):
        if isinstance(a, self.torch.Tensor):
            return a
        return self.torch.as_tensor(a, dtype=self.torch.float64, device=like.device)

    def div(self, a, b):
        # a device 0-d divisor keeps torch on its IEEE division (a host scalar
        # divisor is applied as a multiplication by its reciprocal)
        if not isinstance(b, self.torch.Tensor):
            b = self.torch.full((), float(b), dtype=self.torch.float64, device=a.device)
        return a / b

    def where(self, c, a, b):
        return self.torch.where(c, self._t(a, c), self._t(b, c))

    def sin(self, x):
        return self.torch.sin(x)

    def exp(self, x):
        return self.torch.exp(x)

    def abs(self, x):
        return self.torch.abs(x)

    def square(self, x):
        return self.torch.square(x)

    def floor(self, x):
        return self.torch.floor(x)

    def clip(self, x, lo, hi):
        return self.torch.clamp(x, lo, hi)

    def zeros_like(self, x):
        return self.torch.zeros_like(x)

    def empty_like(self, x):
        return self.torch.empty_like(x)

    def empty(self, shape, like):
        return self.torch.empty(tuple(shape), dtype=self.torch.float64, device=like.device)

    def mask_like(self, x):
        return self.torch.ones_like(x, dtype=self.torch.bool)

    def asint(self, x):
        return x.long()

    def lookup(self, table, index, cache=None):
        # the device copy lives in the caller's cache (an initial condition's
        # closure), so it is freed with the solver that holds that closure
        dev = index[0].device if isinstance(index, tuple) else index.device
        t = cache.get(dev) if cache is not None else None
        if t is None:
            t = self.torch.as_tensor(np.asarray(table), device=dev)
            if cache is not None:
                cache[dev] = t
        return t[index]

    def diff_mean(self, c, axis):
        # numpy's own reduction on the host copy, so the value equals the host path's
        return np.mean(np.diff(c.detach().cpu().numpy(), axis=axis))

    def asarray(self, a, like):
        return self._t(np.asarray(a, dtype=np.float64), like)


_NUMPY = _Numpy()
_TORCH = None


def of(x):
    """The namespace of array x: the torch shim for torch tensors, numpy otherwise."""
    global _TORCH
    if type(x).__module__.startswith("torch"):
        if _TORCH is None:
            _TORCH = _Torch()
        return _TORCH
    return _NUMPY
