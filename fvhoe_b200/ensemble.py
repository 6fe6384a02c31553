"""Batched ensemble of independent 2D problems (libfvh.so, fvh_ensemble_*).

The reference advances one problem per `EulerSolver` (fvhoe/solver.py,
fvhoe/ode.py:94-174). `Ensemble` advances many problems that share every
solver setting except the grid and the initial condition: each SSP-RK3 stage
of every active member runs in one cooperative persistent launch over a work
list of (member, tile) entries, a whole step is replayed from a CUDA graph,
and the tile shape and resident blocks per SM come from an autotuner that
times the candidates on the ensemble's own data. Each member takes its own
CFL dt clamped to the common target and stops when it reaches it, as
`EulerSolver.ssprk3(t_end)` does; in FP64 a member's result equals that of the
same problem run alone, bit for bit.
"""

import ctypes
import os
import sys
from typing import Dict, Sequence

import numpy as np

__all__ = ["Ensemble"]


class Ensemble:
    """members: dicts with `w0` (initial condition), `nx`, `ny` and optionally
    `x`, `y` (domains), `conservative_ic`, `fv_ic`. The keyword arguments are
    EulerSolver's (2D: px = py), shared by every member."""

    def __init__(self, members: Sequence[Dict], px: int = 3, precision: str = "fp32", device: int = 0,
                 use_graph: bool = True, **solver_kwargs):
        import torch

        from . import _capi
        from .solver import EulerSolver, initial_state

        self._capi = _capi
        self.device = torch.device("cuda", device)
        self.members = [dict(m) for m in members]
        if not self.members:
            raise ValueError("an ensemble needs at least one member")
        for m in self.members:
            m.setdefault("x", (0, 1))
            m.setdefault("y", (0, 1))
        kw = dict(solver_kwargs)
        for key in ("w0", "nx", "ny", "nz", "px", "py", "pz", "x", "y", "z", "precision", "progress_bar",
                    "log_troubles", "kernel_path"):
            kw.pop(key, None)
        # the shared settings, validated and encoded exactly as EulerSolver does
        with torch.cuda.device(self.device):
            side = 32
            template = EulerSolver(nx=side, ny=side, px=px, py=px, precision=precision, progress_bar=False,
                                   log_troubles=False, kernel_path="fused2d", **kw)
            cfg = template._cfg
            del template
        self.gamma = kw.get("gamma", 5 / 3)
        self.px = px
        self.precision = precision
        n = len(self.members)
        nx = (ctypes.c_int * n)(*[int(m["nx"]) for m in self.members])
        ny = (ctypes.c_int * n)(*[int(m["ny"]) for m in self.members])
        hx = (ctypes.c_double * n)(*[(m["x"][1] - m["x"][0]) / m["nx"] for m in self.members])
        hy = (ctypes.c_double * n)(*[(m["y"][1] - m["y"][0]) / m["ny"] for m in self.members])
        handle = ctypes.c_void_p()
        st = _capi.lib.fvh_ensemble_create(ctypes.byref(cfg), n, nx, ny, hx, hy, ctypes.byref(handle))
        if st != _capi.OK:
            raise _capi.FvhError(st, (_capi.lib.fvh_ensemble_last_error(None) or b"").decode())
        self._e = handle
        self.cells = np.array([int(m["nx"]) * int(m["ny"]) for m in self.members], dtype=np.int64)

        def build(m):
            return initial_state(m["w0"], int(m["nx"]), int(m["ny"]), 1, px, px, 0, m["x"], m["y"], (0, 1),
                                 gamma=self.gamma, conservative_ic=m.get("conservative_ic", False),
                                 fv_ic=m.get("fv_ic", False))

        # initial states on the host cores (NumPy releases the GIL in its array loops)
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as pool:
            for q, u0 in enumerate(pool.map(build, self.members)):
                self._check(_capi.lib.fvh_ensemble_load(self._e, q, u0.ctypes.data_as(ctypes.c_void_p), None))
        self._check(_capi.lib.fvh_ensemble_configure(self._e, 0 if precision == "fp32" else 1, 0, int(use_graph)))
        self.t_end = None

    def __del__(self):
        e = getattr(self, "_e", None)
        # at interpreter exit the CUDA runtime may already be torn down; the process frees everything
        if e and not sys.is_finalizing():
            self._capi.lib.fvh_ensemble_destroy(e)
            self._e = None

    def _check(self, st):
        if st != self._capi.OK:
            raise self._capi.FvhError(st, (self._capi.lib.fvh_ensemble_last_error(self._e) or b"").decode())

    def _stream(self):
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def __len__(self):
        return len(self.members)

    # -- stepping ------------------------------------------------------------
    def reset(self, t_end: float, t0: float = 0.0):
        """Every member to time t0, aiming at t_end."""
        self.t_end = float(t_end)
        self._check(self._capi.lib.fvh_ensemble_reset(self._e, float(t0), float(t_end), self._stream()))

    def step(self, n: int = 1):
        """n SSP-RK3 steps of every active member (asynchronous)."""
        self._check(self._capi.lib.fvh_ensemble_step(self._e, int(n), self._stream()))

    def set_wait_limit(self, polls: int = 0):
        """Bound of the grid-barrier waits in polls (0: the default, 2^24); a wait
        that runs out ends the stage and status() then raises FVH_ERR_TIMEOUT
        until the next reset."""
        self._check(self._capi.lib.fvh_ensemble_set_wait_limit(self._e, int(polls)))

    def status(self) -> dict:
        n = len(self.members)
        t = (ctypes.c_double * n)()
        steps = (ctypes.c_int * n)()
        active = ctypes.c_int()
        bad = ctypes.c_uint()
        self._check(self._capi.lib.fvh_ensemble_status(self._e, t, steps, ctypes.byref(active), ctypes.byref(bad),
                                                       self._stream()))
        steps = np.array(steps[:], dtype=np.int64)
        return dict(t=np.array(t[:]), steps=steps, active=int(active.value), nonfinite=int(bad.value),
                    cell_updates=int(3 * np.sum(steps * self.cells)))

    def run(self, t_end: float, check_every: int = 8, max_steps: int = 10 ** 7) -> dict:
        """Advances every member to t_end; returns the final status."""
        self.reset(t_end)
        taken = 0
        while taken < max_steps:
            self.step(check_every)
            taken += check_every
            st = self.status()
            if st["active"] == 0:
                return st
        raise RuntimeError("ensemble did not reach its target within max_steps")

    # -- tuning --------------------------------------------------------------
    def configure(self, variant: int, blocks_per_sm: int = 0, use_graph: bool = True):
        self._check(self._capi.lib.fvh_ensemble_configure(self._e, int(variant), int(blocks_per_sm), int(use_graph)))

    def variants(self) -> list:
        out = []
        for v in range(3):
            tx, ty, mb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            smem = ctypes.c_size_t()
            self._check(self._capi.lib.fvh_ensemble_variant_info(self._e, v, ctypes.byref(tx), ctypes.byref(ty),
                                                                 ctypes.byref(mb), ctypes.byref(smem)))
            out.append(dict(variant=v, tile=(tx.value, ty.value), max_blocks_per_sm=mb.value,
                            smem_bytes=smem.value))
        return out

    def autotune(self, steps: int = 2) -> dict:
        """Times every tile variant and block count on this ensemble (states are
        put back afterwards) and keeps the fastest."""
        v, b, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self._capi.lib.fvh_ensemble_autotune(self._e, int(steps), ctypes.byref(v), ctypes.byref(b),
                                                         ctypes.byref(ms), self._stream()))
        return dict(variant=v.value, tile=self.variants()[v.value]["tile"], blocks_per_sm=b.value,
                    ms_per_step=ms.value)

    def graph_info(self) -> dict:
        used = ctypes.c_int()
        err = ctypes.c_char_p()
        self._check(self._capi.lib.fvh_ensemble_graph_info(self._e, ctypes.byref(used), ctypes.byref(err)))
        return dict(graph=bool(used.value), error=(err.value or b"").decode())

    # -- data ----------------------------------------------------------------
    def state(self, q: int) -> np.ndarray:
        """Member q's conserved state (5, nx, ny, 1) as a NumPy array."""
        m = self.members[q]
        out = np.empty((5, int(m["nx"]), int(m["ny"]), 1), dtype=np.float64)
        self._check(self._capi.lib.fvh_ensemble_store(self._e, q, out.ctypes.data_as(ctypes.c_void_p),
                                                      self._stream()))
        return out

    def nbytes(self) -> int:
        return int(self._capi.lib.fvh_ensemble_bytes(self._e))
