"""Time-integration driver (host side).

Same interface as fvhoe/ode.py:25-298 (`ODE`): integrate(T, n, exact,
downbeats, log_every_step, snapshot_dir, overwrite) and the steppers euler,
ssprk2, ssprk3 and rk4, each of which records its name and integrates. The
loop, the downbeat bookkeeping and the snapshot cadence are the reference's;
one step is a single call into the CUDA library (`_device_step`), which runs
all stages of the chosen integrator on the device and returns the step's dt
(shortened to the next downbeat when `exact`, fvhoe/ode.py:11-22).
"""

import math
import os
from abc import ABC, abstractmethod
from typing import Any, Optional

import numpy as np

from .timer import Timer


def _hit_target(t: float, dt: float, target: float = None) -> float:
    """dt shortened so that t + dt does not pass target (fvhoe/ode.py:11-22)."""
    if target is not None and target - t < dt:
        return target - t
    return dt


class SnapshotList(list):
    """The snapshot list (a plain list of dicts in the reference). Snapshots may
    be copied to the host asynchronously; every read of the list first calls
    settle(), which waits for the copies still in flight and completes their
    entries, so a reader always sees finished arrays. It pickles as a plain list."""

    def __init__(self, settle, items=()):
        super().__init__(items)
        self._settle = settle

    def __getitem__(self, i):
        self._settle()
        return super().__getitem__(i)

    def __iter__(self):
        self._settle()
        return super().__iter__()

    def __reversed__(self):
        self._settle()
        return super().__reversed__()

    def __contains__(self, x):
        self._settle()
        return super().__contains__(x)

    def __eq__(self, other):
        self._settle()
        return list.__eq__(self, other)

    __hash__ = None

    def __repr__(self):
        self._settle()
        return super().__repr__()

    def copy(self):
        self._settle()
        return list(super().__iter__())

    def index(self, *args):
        self._settle()
        return super().index(*args)

    def count(self, x):
        self._settle()
        return super().count(x)

    def pop(self, *args):
        self._settle()
        return super().pop(*args)

    def remove(self, x):
        self._settle()
        return super().remove(x)

    def __reduce_ex__(self, protocol):
        self._settle()
        return (list, (list(super().__iter__()),))


class ODE(ABC):
    def _ode_init(self, progress_bar: bool = True):
        self.t = 0.0
        self.timestamps = [0.0]
        self.step_count = 0
        self.timer = Timer(cats=["TOTAL", "SNAPSHOTS"])
        self.snapshots = SnapshotList(self._settle_snapshots)
        self.snapshot_times = []
        self.print_progress_bar = bool(progress_bar)
        self.integrator = None

    # -- stepping -----------------------------------------------------------
    @abstractmethod
    def _device_step(self, integrator: str, target_time: Optional[float]) -> float:
        """Advance am("u") by one step in place and return dt."""

    @abstractmethod
    def f(self, t: float, u) -> tuple:
        """(dt, dudt) of one right-hand-side evaluation."""

    def take_step(self, target_time: float = None):
        # a failed update raises from _device_step (FVH_ERR_NONFINITE); a step
        # that cannot advance the time is refused here, so integrate(T) never
        # spins on a frozen t (the reference's loop, fvhoe/ode.py:157, would)
        dt = self._device_step(self.integrator, target_time)
        if not (math.isfinite(dt) and dt > 0.0):
            raise FloatingPointError(f"step {self.step_count + 1} at t={self.t!r}: dt={dt!r} is not a finite "
                                     "positive time step")
        if self.t + dt == self.t:
            raise FloatingPointError(f"step {self.step_count + 1} at t={self.t!r}: dt={dt!r} does not advance t")
        self.t += dt
        self.timestamps.append(self.t)
        self.step_count += 1
        self.step_helper_function()

    def step_helper_function(self):
        pass

    def snapshot(self):
        self.snapshots.append(None)
        self.snapshot_times.append(self.t)

    def _settle_snapshots(self):
        """Completes snapshots whose host copies are still in flight (none here)."""

    def read_snapshots(self) -> bool:
        return False

    def write_snapshots(self, overwrite: bool = False):
        pass

    # -- driver (fvhoe/ode.py:94-174) ------------------------------------------
    def integrate(self, T: float = None, n: int = None, exact: bool = True, downbeats: Any = None,
                  log_every_step: bool = False, snapshot_dir: str = None, overwrite: bool = False) -> None:
        if T is None:
            self.timer.start("SNAPSHOTS")
            self.snapshot()
            self.timer.stop("SNAPSHOTS")
            self.timer.start("TOTAL")
            for _ in self._progress(range(n)):
                self.take_step()
            self.timer.stop("TOTAL")
            self.timer.start("SNAPSHOTS")
            self.snapshot()
            self.timer.stop("SNAPSHOTS")
            return
        save = snapshot_dir is not None
        if save:
            self.snapshot_dir = os.path.normpath(snapshot_dir)
            if not overwrite and self.read_snapshots():
                return
        bar = self._bar(T)
        if downbeats is None:
            downbeats = []
        elif isinstance(downbeats, np.ndarray):
            downbeats = downbeats.tolist()
        downbeats = sorted(set([0] + list(downbeats) + [T]))[1:]
        target_time = downbeats.pop(0) if exact else None
        self.snapshot()
        self.timer.start("TOTAL")
        while self.t < T:
            self.take_step(target_time=target_time)
            if bar is not None:
                bar.n = self.t
                bar.refresh()
            if self.t == target_time or self.t >= T or log_every_step:
                self.timer.start("SNAPSHOTS")
                self.snapshot()
                self.timer.stop("SNAPSHOTS")
                if downbeats and self.t == target_time:
                    target_time = downbeats.pop(0)
        self.timer.stop("TOTAL")
        if bar is not None:
            bar.close()
        if save:
            self.write_snapshots(overwrite)

    def _progress(self, it):
        if not self.print_progress_bar:
            return it
        from tqdm import tqdm

        return tqdm(it)

    def _bar(self, T):
        if not self.print_progress_bar:
            return None
        from tqdm import tqdm

        return tqdm(total=T, bar_format="{l_bar}{bar}| {n_fmt}/{total_fmt} [{elapsed}]")

    # -- steppers (fvhoe/ode.py:245-298) ------------------------------------------
    def euler(self, *args, **kwargs) -> None:
        self.integrator = "euler"
        self.integrate(*args, **kwargs)

    def ssprk2(self, *args, **kwargs) -> None:
        self.integrator = "ssprk2"
        self.integrate(*args, **kwargs)

    def ssprk3(self, *args, **kwargs) -> None:
        self.integrator = "ssprk3"
        self.integrate(*args, **kwargs)

    def rk4(self, *args, **kwargs) -> None:
        self.integrator = "rk4"
        self.integrate(*args, **kwargs)
