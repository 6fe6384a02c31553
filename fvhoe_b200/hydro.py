"""Variable map and slicing helper of the Euler state (host side).

Same interface as fvhoe/hydro.py:8-140 (`HydroState`): variable 0 is rho,
1..3 the momentum / velocity components, 4 the energy / pressure, 5.. the
passive scalars; calling the object returns index tuples for NumPy-style
slicing of (nvars, nx, ny, nz) arrays.
"""

from functools import lru_cache
from typing import Tuple, Union

import numpy as np

from .array_ns import of


class HydroState:
    def __init__(self, passive_scalars: tuple = (), ndim: int = 4):
        self.passive_scalars = tuple(passive_scalars)
        self.ndim = ndim
        if len(set(self.passive_scalars)) != len(self.passive_scalars):
            raise ValueError("Duplicate passive scalar names.")
        self.variable_map = {
            "rho": 0,
            "vx": 1,
            "mx": 1,
            "vy": 2,
            "my": 2,
            "vz": 3,
            "mz": 3,
            "v": np.arange(1, 4),
            "m": np.arange(1, 4),
            "P": 4,
            "E": 4,
            "active_scalars": np.arange(0, 5),
        }
        for i, name in enumerate(self.passive_scalars, start=5):
            self.variable_map[name] = i
        self.includes_passives = bool(self.passive_scalars)
        if self.includes_passives:
            self.variable_map["passive_scalars"] = np.arange(5, 5 + len(self.passive_scalars))
        self.nvars = 5 + len(self.passive_scalars)

    def __hash__(self):
        return id(self)

    @lru_cache(maxsize=None)
    def __call__(
        self,
        var: Union[str, Tuple[str, ...]] = None,
        x: Tuple[int, int] = None,
        y: Tuple[int, int] = None,
        z: Tuple[int, int] = None,
        axis: int = None,
        cut: Tuple[int, int] = None,
        step: int = None,
    ):
        """Index tuple selecting `var` and the given (start, stop) ranges."""
        out = [slice(None)] * self.ndim
        if var is not None:
            if isinstance(var, str):
                if var not in self.variable_map:
                    raise ValueError(f"Variable '{var}' not found.")
                out[0] = self.variable_map[var]
            elif isinstance(var, tuple):
                missing = set(var) - set(self.variable_map)
                if missing:
                    raise ValueError(f"Variables not found: {missing}")
                out[0] = np.array([self.variable_map[v] for v in var])
            else:
                raise ValueError(f"Invalid type for var: {type(var)}")
        for i, rng in zip((1, 2, 3, axis), (x, y, z, cut)):
            if rng is None:
                continue
            if i >= self.ndim:
                raise ValueError(f"Invalid axis {i} for array with {self.ndim} dimensions.")
            if not isinstance(rng, tuple) or len(rng) != 2:
                raise ValueError(f"Expected a (start, stop) tuple for axis {i}, got {rng!r}")
            out[i] = slice(rng[0] or None, rng[1] or None, step if i == axis else None)
        if len(out) == 1:
            return out[0]
        return tuple(out)


def compute_conservatives(hs: HydroState, w: np.ndarray, gamma: float) -> np.ndarray:
    """Conversion used to build initial conditions (fvhoe/hydro.py:173-196), for
    host arrays or device tensors (array_ns)."""
    u = of(w).empty_like(w)
    rho = w[0]
    u[0] = rho
    u[1:4] = rho * w[1:4]
    ke = u[1] * w[1]
    ke = ke + u[2] * w[2]
    ke = ke + u[3] * w[3]
    u[4] = of(w).div(w[4], gamma - 1) + 0.5 * ke
    if w.shape[0] > 5:
        u[5:] = rho * w[5:]
    return u


def advection_dt(h: float, vx: float = 0.0, vy: float = 0.0, vz: float = 0.0, CFL: float = 0.8) -> float:
    """CFL step of a pure advection problem (fvhoe/hydro.py:249-267)."""
    return CFL * h / (vx + vy + vz)
