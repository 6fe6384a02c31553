"""Initial conditions (host, set-up only).

`InitialCondition` has the interface of fvhoe/initial_conditions.py:11-81:
subclasses implement base_ic(...) returning f(x, y, z) -> (5, ...) primitive
(or, with conservative_ic/fv_ic, conservative) values; build_ic appends the
passive scalars. Any object with the same build_ic method, including the
reference's own classes, can be handed to EulerSolver.

Besides the reference's standard problems, two set-ups of the benchmark
configurations live here: the Kelvin-Helmholtz band with seeded per-cell
noise, and the four-quadrant 2D Riemann problem.
"""

from abc import ABC, abstractmethod
from numbers import Number
from typing import Callable, Dict, Sequence, Tuple

import numpy as np

from .array_ns import of


class InitialCondition(ABC):
    def __init__(self, *args, **kwargs):
        self.args = args
        self.kwargs = kwargs

    @abstractmethod
    def base_ic(self, *args, **kwargs) -> Callable:
        """Returns f(x, y, z) producing a (5, nx, ny, nz) array."""

    def build_ic(self, hs, passive_ic_funcs: Dict[str, Callable] = None) -> Callable:
        if hs.includes_passives:
            missing = set(hs.passive_scalars) - set((passive_ic_funcs or {}).keys())
            if missing:
                raise ValueError(f"Missing IC definitions for passive scalars: {missing}")
        core = self.base_ic(*self.args, **self.kwargs)

        def ic_func(x, y, z):
            out = of(x).empty((5 + len(hs.passive_scalars),) + tuple(np.shape(x)), like=x)
            out[:5] = core(x, y, z)
            for name in hs.passive_scalars:
                out[hs.variable_map[name]] = passive_ic_funcs[name](x, y, z)
            return out

        return ic_func


def _state(like, rho, vx, vy, vz, P):
    """(5,) + like.shape primitive state in like's namespace."""
    out = of(like).empty((5,) + tuple(like.shape), like=like)
    out[0], out[1], out[2], out[3], out[4] = rho, vx, vy, vz, P
    return out


class Sinus(InitialCondition):
    """rho = rho_min + (rho_max - rho_min)(sin(2 pi r)/2 + 1/2), r = sum of the listed coordinates."""

    def base_ic(self, dims="x", rho_min_max=(1, 2), P=1, vx=1, vy=0, vz=0):
        def f(x, y=None, z=None):
            xp = of(x)
            r = xp.zeros_like(x)
            for d, c in zip("xyz", (x, y, z)):
                r = r + (c if d in dims else 0)
            lo, span = rho_min_max[0], rho_min_max[1] - rho_min_max[0]
            return _state(r, span * (0.5 * xp.sin(2 * xp.pi * r) + 0.5) + lo, vx, vy, vz, P)

        return f


class Square(InitialCondition):
    """rho_max inside (0.25, 0.75) along every listed axis, rho_min outside."""

    def base_ic(self, dims="x", rho_min_max=(1, 2), P=1, vx=1, vy=0, vz=0):
        def f(x, y=None, z=None):
            xp = of(x)
            inside = xp.mask_like(x)
            for d, c in zip("xyz", (x, y, z)):
                if d in dims:
                    inside &= (c > 0.25) & (c < 0.75)
            return _state(x, xp.where(inside, rho_min_max[1], rho_min_max[0]), vx, vy, vz, P)

        return f


class Shock1D(InitialCondition):
    """Two constant states split at `position` along one axis (Sod's tube by default)."""

    def base_ic(self, dim="x", position=0.5, rho_left_right=(1, 0.125), P_left_right=(1, 0.1),
                v_left_right=(0, 0)):
        if dim not in ("x", "y", "z"):
            raise ValueError("dim must be 'x', 'y', or 'z'")

        def f(x, y=None, z=None):
            xp = of(x)
            r = {"x": x, "y": y, "z": z}[dim]
            left = r < position
            v = xp.where(left, v_left_right[0], v_left_right[1])
            vel = [v if dim == d else 0 for d in "xyz"]
            return _state(r, xp.where(left, *rho_left_right), *vel, xp.where(left, *P_left_right))

        return f


class DoubleShock1D(InitialCondition):
    """Three constant states separated at two positions along one axis."""

    def base_ic(self, dim="x", positions=(0.1, 0.9), rhos=(1, 1, 1), vs=(0, 0, 0), Ps=(10**3, 10**-2, 10**2)):
        def f(x, y=None, z=None):
            xp = of(x)
            r = {"x": x, "y": y, "z": z}[dim]

            def pick(vals):
                return xp.where(r < positions[0], vals[0], xp.where(r < positions[1], vals[1], vals[2]))

            vel = [pick(vs) if dim == d else 0 for d in "xyz"]
            return _state(r, pick(rhos), *vel, pick(Ps))

        return f


class ShuOsher1D(InitialCondition):
    """Mach-3 shock running into a density sine wave on [0, 10]."""

    def base_ic(self, dim="x"):
        def f(x, y=None, z=None):
            xp = of(x)
            r = {"x": x, "y": y, "z": z}[dim] - 5
            post = r < -4
            v = xp.where(post, 2.629369, 0)
            vel = [v if dim == d else 0 for d in "xyz"]
            return _state(r, xp.where(post, 3.857143, 1 + 0.2 * xp.sin(5 * r)), *vel,
                          xp.where(post, 10.33333, 1))

        return f


class KelvinHelmholtz2D(InitialCondition):
    """Shear band |y - 0.5| < 0.25 with a Gaussian-modulated vy perturbation."""

    def base_ic(self, sigma=0.05 * np.sqrt(2), w0=0.1):
        def f(x, y=None, z=None):
            xp = of(x)
            band = (y > 0.25) & (y < 0.75)
            g = xp.exp(xp.div(-xp.square(y - 0.25), 2 * sigma * sigma)) + xp.exp(
                xp.div(-xp.square(y - 0.75), 2 * sigma * sigma))
            return _state(band, xp.where(band, 2, 1), xp.where(band, 0.5, -0.5),
                          w0 * xp.sin(4 * xp.pi * x) * g, 0, 2.5)

        return f


class KelvinHelmholtzNoise2D(InitialCondition):
    """Kelvin-Helmholtz band of the benchmark configuration.

    rho = 2, vx = +0.5 where |y - 0.5| < 0.25, else rho = 1, vx = -0.5; P = 2.5;
    vy = 0.01 sin(4 pi x) + a per-cell uniform noise in [-amplitude, amplitude]
    drawn by numpy.random.default_rng(seed) on an (nx, ny) grid of the domain.
    The noise is constant inside each cell, so its FV average is exact.
    """

    def base_ic(self, n: Sequence[int] = (64, 64), seed: int = 0, amplitude: float = 1e-3,
                domain=((0.0, 1.0), (0.0, 1.0))):
        noise = np.random.default_rng(seed).uniform(-amplitude, amplitude, size=tuple(n[:2]))
        tables = {}  # device copies of the noise, per device
        (x0, x1), (y0, y1) = domain

        def f(x, y=None, z=None):
            xp = of(x)
            ix = xp.clip(xp.asint(xp.floor(xp.div(x - x0, x1 - x0) * n[0])), 0, n[0] - 1)
            iy = xp.clip(xp.asint(xp.floor(xp.div(y - y0, y1 - y0) * n[1])), 0, n[1] - 1)
            band = xp.abs(y - 0.5) < 0.25
            return _state(band, xp.where(band, 2.0, 1.0), xp.where(band, 0.5, -0.5),
                          0.01 * xp.sin(4 * xp.pi * x) + xp.lookup(noise, (ix, iy), tables), 0.0, 2.5)

        return f


class FourQuadrant2D(InitialCondition):
    """Four constant states split at (xs, ys) drawn from a seed.

    The split point is uniform in [0.3, 0.7]^2; per quadrant rho is
    log-uniform in [0.1, 2], P log-uniform in [0.01, 10], vx and vy uniform in
    [-1, 1]. Quadrant q = (x >= xs) + 2 (y >= ys).
    """

    def base_ic(self, seed: int = 0):
        rng = np.random.default_rng(seed)
        xs, ys = rng.uniform(0.3, 0.7, size=2)
        rho = np.exp(rng.uniform(np.log(0.1), np.log(2.0), size=4))
        P = np.exp(rng.uniform(np.log(0.01), np.log(10.0), size=4))
        vx = rng.uniform(-1, 1, size=4)
        vy = rng.uniform(-1, 1, size=4)
        tables = ({}, {}, {}, {})  # device copies of rho, vx, vy, P, per device

        def f(x, y=None, z=None):
            xp = of(x)
            q = xp.asint(x >= xs) + 2 * xp.asint(y >= ys)
            return _state(q, xp.lookup(rho, q, tables[0]), xp.lookup(vx, q, tables[1]), xp.lookup(vy, q, tables[2]),
                          0.0, xp.lookup(P, q, tables[3]))

        return f


class DoubleMachReflection2D(InitialCondition):
    """A Mach-10 shock through x = 1/6 at y = 0, inclined at 60 degrees to the x
    axis: the shocked state (rho 8, v = (7.145, -4.125), P 116.5) lies left of
    x - y / tan(pi/3) = 1/6, the gas at rest (rho = gamma, P 1) right of it
    (fvhoe/initial_conditions.py:369-399). Used with the low-y wall
    "special-case-double-mach-reflection-y=0"."""

    def base_ic(self, gamma: float = 1.4):
        tan = np.tan(np.pi / 3)

        def f(x, y=None, z=None):
            xp = of(x)
            post = (x - xp.div(y, tan)) < 1 / 6
            return _state(post, xp.where(post, 8, gamma), xp.where(post, 7.145, 0),
                          xp.where(post, -8.25 / 2, 0), 0, xp.where(post, 116.5, 1))

        return f


class ShockTube(InitialCondition):
    """Inside/outside states of a ball ("tube") or an axis-aligned box ("cube")."""

    def base_ic(self, dims="x", center=0.0, radius=0.5, rho_in_out=(1, 0.125), P_in_out=(1, 0.1),
                vx_in_out=(0, 0), vy_in_out=(0, 0), vz_in_out=(0, 0), mode="tube", x_cube=None, y_cube=None,
                z_cube=None):
        def f(x, y=None, z=None):
            xp = of(x)
            if mode == "tube":
                c = (center,) if isinstance(center, Number) else tuple(center)
                if len(c) != len(dims):
                    raise ValueError("center must have the same length as dims")
                rsq = xp.zeros_like(x)
                for d, cd in zip(dims, c):
                    rsq = rsq + ({"x": x, "y": y, "z": z}[d] - cd) ** 2
                inside = rsq <= radius**2
            elif mode == "cube":
                if x_cube is None and y_cube is None and z_cube is None:
                    raise ValueError("at least one cube dimension must be specified")
                inside = xp.mask_like(x)
                for c, rng in zip((x, y, z), (x_cube, y_cube, z_cube)):
                    if rng is not None:
                        inside &= (c >= rng[0]) & (c <= rng[1])
            else:
                raise ValueError(f"unknown mode {mode}")
            return _state(x, xp.where(inside, *rho_in_out), xp.where(inside, *vx_in_out),
                          xp.where(inside, *vy_in_out), xp.where(inside, *vz_in_out), xp.where(inside, *P_in_out))

        return f


class SedovBlast(InitialCondition):
    """Uniform medium with the blast energy in the corner cell (or the central 2^d cells).

    Slot 4 holds E: E0 in the medium and E1 / prod(2 h_d) over the listed axes
    in the blast cells, so the deposit integrates to E1 over the full
    (reflected) domain. Use with conservative_ic=True, fv_ic=True.
    """

    def base_ic(self, mode="corner", dims="xy", rho0=1.0, E0=1e-5, E1=1.0):
        def f(x, y=None, z=None):
            xp = of(x)
            nx, ny, nz = x.shape
            emax = E1
            for d, c, axis in (("x", x, 0), ("y", y, 1), ("z", z, 2)):
                if d in dims:
                    emax /= 2 * xp.diff_mean(c, axis)
            out = _state(x, rho0, 0, 0, 0, E0)
            if mode == "corner":
                out[4, 0, 0, 0] = emax
            elif mode == "center":
                sl = tuple(slice(k // 2 - 1, k // 2 + 1) if d in dims else slice(None)
                           for d, k in zip("xyz", (nx, ny, nz)))
                out[(4,) + sl] = emax
            else:
                raise ValueError(f"unknown mode {mode}")
            return out

        return f


class ArrayIC(InitialCondition):
    """A precomputed (nvars, nx, ny, nz) array (use with conservative_ic=fv_ic=True)."""

    def base_ic(self, array: np.ndarray = None):
        arr = np.asarray(array, dtype=np.float64)

        def f(x, y=None, z=None):
            return arr[:5] if of(x) is of(arr) else of(x).asarray(arr[:5], like=x)

        return f

    def build_ic(self, hs, passive_ic_funcs=None):
        arr = np.asarray(self.kwargs.get("array", self.args[0] if self.args else None), dtype=np.float64)

        def ic_func(x, y, z):
            if arr.shape[1:] != tuple(np.shape(x)):
                raise ValueError(f"array shape {arr.shape[1:]} does not match the mesh {tuple(np.shape(x))}")
            return arr.copy() if of(x) is of(arr) else of(x).asarray(arr, like=x)

        return ic_func
