"""Mesh and finite-volume averaging of initial conditions (host, set-up only).

Same interfaces as fvhoe/fv.py:12-85 (`fv_uniform_meshgen` without slab
coordinates) and :227-277 (`fv_average` with Gauss-Legendre quadrature).
These run once per solver, on the host, before the state moves to the GPU.
"""

from functools import lru_cache
from typing import Callable, Tuple

import numpy as np


def fv_uniform_meshgen(n, x=(0, 1), y=(0, 1), z=(0, 1)):
    """Cell-centre coordinates X, Y, Z of shape (nx, ny, nz)."""
    centres = []
    for count, (lo, hi) in zip(n, (x, y, z)):
        edges = np.linspace(lo, hi, count + 1)
        centres.append(0.5 * (edges[1:] + edges[:-1]))
    return np.meshgrid(*centres, indexing="ij")


@lru_cache(maxsize=16)
def legendre_quadrature(p: int) -> Tuple[np.ndarray, np.ndarray]:
    """ceil((p+1)/2) Gauss-Legendre nodes and weights on [-1/2, 1/2], weights summing to 1."""
    nodes, weights = np.polynomial.legendre.leggauss(-(-(p + 1) // 2))
    return nodes / 2, weights / 2


def fv_average(f: Callable, x, y, z, h, p=(0, 0, 0)) -> np.ndarray:
    """Cell averages of f(x, y, z) by tensor-product Gauss-Legendre quadrature."""
    rules = [legendre_quadrature(pi) for pi in p]
    out = np.zeros_like(f(x, y, z))
    for xp, xw in zip(*rules[0]):
        for yp, yw in zip(*rules[1]):
            for zp, zw in zip(*rules[2]):
                out += (xw * yw * zw) * f(x=x + xp * h[0], y=y + yp * h[1], z=z + zp * h[2])
    return out
