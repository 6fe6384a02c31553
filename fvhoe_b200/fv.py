"""Mesh and finite-volume averaging of initial conditions (set-up only).

Same interfaces as fvhoe/fv.py:12-85 (`fv_uniform_meshgen`; the ghost-slab
coordinates are `slab_meshgen`) and :227-277 (`fv_average` with
Gauss-Legendre quadrature). These run once per solver: the averaging on the
host, or on the device for the library's initial conditions with
`EulerSolver(ic_on_device=True)`; the slab coordinates of Dirichlet
boundaries on the host.
"""

from functools import lru_cache
from itertools import product
from typing import Callable, Dict, Tuple

import numpy as np

from .array_ns import of


def fv_uniform_meshgen(n, x=(0, 1), y=(0, 1), z=(0, 1)):
    """Cell-centre coordinates X, Y, Z of shape (nx, ny, nz)."""
    centres = []
    for count, (lo, hi) in zip(n, (x, y, z)):
        edges = np.linspace(lo, hi, count + 1)
        centres.append(0.5 * (edges[1:] + edges[:-1]))
    return np.meshgrid(*centres, indexing="ij")


def slab_meshgen(n, x=(0, 1), y=(0, 1), z=(0, 1), thickness=(0, 0, 0)) -> Dict[str, tuple]:
    """Cell centres of the ghost slabs {'xl': (X, Y, Z), 'xr': ..., 'zr': ...}
    built as fvhoe/fv.py:53-84 builds them: each slab is `thickness` cells deep
    along its axis and spans the other axes with their slabs included."""
    h = ((x[1] - x[0]) / n[0], (y[1] - y[0]) / n[1], (z[1] - z[0]) / n[2])
    gwx, gwy, gwz = thickness
    out = {}
    for dim, pos in product("xyz", "lr"):
        sizes = (gwx if dim == "x" else n[0] + 2 * gwx, gwy if dim == "y" else n[1] + 2 * gwy,
                 gwz if dim == "z" else n[2] + 2 * gwz)
        ranges = []
        for d, (lo, hi), hd, gd in zip("xyz", (x, y, z), h, thickness):
            if d == dim:
                ranges.append({"l": (lo - hd * gd, lo), "r": (hi, hi + hd * gd)}[pos])
            else:
                ranges.append((lo - hd * gd, hi + hd * gd))
        out[dim + pos] = tuple(fv_uniform_meshgen(sizes, *ranges))
    return out


def trim_slab(coords, buffer, gw, axis: int, pos: str):
    """The part of a slab (from slab_meshgen with thickness `buffer`) that a
    ghost fill of width gw uses: the gw layers next to the domain along `axis`,
    the interior plus gw layers along the others (fvhoe/boundary_conditions.py:231-289)."""
    sl = []
    for a in range(3):
        excess = buffer[a] - gw[a]
        if excess < 0:
            raise ValueError(f"Cannot apply bc to region of thickness {gw[a]} with a buffer of thickness {buffer[a]}")
        cut = {"l": (-gw[a], 0), "r": (0, gw[a])}[pos] if a == axis else (excess, -excess)
        sl.append(slice(cut[0] or None, cut[1] or None))
    return tuple(c[tuple(sl)] for c in coords)


@lru_cache(maxsize=16)
def legendre_quadrature(p: int) -> Tuple[np.ndarray, np.ndarray]:
    """ceil((p+1)/2) Gauss-Legendre nodes and weights on [-1/2, 1/2], weights summing to 1."""
    nodes, weights = np.polynomial.legendre.leggauss(-(-(p + 1) // 2))
    return nodes / 2, weights / 2


def fv_average(f: Callable, x, y, z, h, p=(0, 0, 0)):
    """Cell averages of f(x, y, z) by tensor-product Gauss-Legendre quadrature,
    for host arrays or device tensors (the same sums in the same order)."""
    rules = [legendre_quadrature(pi) for pi in p]
    first = f(x, y, z)
    out = of(first).zeros_like(first)
    for xq, xw in zip(*rules[0]):
        for yq, yw in zip(*rules[1]):
            for zq, zw in zip(*rules[2]):
                out += float(xw * yw * zw) * f(x=x + float(xq * h[0]), y=y + float(yq * h[1]),
                                               z=z + float(zq * h[2]))
    return out
