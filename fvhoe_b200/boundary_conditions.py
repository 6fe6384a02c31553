"""Boundary-condition specification (host side).

Same constructor as fvhoe/boundary_conditions.py:154-229 (`BoundaryCondition`
with x, y, z kinds given as one value or a (low, high) pair, and x_value,
y_value, z_value for Dirichlet sides). The ghost cells themselves are never
materialised: the CUDA kernels read the interior through per-axis index maps
(periodic wrap, mirror, mirror with the normal momentum negated, or edge
repeat), which is what the reference's slab copies produce, and read the
ghost values of "dirichlet" and "ic" sides from arrays the solver evaluates
at the reference's slab coordinates (fvhoe/boundary_conditions.py:18-55).
The low y side may be "special-case-double-mach-reflection-y=0", the wall of
the double Mach reflection problem (:374-395): free where the ghost column's
x centre is below 1/6, reflective elsewhere.
"""

from dataclasses import dataclass, field
from typing import Any, Tuple, Union

import numpy as np

DMR_Y0 = "special-case-double-mach-reflection-y=0"
SUPPORTED = ("periodic", "outflow", "reflective", "free", "dirichlet", "ic", DMR_Y0)


def dmr_split(n, x, y, z, buffer) -> int:
    """First x index (ghost cells negative) where the double-Mach-reflection
    wall turns reflective. The reference picks free ghost values where the
    column's x centre on its low-y slab coordinates (`buffer` cells deep per
    axis) is below 1/6 (fvhoe/boundary_conditions.py:375-395); the centres
    increase with the index, so the free columns are a prefix."""
    from .fv import slab_meshgen

    X = slab_meshgen(n, x, y, z, buffer)["yl"][0][:, 0, 0]
    free = X < 1 / 6
    split = free.size if free.all() else int(np.argmin(free))
    if free[split:].any():
        raise ValueError("slab x centres are not increasing")
    return split - buffer[0]


@dataclass
class BoundaryCondition:
    x: Union[str, Tuple[str, str]] = "periodic"
    y: Union[str, Tuple[str, str]] = "periodic"
    z: Union[str, Tuple[str, str]] = "periodic"
    x_value: Any = None
    y_value: Any = None
    z_value: Any = None
    slab_coords: Any = field(default=None, repr=False)
    array_manager: Any = field(default=None, repr=False)
    hydro_state: Any = field(default=None, repr=False)

    def __post_init__(self):
        for dim in "xyz":
            for suffix in ("", "_value"):
                value = getattr(self, f"{dim}{suffix}")
                if isinstance(value, tuple):
                    if len(value) != 2:
                        raise ValueError(f"Invalid length of {dim}{suffix} tuple")
                elif isinstance(value, list):
                    raise ValueError(f"Invalid type of {dim}{suffix}: list")
                else:
                    setattr(self, f"{dim}{suffix}", (value, value))

    def kinds(self, active: Tuple[bool, bool, bool]):
        """(low, high) kinds per axis; raises for unknown kinds and misplaced ones."""
        out = []
        for dim, on in zip("xyz", active):
            pair = getattr(self, dim)
            if on:
                for kind in pair:
                    if kind not in SUPPORTED:
                        raise ValueError(f"Unknown bc type '{kind}'")
                if pair[1] == DMR_Y0 or (pair[0] == DMR_Y0 and dim != "y"):
                    raise ValueError(f"'{DMR_Y0}' is defined on the low y side only")
                if pair[1] == "periodic" and pair[0] != "periodic":
                    raise ValueError(f"a periodic high boundary on {dim} needs a periodic low boundary")
                values = getattr(self, f"{dim}_value")
                for kind, value in zip(pair, values):
                    if kind == "dirichlet" and not (callable(value) or isinstance(value, np.ndarray)):
                        raise ValueError(f"Invalid boundary of type '{value}'.")
            out.append(tuple(pair))
        return tuple(out)

    def to_dict(self) -> dict:
        return dict(x=self.x, y=self.y, z=self.z)
