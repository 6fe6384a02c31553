"""Boundary-condition specification (host side).

Same constructor as fvhoe/boundary_conditions.py:154-229 (`BoundaryCondition`
with x, y, z kinds given as one value or a (low, high) pair, and x_value,
y_value, z_value for Dirichlet sides). The ghost cells themselves are never
materialised: the CUDA kernels read the interior through per-axis index maps
(periodic wrap, mirror, mirror with the normal momentum negated, or edge
repeat), which is what the reference's slab copies produce, and read the
ghost values of "dirichlet" and "ic" sides from arrays the solver evaluates
at the reference's slab coordinates (fvhoe/boundary_conditions.py:18-55).
"""

from dataclasses import dataclass, field
from typing import Any, Tuple, Union

import numpy as np

SUPPORTED = ("periodic", "outflow", "reflective", "free", "dirichlet", "ic")
# the reference's own branch for this kind calls _set_free_bc without its first
# argument (fvhoe/boundary_conditions.py:382), so it cannot run there either
NOT_SUPPORTED = ("special-case-double-mach-reflection-y=0",)


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
        """(low, high) kinds per axis; raises for kinds the CUDA backend does not provide."""
        out = []
        for dim, on in zip("xyz", active):
            pair = getattr(self, dim)
            if on:
                for kind in pair:
                    if kind in NOT_SUPPORTED:
                        raise NotImplementedError(
                            f"boundary '{kind}' on {dim} is not provided by the CUDA backend "
                            f"(supported: {', '.join(SUPPORTED)})"
                        )
                    if kind not in SUPPORTED:
                        raise ValueError(f"Unknown bc type '{kind}'")
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
