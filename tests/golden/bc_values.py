"""Boundary values of the Dirichlet golden fixtures.

Shared by make_golden.py (which hands them to the reference's
BoundaryCondition) and the tests (which hand them to the oracle and to
fvhoe_b200): a fixture names its values in its JSON config, `resolve` turns a
name back into the array or function. Every function returns conserved
variables (rho, mx, my, mz, E) for gamma = 1.4, evaluated at the slab cell
centres x, y, z and, for "dirichlet" sides, the step's start time t.
"""

import numpy as np

GAMMA = 1.4


def _conserved(rho, vx, vy, vz, P):
    rho = np.asarray(rho, dtype=float)
    shape = np.broadcast(rho, vx, vy, vz, P).shape
    out = np.empty((5,) + shape)
    out[0] = rho
    out[1] = rho * vx
    out[2] = rho * vy
    out[3] = rho * vz
    out[4] = P / (GAMMA - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return out


def inflow_state():
    """A constant state entering from the low x side."""
    return _conserved(1.2, 0.6, -0.1, 0.0, 1.1).reshape(5)


def wall_y_low(x, y, z, t):
    """A time-dependent density wave on the low y side."""
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * x) + t
    return _conserved(rho, 0.1 + 0 * x, 0.3 + 0 * x, 0 * x, 1.0 + 0 * x)


def wall_y_high(x, y, z, t):
    """A state that slows down with time on the high y side."""
    rho = 1.5 + 0.1 * np.cos(2 * np.pi * x)
    return _conserved(rho, -0.2 + 0 * x, -0.4 * (1.0 - t) + 0 * x, 0 * x, 1.3 + 0 * x)


def box_x_low(x, y, z, t):
    """A smooth 3D state on the low x side of a box."""
    rho = 1.0 + 0.1 * np.sin(2 * np.pi * (y + z)) + 0.5 * t
    return _conserved(rho, 0.2 + 0 * x, 0.1 * np.cos(2 * np.pi * z), -0.1 + 0 * x, 0.9 + 0.1 * y)


def box_z_high(x, y, z, t):
    """A smooth 3D state on the high z side of a box."""
    rho = 0.8 + 0.1 * x * y
    return _conserved(rho, 0 * x, 0.05 + 0 * x, -0.3 + 0.2 * t + 0 * x, 1.0 + 0 * x)


def dmr_inflow():
    """The shocked gas of the double Mach reflection entering from the low x side."""
    return _conserved(8.0, 7.145, -8.25 / 2, 0.0, 116.5).reshape(5)


def dmr_top(x, y, z, t):
    """The high y side of the double Mach reflection: shocked gas left of the
    Mach-10 shock, inclined at 60 degrees and moving at 10 / sin(60 deg)
    along x (Woodward and Colella's set-up), gas at rest right of it."""
    theta = np.pi / 3
    front = 10 * t / np.sin(theta) + 1 / 6 + y / np.tan(theta)
    post = x < front
    return _conserved(np.where(post, 8.0, GAMMA), np.where(post, 7.145, 0.0), np.where(post, -8.25 / 2, 0.0),
                      0 * x, np.where(post, 116.5, 1.0))


VALUES = {
    "inflow_state": inflow_state,
    "wall_y_low": wall_y_low,
    "wall_y_high": wall_y_high,
    "box_x_low": box_x_low,
    "box_z_high": box_z_high,
    "dmr_inflow": dmr_inflow,
    "dmr_top": dmr_top,
}
ARRAYS = {"inflow_state", "dmr_inflow"}


def resolve(name):
    """The BoundaryCondition value a name stands for (None stays None)."""
    if name is None:
        return None
    if name in ARRAYS:
        return VALUES[name]()
    return VALUES[name]
