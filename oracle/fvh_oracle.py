"""NumPy restatement of FVHOE's per-stage update (test infrastructure only).

Every function cites the reference file:line it restates (paths inside the
jpalafou/FVHOE project). The restatement keeps the reference's floating-point
evaluation order on purpose (left-to-right stencil accumulation from +0, the
same association of every product and sum), because the CUDA path is checked
against this module for equality, not closeness.

Arrays use the reference layout: (nvars, nx, ny, nz), C order, so z is the
contiguous axis; variable 0 = rho, 1..3 = momentum / velocity, 4 = E / P,
5.. = passive scalars.
"""

from dataclasses import dataclass, field
from fractions import Fraction
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

__all__ = [
    "OracleConfig",
    "stencil_weights",
    "stencil_radius",
    "sweep",
    "pad_with_ghosts",
    "conservatives_to_primitives",
    "primitives_to_conservatives",
    "sound_speed",
    "fv_primitives",
    "cfl_dt",
    "riemann_flux",
    "hydrofluxes",
    "flux_divergence",
    "detect_trouble",
    "smooth_extrema_alpha",
    "face_trouble",
    "rhs",
    "step",
    "hit_target",
    "VARIABLE_INDEX",
]

# ---------------------------------------------------------------------------
# stencil weights (fvhoe/stencils.py:5-22, 25-178, 181-255)
# ---------------------------------------------------------------------------
# Each rule is stored as (denominator, integer numerators); the float64 weight
# is the correctly rounded value of the exact rational, which is what the
# reference's `a / b` literals evaluate to.
_LEFT_FACE = {
    0: (1, (1,)),
    1: (4, (1, 4, -1)),
    2: (6, (2, 5, -1)),
    3: (24, (-1, 10, 20, -6, 1)),
    4: (60, (-3, 27, 47, -13, 2)),
    5: (120, (1, -10, 59, 94, -31, 8, -1)),
    6: (420, (4, -38, 214, 319, -101, 25, -3)),
    7: (1680, (-3, 34, -194, 898, 1276, -446, 142, -30, 3)),
    8: (2520, (-5, 55, -305, 1375, 1879, -641, 199, -41, 4)),
}
# centre-point interpolation and transverse (point -> average) rules for even
# degrees; an odd degree p uses the rule of degree p - 1 padded by one zero tap
# on each side (fvhoe/stencils.py:47-49, 59-60, 77-81, 125-139; 190, 196-205, 218-232)
_CENTRE_EVEN = {
    0: (1, (1,)),
    2: (24, (-1, 26, -1)),
    4: (1920, (9, -116, 2134, -116, 9)),
    6: (107520, (-75, 954, -7621, 121004, -7621, 954, -75)),
    8: (
        10321920,
        (1225, -17000, 125884, -800216, 11702134, -800216, 125884, -17000, 1225),
    ),
}
_TRANSVERSE_EVEN = {
    0: (1, (1,)),
    2: (24, (1, 22, 1)),
    4: (5760, (-17, 308, 5178, 308, -17)),
    6: (967680, (367, -5058, 57249, 862564, 57249, -5058, 367)),
    8: (
        464486400,
        (
            -27859,
            399032,
            -3207892,
            29039624,
            412080590,
            29039624,
            -3207892,
            399032,
            -27859,
        ),
    ),
}


def stencil_radius(p: int) -> int:
    """Taps to each side of the centre, ceil(p/2) (fvhoe/stencils.py:5-22)."""
    return -(-int(p) // 2)


def _rational_rule(p: int, kind: str) -> Tuple[Fraction, ...]:
    if not 0 <= p <= 8:
        raise NotImplementedError(f"p={p}")
    if kind == "l":
        den, nums = _LEFT_FACE[p]
        return tuple(Fraction(n, den) for n in nums)
    if kind == "r":
        return tuple(reversed(_rational_rule(p, "l")))
    table = {"c": _CENTRE_EVEN, "t": _TRANSVERSE_EVEN}[kind]
    even = p if p % 2 == 0 else p - 1
    den, nums = table[even]
    rule = tuple(Fraction(n, den) for n in nums)
    if p % 2 == 1:
        rule = (Fraction(0),) + rule + (Fraction(0),)
    return rule


def stencil_weights(p: int, kind: str) -> np.ndarray:
    """float64 weights of one rule.

    kind: "l"/"c"/"r" conservative interpolation to the left face, centre or
    right face (fvhoe/stencils.py:25-178; "r" is "l" reversed, :42-43), or "t"
    for transverse reconstruction (fvhoe/stencils.py:181-255).
    """
    return np.array([float(w) for w in _rational_rule(p, kind)], dtype=np.float64)


def sweep(a: np.ndarray, weights: np.ndarray, axis: int) -> np.ndarray:
    """One stencil pass along `axis`; the result is shorter by len(weights)-1.

    Accumulates w_k * a[k + i] left to right starting from +0
    (fvhoe/fv.py:106-140 with the slices of fvhoe/fv.py:88-103).
    """
    k = len(weights)
    n_out = a.shape[axis] - (k - 1)
    if n_out < 0:
        raise ValueError("array too short for stencil")
    shape = list(a.shape)
    shape[axis] = n_out
    out = np.zeros(shape, dtype=np.float64)
    index = [slice(None)] * a.ndim
    for j in range(k):
        index[axis] = slice(j, j + n_out)
        out += weights[j] * a[tuple(index)]
    return out


# ---------------------------------------------------------------------------
# variable map (fvhoe/hydro.py:8-67)
# ---------------------------------------------------------------------------
VARIABLE_INDEX = {
    "rho": 0,
    "vx": 1,
    "mx": 1,
    "vy": 2,
    "my": 2,
    "vz": 3,
    "mz": 3,
    "P": 4,
    "E": 4,
}


# ---------------------------------------------------------------------------
# configuration
# ---------------------------------------------------------------------------
@dataclass
class OracleConfig:
    """Solver settings that matter to one right-hand-side evaluation.

    Mirrors the constructor arguments of fvhoe/solver.py:42-84 that reach the
    hot path; `bc` holds (low, high) kinds per axis from
    {"periodic", "outflow", "reflective", "free", "dirichlet", "ic"};
    `bc_values` the value of each "dirichlet" side (an array of nvars
    conserved values, or a function of x, y, z, t) and of each "ic" side (the
    pointwise conserved initial condition, a function of x, y, z); `t` is the
    time the boundary functions see (the step's start time,
    fvhoe/solver.py:784).
    """

    n: Tuple[int, int, int]
    p: Tuple[int, int, int]
    h: Tuple[float, float, float]
    nvars: int = 5
    gamma: float = 5 / 3
    CFL: float = 0.8
    fixed_dt: Optional[float] = None
    riemann_solver: str = "hllc"
    bc: Tuple[Tuple[str, str], Tuple[str, str], Tuple[str, str]] = (
        ("periodic", "periodic"),
        ("periodic", "periodic"),
        ("periodic", "periodic"),
    )
    a_posteriori_slope_limiting: bool = False
    slope_limiter: Optional[str] = "minmod"
    force_trouble: bool = False
    NAD: float = 1e-2
    NAD_mode: str = "global"
    NAD_range: str = "relative"
    NAD_vars: Optional[Tuple[str, ...]] = None
    PAD: Optional[Dict[str, Tuple[float, float]]] = field(
        default_factory=lambda: {"rho": (0.0, np.inf), "P": (0.0, np.inf)}
    )
    SED: bool = True
    SED_tolerance: float = 1e-10
    convex: bool = False
    csq_floor: float = 1e-10
    domain: Tuple[Tuple[float, float], ...] = ((0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    bc_values: Optional[Tuple] = None
    slab_buffer_size: int = 30
    t: float = 0.0

    @property
    def active(self) -> Tuple[bool, bool, bool]:
        """An axis takes part unless it has one cell and p = 0 (fvhoe/solver.py:244-254)."""
        return tuple(not (self.n[a] == 1 and self.p[a] == 0) for a in range(3))

    @property
    def dims(self) -> str:
        return "".join(d for d, on in zip("xyz", self.active) if on)

    @property
    def ndim(self) -> int:
        return sum(self.active)


# ---------------------------------------------------------------------------
# ghost cells (fvhoe/boundary_conditions.py:60-151, 306-402)
# ---------------------------------------------------------------------------
def _ghost_source(n: int, g: int, low: str, high: str):
    """Source index and reflective flag for each of the n + 2g padded cells."""
    idx = np.arange(-g, n + g)
    src = idx.copy()
    flip = np.zeros(idx.shape, dtype=bool)
    lo = idx < 0
    hi = idx >= n
    for mask, kind, side in ((lo, low, "l"), (hi, high, "r")):
        if not mask.any():
            continue
        if kind in ("periodic", "outflow", "reflective") and g > n:
            raise ValueError(f"{g} ghost cells exceed the {n} interior cells")
        if kind == "periodic":
            src[mask] = idx[mask] + (n if side == "l" else -n)
        elif kind in ("outflow", "reflective"):
            src[mask] = (-1 - idx[mask]) if side == "l" else (2 * n - 1 - idx[mask])
            if kind == "reflective":
                flip[mask] = True
        elif kind == "free":
            src[mask] = 0 if side == "l" else n - 1
        else:
            raise ValueError(f"unsupported boundary '{kind}'")
    return src, flip


def _slab_meshgen(n, domain, thickness):
    """Cell centres of the ghost slabs, {'xl': (X, Y, Z), ...} (fvhoe/fv.py:53-84)."""
    def centres(count, lo, hi):
        edges = np.linspace(lo, hi, count + 1)
        return 0.5 * (edges[1:] + edges[:-1])

    h = [(domain[a][1] - domain[a][0]) / n[a] for a in range(3)]
    out = {}
    for a, dim in enumerate("xyz"):
        for pos in "lr":
            axes = []
            for b in range(3):
                lo, hi = domain[b]
                gb = thickness[b]
                if b == a:
                    rng = (lo - h[b] * gb, lo) if pos == "l" else (hi, hi + h[b] * gb)
                    axes.append(centres(gb, *rng))
                else:
                    axes.append(centres(n[b] + 2 * gb, lo - h[b] * gb, hi + h[b] * gb))
            out[dim + pos] = tuple(np.meshgrid(*axes, indexing="ij"))
    return out


def _dirichlet_slab(cfg, axis: int, side: int, g: Sequence[int]) -> np.ndarray:
    """Ghost values of a "dirichlet" or "ic" side for a fill of g cells per
    axis (fvhoe/boundary_conditions.py:18-55, 231-289, 334-347): the slab
    coordinates are built slab_buffer_size deep and trimmed to g."""
    buffer = tuple(cfg.slab_buffer_size if act else 0 for act in cfg.active)
    pos = "lr"[side]
    coords = _slab_meshgen(cfg.n, cfg.domain, buffer)["xyz"[axis] + pos]
    sl = []
    for a in range(3):
        excess = buffer[a] - g[a]
        cut = ((-g[a], 0) if pos == "l" else (0, g[a])) if a == axis else (excess, -excess)
        sl.append(slice(cut[0] or None, cut[1] or None))
    X, Y, Z = (c[tuple(sl)] for c in coords)
    kind = cfg.bc[axis][side]
    value = cfg.bc_values[axis][side]
    if kind == "ic":
        return value(x=X, y=Y, z=Z)
    if callable(value):
        return value(x=X, y=Y, z=Z, t=cfg.t)
    return np.ones((cfg.nvars,) + X.shape) * np.asarray(value).reshape(-1, 1, 1, 1)


DMR_Y0 = "special-case-double-mach-reflection-y=0"


def _fill_axis(u: np.ndarray, g: int, axis: int, low: str, high: str) -> np.ndarray:
    """u padded by g ghost cells of the given kinds along one spatial axis."""
    src, flip = _ghost_source(u.shape[axis + 1], g, low, high)
    out = np.take(u, src, axis=axis + 1)
    if flip.any():
        sel = [slice(None)] * 4
        sel[0] = 1 + axis
        sel[axis + 1] = flip
        out[tuple(sel)] *= -1.0
    return out


def _dmr_free_columns(cfg, g: Sequence[int]) -> np.ndarray:
    """Mask over the n_x + 2 g_x padded x columns: True where the low-y slab's
    x centre (built slab_buffer_size deep, trimmed to g_x ghosts) is below 1/6
    (fvhoe/boundary_conditions.py:375-377)."""
    buffer = tuple(cfg.slab_buffer_size if act else 0 for act in cfg.active)
    X = _slab_meshgen(cfg.n, cfg.domain, buffer)["yl"][0][:, 0, 0]
    excess = buffer[0] - g[0]
    X = X[excess:X.size - excess]
    return X < 1 / 6


def pad_with_ghosts(u: np.ndarray, g: Sequence[int], bc, cfg=None) -> np.ndarray:
    """Pad (nvars, nx, ny, nz) by g[a] ghost cells per spatial axis.

    periodic copies the opposite interior, outflow mirrors, reflective mirrors
    and negates the normal momentum, free repeats the edge cell
    (fvhoe/boundary_conditions.py:60-151), "dirichlet" and "ic" sides take
    the values of cfg (:18-55), the double-Mach-reflection wall on the low y
    side is free or reflective by column (:374-395); axes are filled x, then
    y, then z, each slab
    spanning the ghost layers of the axes filled before it, so corner ghosts
    take the last axis' treatment of the earlier axes' values (:324-400).
    """
    out = u
    for axis in range(3):
        if g[axis] == 0:
            continue
        kinds = list(bc[axis])
        dirichlet = [k in ("dirichlet", "ic") for k in kinds]
        mapped = [k if not d else "free" for k, d in zip(kinds, dirichlet)]
        n_a = out.shape[axis + 1]
        if kinds[0] == DMR_Y0:
            # the double-Mach-reflection wall: both fills, chosen per x column
            # by the low-y slab's x centre (fvhoe/boundary_conditions.py:374-395)
            if axis != 1:
                raise ValueError(f"'{DMR_Y0}' is defined on the low y side only")
            free = _fill_axis(out, g[axis], axis, "free", mapped[1])
            refl = _fill_axis(out, g[axis], axis, "reflective", mapped[1])
            out = np.where(_dmr_free_columns(cfg, g)[None, :, None, None], free, refl)
        else:
            out = _fill_axis(out, g[axis], axis, *mapped)
        for side in range(2):
            if not dirichlet[side]:
                continue
            values = _dirichlet_slab(cfg, axis, side, g)
            # the axes after this one are not padded yet: their interior part
            sel = [slice(None)] * 4
            for b in range(axis + 1, 3):
                sel[b + 1] = slice(g[b], g[b] + cfg.n[b])
            values = values[tuple(sel)]
            dst = [slice(None)] * 4
            dst[axis + 1] = slice(0, g[axis]) if side == 0 else slice(n_a + g[axis], n_a + 2 * g[axis])
            out[tuple(dst)] = values
    return out


# ---------------------------------------------------------------------------
# thermodynamics (fvhoe/hydro.py:146-210, 270-294)
# ---------------------------------------------------------------------------
def conservatives_to_primitives(u: np.ndarray, gamma: float) -> np.ndarray:
    """v = m / rho, P = (gamma - 1)(E - 0.5 sum m v), passives / rho (fvhoe/hydro.py:146-170)."""
    w = np.empty_like(u)
    rho = u[0]
    w[0] = rho
    w[1:4] = u[1:4] / rho
    ke = u[1] * w[1]
    ke = ke + u[2] * w[2]
    ke = ke + u[3] * w[3]
    w[4] = (gamma - 1) * (u[4] - 0.5 * ke)
    if u.shape[0] > 5:
        w[5:] = u[5:] / rho
    return w


def primitives_to_conservatives(w: np.ndarray, gamma: float) -> np.ndarray:
    """m = rho v, E = P/(gamma-1) + 0.5 sum m v, passives * rho (fvhoe/hydro.py:173-196)."""
    u = np.empty_like(w)
    rho = w[0]
    u[0] = rho
    u[1:4] = rho * w[1:4]
    ke = u[1] * w[1]
    ke = ke + u[2] * w[2]
    ke = ke + u[3] * w[3]
    u[4] = w[4] / (gamma - 1) + 0.5 * ke
    if w.shape[0] > 5:
        u[5:] = rho * w[5:]
    return u


def sound_speed(w: np.ndarray, gamma: float, csq_floor: float) -> np.ndarray:
    """sqrt(gamma P / rho) with csq floored (fvhoe/hydro.py:199-210)."""
    csq = gamma * w[4] / w[0]
    return np.sqrt(np.where(csq > csq_floor, csq, csq_floor))


def cfl_dt(w: np.ndarray, cfg: OracleConfig) -> float:
    """CFL h / max(sum_d |v_d| + ndim c) over the padded array (fvhoe/hydro.py:270-294).

    h is the smallest spacing of all three axes (fvhoe/solver.py:508-515).
    """
    c = sound_speed(w, cfg.gamma, cfg.csq_floor)
    va = np.abs(w[1:4])
    s = va[0] + va[1]
    s = s + va[2]
    return float(cfg.CFL * min(cfg.h) / np.max(s + cfg.ndim * c))


# ---------------------------------------------------------------------------
# finite-volume primitives (fvhoe/solver.py:753-792, fvhoe/fv.py:175-224)
# ---------------------------------------------------------------------------
def fv_primitives(
    u: np.ndarray,
    cfg: OracleConfig,
    p: Sequence[int],
    gw: Sequence[int],
    fv_average: bool = True,
) -> np.ndarray:
    """Finite-volume (or cell-centre) primitives with gw ghost cells per axis.

    Ghost-fill u with gw + 2 ceil(p/2) cells (ceil(p/2) for centres), sweep
    centre interpolation along x, y, z, convert to primitives, then sweep
    transverse reconstruction along x, y, z (fvhoe/solver.py:753-792).
    """
    factor = 2 if fv_average else 1
    g = [gw[a] + factor * stencil_radius(p[a]) for a in range(3)]
    a_bc = pad_with_ghosts(u, g, cfg.bc, cfg)
    for axis in range(3):
        a_bc = sweep(a_bc, stencil_weights(p[axis], "c"), axis + 1)
    w = conservatives_to_primitives(a_bc, cfg.gamma)
    if fv_average:
        for axis in range(3):
            w = sweep(w, stencil_weights(p[axis], "t"), axis + 1)
    return w


# ---------------------------------------------------------------------------
# Riemann solvers (fvhoe/riemann_solvers.py)
# ---------------------------------------------------------------------------
def _physical_flux(w, u, axis, include_pressure=True):
    """Toro's Euler flux along one axis (fvhoe/hydro.py:213-246)."""
    v = w[1 + axis]
    out = np.empty_like(w)
    out[0] = v * w[0]
    out[1:4] = v * u[1:4]
    out[4] = v * u[4]
    if include_pressure:
        out[1 + axis] = out[1 + axis] + w[4]
        out[4] = out[4] + v * w[4]
    if w.shape[0] > 5:
        out[5:] = v * u[5:]
    return out


def _nan_max(a, b):
    return np.maximum(a, b)


def riemann_flux(wl, wr, axis, cfg: OracleConfig) -> np.ndarray:
    """Interface flux from left/right primitive states.

    hllc: fvhoe/riemann_solvers.py:91-197 (Sl/Sr from min/max velocity -/+ the
    larger sound speed; transverse quantities upwinded by the sign of the
    sampled velocity). llf: :48-88. advection_upwind: :13-45.
    """
    g = cfg.gamma
    floor = cfg.csq_floor
    ul = primitives_to_conservatives(wl, g)
    ur = primitives_to_conservatives(wr, g)
    if cfg.riemann_solver == "advection_upwind":
        fl = _physical_flux(wl, ul, axis, include_pressure=False)
        fr = _physical_flux(wr, ur, axis, include_pressure=False)
        v = wl[1 + axis][np.newaxis]
        return np.where(v > 0, fl, np.where(v < 0, fr, 0))
    if cfg.riemann_solver == "llf":
        fl = _physical_flux(wl, ul, axis)
        fr = _physical_flux(wr, ur, axis)
        sl = np.abs(wl[1 + axis]) + sound_speed(wl, g, floor)
        sr = np.abs(wr[1 + axis]) + sound_speed(wr, g, floor)
        smax = _nan_max(sl, sr)
        return 0.5 * (fl + fr) - 0.5 * smax * (ur - ul)
    if cfg.riemann_solver != "hllc":
        raise ValueError(f"unknown Riemann solver {cfg.riemann_solver}")
    cl = sound_speed(wl, g, floor)
    cr = sound_speed(wr, g, floor)
    cmax = _nan_max(cl, cr)
    vl, vr = wl[1 + axis], wr[1 + axis]
    rl, rr = wl[0], wr[0]
    pl, pr = wl[4], wr[4]
    el, er = ul[4], ur[4]
    s_l = np.minimum(vl, vr) - cmax
    s_r = np.maximum(vl, vr) + cmax
    rcl = rl * (vl - s_l)
    rcr = rr * (s_r - vr)
    v_star = (rcl * vl + rcr * vr + pl - pr) / (rcl + rcr)
    p_star = (rcl * pr + rcr * pl + rcl * rcr * (vl - vr)) / (rcl + rcr)
    r_star_l = rl * (s_l - vl) / (s_l - v_star)
    e_star_l = ((s_l - vl) * el - pl * vl + p_star * v_star) / (s_l - v_star)
    r_star_r = rr * (s_r - vr) / (s_r - v_star)
    e_star_r = ((s_r - vr) * er - pr * vr + p_star * v_star) / (s_r - v_star)

    def pick(a_l, a_sl, a_sr, a_r):
        return np.where(s_l > 0, a_l, np.where(v_star > 0, a_sl, np.where(s_r > 0, a_sr, a_r)))

    r_g = pick(rl, r_star_l, r_star_r, rr)
    v_g = pick(vl, v_star, v_star, vr)
    p_g = pick(pl, p_star, p_star, pr)
    e_g = pick(el, e_star_l, e_star_r, er)
    out = np.empty_like(ul)
    out[0] = r_g * v_g
    for t in range(3):
        if t == axis:
            out[1 + t] = r_g * v_g * v_g + p_g
        else:
            up = np.where(v_g > 0, wl[1 + t], np.where(v_g < 0, wr[1 + t], 0))
            out[1 + t] = r_g * v_g * up
    out[4] = v_g * (e_g + p_g)
    if wl.shape[0] > 5:
        up = np.where(v_g > 0, wl[5:], np.where(v_g < 0, wr[5:], 0))
        out[5:] = r_g * v_g * up
    return out


# ---------------------------------------------------------------------------
# MUSCL (fvhoe/slope_limiting.py:24-84)
# ---------------------------------------------------------------------------
def _limited_slope(dl, dr, limiter):
    if limiter == "minmod":
        den = np.where(dl > 0, np.where(dl > 1e-16, dl, 1e-16), np.where(dl < -1e-16, dl, -1e-16))
        ratio = dr / den
        ratio = np.where(ratio < 1, ratio, 1)
        return np.where(ratio > 0, ratio, 0) * dl
    if limiter == "moncen":
        dc = 0.5 * (dl + dr)
        s = np.minimum(np.abs(2 * dl), np.abs(2 * dr))
        s = np.sign(dc) * np.minimum(s, np.abs(dc))
        return np.where(dl * dr >= 0, s, 0)
    if limiter is None:
        return 0.5 * (dl + dr)
    raise ValueError(f"unknown slope limiter {limiter}")


def _muscl_faces(w, axis, limiter):
    """Slope-limited p=1 left/right face values along `axis` (fvhoe/slope_limiting.py:24-53)."""
    n = w.shape[axis]

    def sh(k):
        sel = [slice(None)] * w.ndim
        sel[axis] = slice(k, k + n - 2)
        return w[tuple(sel)]

    dl = sh(1) - sh(0)
    dr = sh(2) - sh(1)
    s = _limited_slope(dl, dr, limiter)
    return sh(1) - 0.5 * s, sh(1) + 0.5 * s


# ---------------------------------------------------------------------------
# fluxes (fvhoe/solver.py:456-651, 734-751)
# ---------------------------------------------------------------------------
def hydrofluxes(u: np.ndarray, cfg: OracleConfig, p: Sequence[int], limiter=None):
    """dt and the face fluxes [F, G, H] (None for inactive axes) at degree p.

    Per axis d: centre sweeps along (d+2)%3 then (d+1)%3, left/right face
    sweeps (or MUSCL when limiting at p=1) along d, the Riemann solve between
    cell i's right face and cell i+1's left face, transverse sweeps along the
    two other axes in ascending order, then trimming of the excess ghosts
    (fvhoe/solver.py:491-651).
    """
    act = cfg.active
    if limiter is not None and max(p) > 1:
        raise ValueError("slope limiting needs p <= 1")
    r = stencil_radius(max(p))
    gw = max(r + 1, 2 * r)
    gws = [gw if act[a] else 0 for a in range(3)]
    w_bc = fv_primitives(u, cfg, p, gws)
    dt = cfl_dt(w_bc, cfg) if cfg.fixed_dt is None else cfg.fixed_dt
    fluxes = [None, None, None]
    for d in range(3):
        if not act[d]:
            continue
        a1, a2 = (d + 2) % 3, (d + 1) % 3
        wf = sweep(w_bc, stencil_weights(p[a1], "c"), a1 + 1)
        wf = sweep(wf, stencil_weights(p[a2], "c"), a2 + 1)
        if limiter is not None and p[d] == 1:
            w_l, w_r = _muscl_faces(wf, d + 1, limiter)
        else:
            w_l = sweep(wf, stencil_weights(p[d], "l"), d + 1)
            w_r = sweep(wf, stencil_weights(p[d], "r"), d + 1)
        m = w_r.shape[d + 1]
        sel_l = [slice(None)] * 4
        sel_r = [slice(None)] * 4
        sel_l[d + 1] = slice(0, m - 1)
        sel_r[d + 1] = slice(1, m)
        f = riemann_flux(w_r[tuple(sel_l)], w_l[tuple(sel_r)], d, cfg)
        for t in range(3):
            if t != d:
                f = sweep(f, stencil_weights(p[t], "t"), t + 1)
        trim = [0, 0, 0, 0]
        for a in range(3):
            if not act[a]:
                continue
            ra = stencil_radius(p[a])
            trim[a + 1] = gw - ra - 1 if a == d else gw - 2 * ra
        sel = tuple(slice(t or None, -t or None) for t in trim)
        fluxes[d] = f[sel]
    return dt, fluxes


def flux_divergence(fluxes, cfg: OracleConfig) -> np.ndarray:
    """-(1/h_d)(F_{i+1/2} - F_{i-1/2}) summed over x, y, z (fvhoe/solver.py:734-751)."""
    dudt = 0.0
    for d in range(3):
        f = fluxes[d]
        if f is None or not cfg.active[d]:
            continue
        hi = [slice(None)] * 4
        lo = [slice(None)] * 4
        hi[d + 1] = slice(1, None)
        lo[d + 1] = slice(None, -1)
        dudt += -(1 / cfg.h[d]) * (f[tuple(hi)] - f[tuple(lo)])
    return dudt


# ---------------------------------------------------------------------------
# troubled-cell detection (fvhoe/slope_limiting.py:87-244, SED :8-95 of
# fvhoe/smooth_extrema_detection.py)
# ---------------------------------------------------------------------------
def _sed_line(a: np.ndarray, axis: int, eps: float) -> np.ndarray:
    """alpha along one axis; the result is 6 cells shorter on that axis
    (fvhoe/smooth_extrema_detection.py:8-50)."""

    def sh(x, k, length):
        sel = [slice(None)] * x.ndim
        sel[axis] = slice(k, k + length)
        return x[tuple(sel)]

    n = a.shape[axis]
    du = 0.5 * (sh(a, 2, n - 2) - sh(a, 0, n - 2))
    d2u = 0.5 * (sh(du, 2, n - 4) - sh(du, 0, n - 4))
    dv = 0.5 * d2u
    dv = np.where(np.abs(dv) <= eps, np.where(dv >= 0, eps, -eps), dv)
    v_l = sh(du, 0, n - 4) - sh(du, 1, n - 4)
    alpha_l = -np.where(dv < 0, np.where(v_l > 0, v_l, 0), np.where(v_l < 0, v_l, 0)) / dv
    alpha_l = np.where(alpha_l < 1, alpha_l, 1)
    v_r = sh(du, 2, n - 4) - sh(du, 1, n - 4)
    alpha_r = np.where(dv > 0, np.where(v_r > 0, v_r, 0), np.where(v_r < 0, v_r, 0)) / dv
    alpha_r = np.where(np.abs(dv) <= eps, 1, alpha_r)
    alpha_r = np.where(alpha_r < alpha_l, alpha_r, alpha_l)
    alpha = np.minimum(alpha_l, alpha_r)
    return np.minimum(np.minimum(sh(alpha, 2, n - 6), sh(alpha, 1, n - 6)), sh(alpha, 0, n - 6))


def _crop(a: np.ndarray, axes: Sequence[int], k: int = 3) -> np.ndarray:
    sel = [slice(None)] * a.ndim
    for ax in axes:
        sel[ax] = slice(k, -k)
    return a[tuple(sel)]


def smooth_extrema_alpha(a: np.ndarray, dims: str, eps: float) -> np.ndarray:
    """alpha = min over active axes of the per-axis detector, each computed on
    the interior lines of the other axes (fvhoe/smooth_extrema_detection.py:53-95)."""
    ax = {"x": 1, "y": 2, "z": 3}
    if len(dims) == 1:
        return _sed_line(a, ax[dims], eps)
    if len(dims) == 2:
        a1, a2 = ax[dims[0]], ax[dims[1]]
        return np.minimum(_sed_line(_crop(a, [a2]), a1, eps), _sed_line(_crop(a, [a1]), a2, eps))
    if len(dims) == 3:
        alpha_xy = smooth_extrema_alpha(_crop(a, [3]), "xy", eps)
        alpha_z = _sed_line(_crop(_crop(a, [1]), [2]), 3, eps)
        return np.minimum(alpha_xy, alpha_z)
    raise ValueError(f"invalid dims {dims}")


def _box_extrema(a: np.ndarray, axes: Sequence[int]):
    """3^d neighbourhood max / min, cropped by 3 on the active axes
    (fvhoe/slope_limiting.py:126-162; the constant-0 border of the filter only
    reaches cells that the crop removes)."""
    big = a
    small = a
    for axis in axes:
        n = big.shape[axis]

        def sh(x, k):
            sel = [slice(None)] * x.ndim
            sel[axis] = slice(k, k + n - 2)
            return x[tuple(sel)]

        big = np.maximum(np.maximum(sh(big, 0), sh(big, 1)), sh(big, 2))
        small = np.minimum(np.minimum(sh(small, 0), sh(small, 1)), sh(small, 2))
    return _crop(big, axes, 2), _crop(small, axes, 2)


def detect_trouble(w: np.ndarray, w_star: np.ndarray, cfg: OracleConfig):
    """Troubled cells from FV primitives before (w) and after (w_star) the
    unlimited update, both with 3 ghost cells on the active axes.

    Returns (trouble int64, NAD violation magnitude, PAD violation magnitude),
    each (nx, ny, nz) (fvhoe/slope_limiting.py:87-244). Only the last PAD key
    is effective, as in the reference loop (:229-237).
    """
    dims = cfg.dims
    axes = [1 + "xyz".index(d) for d in dims]
    w_in = _crop(w_star, axes)
    big, small = _box_extrema(w, axes)
    eps = cfg.NAD
    if cfg.NAD_range == "relative":
        if cfg.NAD_mode == "global":
            rng = np.max(w, axis=(1, 2, 3), keepdims=True) - np.min(w, axis=(1, 2, 3), keepdims=True)
        elif cfg.NAD_mode == "local":
            rng = big - small
        else:
            raise ValueError(f"unknown NAD mode {cfg.NAD_mode}")
        ind = w_in - small
        ind = np.minimum(ind, big - w_in)
        nad_v = ind < -eps * rng
    elif cfg.NAD_range == "absolute":
        if cfg.NAD_mode == "global":
            lower = (1 - eps) * np.min(w, axis=(1, 2, 3), keepdims=True)
            upper = (1 + eps) * np.max(w, axis=(1, 2, 3), keepdims=True)
        elif cfg.NAD_mode == "local":
            lower = (1 - eps) * small
            upper = (1 + eps) * big
        else:
            raise ValueError(f"unknown NAD mode {cfg.NAD_mode}")
        ind = np.minimum(w_in - lower, upper - w_in)
        nad_v = ind < 0.0
    else:
        raise ValueError(f"unknown NAD range {cfg.NAD_range}")
    if cfg.SED:
        alpha = smooth_extrema_alpha(w_star, dims, cfg.SED_tolerance)
        nad_v = np.where(alpha < 1, nad_v, 0)
    if cfg.NAD_vars is not None:
        keep = np.zeros((5, 1, 1, 1))
        keep[np.array([VARIABLE_INDEX[v] for v in cfg.NAD_vars])] = 1
        nad_v = np.where(keep, nad_v, 0)
    nad = np.any(nad_v, axis=0)
    nad_mag = np.where(nad, -np.min(ind, axis=0), 0)
    pad_ind = np.zeros_like(nad_mag)
    if cfg.PAD is not None:
        for var, (lo, hi) in cfg.PAD.items():
            pad_ind = w_in[VARIABLE_INDEX[var]] - lo
            pad_ind = np.minimum(pad_ind, hi - w_in[VARIABLE_INDEX[var]])
    pad = np.where(pad_ind < 0.0, 1, 0)
    pad_mag = np.where(pad, -pad_ind, 0)
    trouble = np.where(pad, 1, nad)
    return trouble, nad_mag, pad_mag


def face_trouble(trouble: np.ndarray, cfg: OracleConfig):
    """Face weights theta per axis, shape (1, n_d + 1, ...) (fvhoe/slope_limiting.py:247-442).

    Simple mode: a face is troubled when either neighbour is (:364-380).
    Convex mode (1D/2D): graded weights 1, 0.75, 0.5, 0.25 (:281-363, 387-442).
    """
    nx, ny, nz = trouble.shape
    tx = np.zeros((nx + 1, ny, nz))
    ty = np.zeros((nx, ny + 1, nz))
    tz = np.zeros((nx, ny, nz + 1))
    dims = cfg.dims
    if cfg.convex:
        _convex_faces(trouble, cfg, tx, ty, tz)
    else:
        if "x" in dims:
            tx[1:] = trouble
            tx[:-1] = np.maximum(tx[:-1], trouble)
        if "y" in dims:
            ty[:, 1:] = trouble
            ty[:, :-1] = np.maximum(ty[:, :-1], trouble)
        if "z" in dims:
            tz[:, :, 1:] = trouble
            tz[:, :, :-1] = np.maximum(tz[:, :, :-1], trouble)
    return tx[np.newaxis], ty[np.newaxis], tz[np.newaxis]


def _convex_faces(trouble, cfg, tx, ty, tz):
    dims = cfg.dims
    act = [d in dims for d in "xyz"]
    shape = [s + 4 if a else 1 for s, a in zip(trouble.shape, act)]
    t = np.zeros(shape)
    t[tuple(slice(2, -2) if a else slice(None) for a in act)] = trouble
    periodic = [cfg.bc[a] == ("periodic", "periodic") for a in range(3)]
    if periodic[0] and act[0]:
        t[:2, 2:-2, 2:-2] = trouble[-2:, :, :]
        t[-2:, 2:-2, 2:-2] = trouble[:2, :, :]
    if periodic[1] and act[1]:
        t[2:-2, :2, 2:-2] = trouble[:, -2:, :]
        t[2:-2, -2:, 2:-2] = trouble[:, :2, :]
    if periodic[2] and act[2]:
        t[2:-2, 2:-2, :2] = trouble[2:-2, 2:-2, -2:]
        t[2:-2, 2:-2, -2:] = trouble[2:-2, 2:-2, :2]
    sel = [0, 0, 0]
    nact = sum(act)
    if nact == 1:
        sel["xyz".index(dims)] = slice(None)
        line = t[tuple(sel)]
        th = line.copy()
        th[:-1] = np.maximum(0.75 * line[1:], th[:-1])
        th[1:] = np.maximum(0.75 * line[:-1], th[1:])
        th[:-1] = np.maximum(0.25 * (th[1:] > 0), th[:-1])
        th[1:] = np.maximum(0.25 * (th[:-1] > 0), th[1:])
        faces = np.maximum(th[1:-2], th[2:-1])
        target = {"x": tx, "y": ty, "z": tz}[dims]
        shp = [1, 1, 1]
        shp["xyz".index(dims)] = -1
        target[...] = faces.reshape(shp)
    elif nact == 2:
        d1, d2 = dims[0], dims[1]
        sel["xyz".index(d1)] = slice(None)
        sel["xyz".index(d2)] = slice(None)
        plane = t[tuple(sel)]
        th = plane.copy()
        th[:, :-1] = np.maximum(0.75 * plane[:, 1:], th[:, :-1])
        th[:, 1:] = np.maximum(0.75 * plane[:, :-1], th[:, 1:])
        th[:-1, :] = np.maximum(0.75 * plane[1:, :], th[:-1, :])
        th[1:, :] = np.maximum(0.75 * plane[:-1, :], th[1:, :])
        th[:-1, :-1] = np.maximum(0.5 * plane[1:, 1:], th[:-1, :-1])
        th[:-1, 1:] = np.maximum(0.5 * plane[1:, :-1], th[:-1, 1:])
        th[1:, :-1] = np.maximum(0.5 * plane[:-1, 1:], th[1:, :-1])
        th[1:, 1:] = np.maximum(0.5 * plane[:-1, :-1], th[1:, 1:])
        th[:, :-1] = np.maximum(0.25 * (th[:, 1:] > 0), th[:, :-1])
        th[:, 1:] = np.maximum(0.25 * (th[:, :-1] > 0), th[:, 1:])
        th[:-1, :] = np.maximum(0.25 * (th[1:, :] > 0), th[:-1, :])
        th[1:, :] = np.maximum(0.25 * (th[:-1, :] > 0), th[1:, :])
        f1 = np.maximum(th[2:-1, 2:-2], th[1:-2, 2:-2])
        f2 = np.maximum(th[2:-2, 2:-1], th[2:-2, 1:-2])
        nx, ny, nz = trouble.shape
        if dims in ("xy", "yx"):
            tx[...] = f1.reshape(nx + 1, ny, 1)
            ty[...] = f2.reshape(nx, ny + 1, 1)
        elif dims in ("yz", "zy"):
            ty[...] = f1.reshape(1, ny + 1, nz)
            tz[...] = f2.reshape(1, ny, nz + 1)
        else:
            tx[...] = f1.reshape(nx + 1, 1, nz)
            tz[...] = f2.reshape(nx, 1, nz + 1)
    else:
        raise NotImplementedError("3D convex broadcast not implemented")


# ---------------------------------------------------------------------------
# one RHS evaluation (fvhoe/solver.py:422-454, 653-732)
# ---------------------------------------------------------------------------
def rhs(u: np.ndarray, cfg: OracleConfig, predicted: Optional[np.ndarray] = None):
    """(dt, dudt, info) for one stage.

    info holds the high-order fluxes, the candidate, the detector outputs and
    the face weights when a-posteriori limiting is on (fvhoe/solver.py:429-454).
    `predicted` (bool, (nx, ny, nz)) adds cells whose faces take the fallback
    flux whatever the check says: the learned predictor's mode, which has no
    counterpart in the reference; the detector outputs stay the check's.
    """
    dt, fluxes = hydrofluxes(u, cfg, cfg.p)
    info = {"dt": dt}
    if cfg.a_posteriori_slope_limiting:
        act = cfg.active
        ustar = u + dt * flux_divergence(fluxes, cfg)
        g3 = [3 if act[a] else 0 for a in range(3)]
        w = fv_primitives(u, cfg, cfg.p, g3)
        w_star = fv_primitives(ustar, cfg, cfg.p, g3)
        trouble, nad_mag, pad_mag = detect_trouble(w[:5], w_star[:5], cfg)
        if cfg.force_trouble:
            trouble = np.ones_like(trouble, dtype=bool)
        info.update(ustar=ustar, trouble=trouble, nad_mag=nad_mag, pad_mag=pad_mag)
        blend = trouble if predicted is None else (trouble | np.asarray(predicted, dtype=bool))
        if np.any(blend):
            p_fb = tuple(int(cfg.p[a] > 0) for a in range(3))
            _, low = hydrofluxes(u, cfg, p_fb, limiter=cfg.slope_limiter)
            thetas = face_trouble(blend, cfg)
            for d in range(3):
                if act[d]:
                    fluxes[d] = (1 - thetas[d]) * fluxes[d] + thetas[d] * low[d]
            info["theta"] = thetas
    info["fluxes"] = fluxes
    return dt, flux_divergence(fluxes, cfg), info


# ---------------------------------------------------------------------------
# SSP-RK steppers (fvhoe/ode.py:11-22, 245-298)
# ---------------------------------------------------------------------------
def hit_target(t: float, dt: float, target: Optional[float]) -> float:
    """Shorten dt so that t + dt does not pass the target (fvhoe/ode.py:11-22)."""
    if target is not None and target - t < dt:
        return target - t
    return dt


def step(u: np.ndarray, t: float, cfg: OracleConfig, integrator: str = "ssprk3", target=None):
    """One time step; returns (dt, u_next, per-stage infos) (fvhoe/ode.py:245-298).
    Boundary functions see the step's start time in every stage (fvhoe/solver.py:784)."""
    from dataclasses import replace

    cfg = replace(cfg, t=t)
    infos = []

    def f(x):
        dt_, k_, info_ = rhs(x, cfg)
        infos.append(info_)
        return dt_, k_

    if integrator == "euler":
        dt, k0 = f(u)
        dt = hit_target(t, dt, target)
        return dt, u + dt * k0, infos
    if integrator == "ssprk2":
        dt, k0 = f(u)
        dt = hit_target(t, dt, target)
        u1 = u + dt * k0
        _, k1 = f(u1)
        return dt, 0.5 * u + 0.5 * (u1 + dt * k1), infos
    if integrator == "ssprk3":
        dt, k0 = f(u)
        dt = hit_target(t, dt, target)
        _, k1 = f(u + dt * k0)
        _, k2 = f(u + 0.25 * dt * k0 + 0.25 * dt * k1)
        return dt, u + (1 / 6) * dt * (k0 + k1 + 4 * k2), infos
    if integrator == "rk4":
        dt, k0 = f(u)
        dt = hit_target(t, dt, target)
        _, k1 = f(u + 0.5 * dt * k0)
        _, k2 = f(u + 0.5 * dt * k1)
        _, k3 = f(u + dt * k2)
        return dt, u + (1 / 6) * dt * (k0 + 2 * k1 + 2 * k2 + k3), infos
    raise ValueError(f"unknown integrator {integrator}")
