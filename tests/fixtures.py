"""Helpers shared by the tests: golden fixtures, oracle configs, solver builders."""

import glob
import json
import os

import numpy as np

from oracle import fvh_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _bc_values_module():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bc_values", os.path.join(GOLDEN, "bc_values.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def fixture_ic(c):
    """The initial-condition object a fixture names (for its "ic" boundaries), or None."""
    spec = c.get("ic_spec")
    if not spec:
        return None
    import fvhoe_b200 as F

    cls = {"Shock1D": F.Shock1D, "Sinus": F.Sinus, "FourQuadrant": F.FourQuadrant2D}[spec["cls"]]
    return cls(**spec["kwargs"])


def pointwise_u0(c):
    """The pointwise conserved initial condition u0(x, y, z) of a fixture with an ic_spec."""
    from fvhoe_b200.hydro import HydroState, compute_conservatives

    ic = fixture_ic(c).build_ic(HydroState(), None)
    return lambda x, y, z: compute_conservatives(HydroState(), ic(x, y, z), gamma=c["gamma"])


def bc_values(c, for_oracle=False):
    """Per axis, the (low, high) boundary values of a fixture: arrays or functions
    for "dirichlet" sides; for the oracle, also u0 for "ic" sides."""
    names = c.get("bc_values") or [[None, None]] * 3
    mod = _bc_values_module()
    out = []
    for a in range(3):
        pair = []
        for s in range(2):
            if for_oracle and c["bc"][a][s] == "ic":
                pair.append(pointwise_u0(c))
            else:
                pair.append(mod.resolve(names[a][s]))
        out.append(tuple(pair))
    return tuple(out)


def golden_files(kind=None):
    pat = "*.npz" if kind is None else f"{kind}_*.npz"
    return sorted(glob.glob(os.path.join(GOLDEN, pat)))


def load(path):
    d = np.load(path)
    cfg = json.loads(str(d["config"]))
    return cfg, {k: d[k] for k in d.files if k != "config"}


def pad_from_json(pad):
    if pad is None:
        return None
    conv = {"inf": np.inf, "-inf": -np.inf}
    return {k: tuple(conv.get(v, v) if isinstance(v, str) else float(v) for v in b) for k, b in pad.items()}


def oracle_config(c) -> O.OracleConfig:
    return O.OracleConfig(
        n=tuple(c["n"]), p=tuple(c["p"]), h=tuple(c["h"]), nvars=c["nvars"], gamma=c["gamma"], CFL=c["CFL"],
        fixed_dt=c["fixed_dt"], riemann_solver=c["riemann_solver"], bc=tuple(tuple(b) for b in c["bc"]),
        a_posteriori_slope_limiting=c["a_posteriori_slope_limiting"], slope_limiter=c["slope_limiter"],
        force_trouble=c["force_trouble"], NAD=c["NAD"], NAD_mode=c["NAD_mode"], NAD_range=c["NAD_range"],
        NAD_vars=tuple(c["NAD_vars"]) if c["NAD_vars"] else None, PAD=pad_from_json(c["PAD"]), SED=c["SED"],
        SED_tolerance=c["SED_tolerance"], convex=c["convex"], csq_floor=c["csq_floor"],
        domain=tuple(tuple(d) for d in c["domain"]), bc_values=bc_values(c, for_oracle=True),
        slab_buffer_size=c.get("slab_buffer_size", 30),
    )


def solver_kwargs(c, u0, **extra):
    """EulerSolver arguments reproducing a fixture's problem from its stored initial state."""
    from fvhoe_b200 import ArrayIC, BoundaryCondition

    bc = c["bc"]
    vals = bc_values(c)
    ic = fixture_ic(c)
    kw = dict(
        w0=ArrayIC(array=u0[:5]) if ic is None else ic, conservative_ic=ic is None, fv_ic=ic is None,
        nx=c["n"][0], ny=c["n"][1], nz=c["n"][2], px=c["p"][0], py=c["p"][1], pz=c["p"][2],
        x=tuple(c["domain"][0]), y=tuple(c["domain"][1]), z=tuple(c["domain"][2]),
        CFL=c["CFL"], fixed_dt=c["fixed_dt"], gamma=c["gamma"],
        bc=BoundaryCondition(x=tuple(bc[0]), y=tuple(bc[1]), z=tuple(bc[2]), x_value=vals[0], y_value=vals[1],
                             z_value=vals[2]),
        riemann_solver=c["riemann_solver"], a_posteriori_slope_limiting=c["a_posteriori_slope_limiting"],
        slope_limiter=c["slope_limiter"], force_trouble=c["force_trouble"], NAD=c["NAD"], NAD_mode=c["NAD_mode"],
        NAD_range=c["NAD_range"], NAD_vars=tuple(c["NAD_vars"]) if c["NAD_vars"] else None,
        PAD=pad_from_json(c["PAD"]), SED=c["SED"], SED_tolerance=c["SED_tolerance"], convex=c["convex"],
        csq_floor=c["csq_floor"], progress_bar=False,
    )
    if c["nvars"] > 5:
        names = [f"s{i}" for i in range(c["nvars"] - 5)]
        kw["w0_passives"] = {nm: (lambda x, y, z: np.zeros_like(x)) for nm in names}
        kw["w0"] = _FullArrayIC(u0)
    kw.update(extra)
    return kw


class _FullArrayIC:
    """IC object returning a stored conserved array including passive scalars."""

    def __init__(self, u0):
        self.u0 = np.asarray(u0, dtype=np.float64)

    def build_ic(self, hs, passive_ic_funcs=None):
        arr = self.u0

        def ic_func(x, y, z):
            return arr.copy()

        return ic_func
