"""Helpers shared by the tests: golden fixtures, oracle configs, solver builders."""

import glob
import json
import os

import numpy as np

from oracle import fvh_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


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
    )


def solver_kwargs(c, u0, **extra):
    """EulerSolver arguments reproducing a fixture's problem from its stored initial state."""
    from fvhoe_b200 import ArrayIC, BoundaryCondition

    bc = c["bc"]
    kw = dict(
        w0=ArrayIC(array=u0[:5]), conservative_ic=True, fv_ic=True,
        nx=c["n"][0], ny=c["n"][1], nz=c["n"][2], px=c["p"][0], py=c["p"][1], pz=c["p"][2],
        x=tuple(c["domain"][0]), y=tuple(c["domain"][1]), z=tuple(c["domain"][2]),
        CFL=c["CFL"], fixed_dt=c["fixed_dt"], gamma=c["gamma"],
        bc=BoundaryCondition(x=tuple(bc[0]), y=tuple(bc[1]), z=tuple(bc[2])),
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
