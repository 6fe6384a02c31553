"""Generate the golden fixtures under tests/golden/ by running the reference.

Run in a checkout where the reference FVHOE package is importable:

    python tests/golden/make_golden.py --reference <FVHOE checkout>

(or set FVHOE_REFERENCE to the checkout instead of passing --reference).

The reference imports matplotlib for plotting only; a placeholder package in
tests/golden/_mpl_stub stands in for it. Every fixture stores the solver
settings (as JSON), the initial conserved state and the reference's outputs,
so tests on machines without the reference can rebuild the same problem.

Outputs:
  rhs_<name>.npz    one right-hand-side evaluation: dt, dudt, trouble, NAD/PAD
                    magnitudes (when a-posteriori limiting is on)
  steps_<name>.npz  a few time steps: u after each step, dt per step and the
                    trouble flags of every stage
"""

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _setup(reference):
    sys.path.insert(0, reference)
    sys.path.insert(0, os.path.join(HERE, "_mpl_stub"))
    sys.path.insert(0, HERE)


def _patch_dmr_free_bc():
    """Let the reference's double-Mach-reflection branch run.

    That branch (fvhoe/boundary_conditions.py:374-395) calls
    _set_free_bc(u, slab_thickness, axis=..., pos=...) without the HydroState
    argument the function takes first (:60-85), so it raises TypeError. The
    wrapper installed here supplies a HydroState for such calls and leaves
    every other call alone; the branch's own free and reflective fills and
    its per-column combination then produce the fixture."""
    import fvhoe.boundary_conditions as bcm
    from fvhoe.hydro import HydroState

    orig = bcm._set_free_bc
    if getattr(orig, "dmr_patched", False):
        return

    def set_free_bc(*args, **kwargs):
        if args and isinstance(args[0], np.ndarray):
            return orig(HydroState(), *args, **kwargs)
        return orig(*args, **kwargs)

    set_free_bc.dmr_patched = True
    bcm._set_free_bc = set_free_bc


def _json_pad(pad):
    if pad is None:
        return None
    return {k: [("inf" if v == np.inf else "-inf" if v == -np.inf else v) for v in b] for k, b in pad.items()}


def build_cases():
    from fvhoe.initial_conditions import (
        DoubleMachReflection2D,
        DoubleShock1D,
        InitialCondition,
        SedovBlast,
        Shock1D,
        Sinus,
    )

    class KelvinHelmholtzNoise(InitialCondition):
        """rho=2, vx=+0.5 in |y-0.5|<0.25 else rho=1, vx=-0.5; P=2.5;
        vy = 0.01 sin(4 pi x) + per-cell uniform noise of amplitude 1e-3."""

        def base_ic(self, n=(32, 32), seed=0, amp=1e-3):
            noise = np.random.default_rng(seed).uniform(-amp, amp, size=n)

            def f(x, y, z):
                ix = np.clip(np.floor(x * n[0]).astype(int), 0, n[0] - 1)
                iy = np.clip(np.floor(y * n[1]).astype(int), 0, n[1] - 1)
                inner = np.abs(y - 0.5) < 0.25
                out = np.empty((5,) + x.shape)
                out[0] = np.where(inner, 2.0, 1.0)
                out[1] = np.where(inner, 0.5, -0.5)
                out[2] = 0.01 * np.sin(4 * np.pi * x) + noise[ix, iy]
                out[3] = 0.0
                out[4] = 2.5
                return out

            return f

    class FourQuadrant(InitialCondition):
        """Four constant states split at (xs, ys); states drawn from a seed."""

        def base_ic(self, seed=0):
            rng = np.random.default_rng(seed)
            xs, ys = rng.uniform(0.3, 0.7, size=2)
            rho = np.exp(rng.uniform(np.log(0.1), np.log(2.0), size=4))
            P = np.exp(rng.uniform(np.log(0.01), np.log(10.0), size=4))
            vx = rng.uniform(-1, 1, size=4)
            vy = rng.uniform(-1, 1, size=4)

            def f(x, y, z):
                q = (x >= xs).astype(int) + 2 * (y >= ys).astype(int)
                out = np.empty((5,) + x.shape)
                out[0] = rho[q]
                out[1] = vx[q]
                out[2] = vy[q]
                out[3] = 0.0
                out[4] = P[q]
                return out

            return f

    def shock(dim):
        return Shock1D(dim=dim)

    cases = []

    def add(kind, name, ic, n, p, steps=0, integrator="ssprk3", **kw):
        cases.append(dict(kind=kind, name=name, ic=ic, n=n, p=p, steps=steps, integrator=integrator, kw=kw))

    lim = dict(a_posteriori_slope_limiting=True, NAD=1e-5)
    # 1D Sod-type shocks along each axis, every degree
    for p in range(9):
        add("rhs", f"shock_x_p{p}", shock("x"), (64, 1, 1), (p, 0, 0), gamma=1.4,
            bc=dict(x="outflow"), riemann_solver="hllc", **(lim if p > 0 else {}))
    for dim in "yz":
        n = tuple(64 if d == dim else 1 for d in "xyz")
        p = tuple(5 if d == dim else 0 for d in "xyz")
        add("rhs", f"shock_{dim}_p5", shock(dim), n, p, gamma=1.4,
            bc={dim: "outflow"}, riemann_solver="hllc", **lim)
    add("rhs", "doubleshock_x_p8_llf", DoubleShock1D(dim="x"), (100, 1, 1), (8, 0, 0), gamma=1.4,
        bc=dict(x="reflective"), riemann_solver="llf", a_posteriori_slope_limiting=True)
    add("rhs", "doubleshock_x_p7_hllc_convex", DoubleShock1D(dim="x"), (100, 1, 1), (7, 0, 0), gamma=1.4,
        bc=dict(x="reflective"), riemann_solver="hllc", a_posteriori_slope_limiting=True, convex=True)
    add("rhs", "sinus_x_p3_upwind", Sinus(dims="x", vx=1), (64, 1, 1), (3, 0, 0),
        riemann_solver="advection_upwind", fixed_dt=0.004)
    add("rhs", "shock_x_p3_free_passives", shock("x"), (64, 1, 1), (3, 0, 0), gamma=1.4,
        bc=dict(x="free"), riemann_solver="hllc", passives=True, **lim)
    add("rhs", "shock_x_p3_moncen", shock("x"), (64, 1, 1), (3, 0, 0), gamma=1.4,
        bc=dict(x="outflow"), riemann_solver="hllc", slope_limiter="moncen", **lim)
    # 2D Kelvin-Helmholtz with noise
    kh = lambda n: KelvinHelmholtzNoise(n=n[:2], seed=7)  # noqa: E731
    for p in (2, 3, 5, 7):
        add("rhs", f"kh_p{p}", kh((32, 32, 1)), (32, 32, 1), (p, p, 0), gamma=1.4,
            riemann_solver="hllc", **lim)
    add("rhs", "kh_p5_llf", kh((32, 32, 1)), (32, 32, 1), (5, 5, 0), gamma=1.4, riemann_solver="llf", **lim)
    add("rhs", "kh_p3_rect", kh((40, 24, 1)), (40, 24, 1), (3, 3, 0), gamma=1.4, riemann_solver="hllc", **lim)
    for mode, rng in (("global", "absolute"), ("local", "relative"), ("local", "absolute")):
        add("rhs", f"kh_p3_{mode}_{rng}", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), gamma=1.4,
            riemann_solver="hllc", a_posteriori_slope_limiting=True, NAD=1e-3, NAD_mode=mode, NAD_range=rng)
    add("rhs", "kh_p3_nadvars", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), gamma=1.4,
        riemann_solver="hllc", NAD_vars=("rho", "P"), **lim)
    add("rhs", "kh_p3_pad_rho", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), gamma=1.4,
        riemann_solver="hllc", PAD={"P": (0.0, np.inf), "rho": (1.2, 1.8)}, **lim)
    add("rhs", "kh_p3_nosed", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), gamma=1.4,
        riemann_solver="hllc", SED=False, **lim)
    add("rhs", "kh_p3_force", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), gamma=1.4,
        riemann_solver="hllc", force_trouble=True, **lim)
    add("rhs", "kh_p3_convex", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), gamma=1.4,
        riemann_solver="hllc", convex=True, **lim)
    # 2D Sedov in each plane, reflective at the low walls
    for dims in ("xy", "yz", "zx"):
        n = tuple(32 if d in dims else 1 for d in "xyz")
        p = tuple(3 if d in dims else 0 for d in "xyz")
        add("rhs", f"sedov_{dims}_p3", SedovBlast(dims=dims), n, p, gamma=1.4, conservative_ic=True, fv_ic=True,
            bc={d: ("reflective", "outflow") for d in dims}, riemann_solver="hllc",
            a_posteriori_slope_limiting=True)
    # four quadrants
    add("rhs", "quad_p3", FourQuadrant(seed=3), (32, 32, 1), (3, 3, 0), gamma=1.4,
        bc=dict(x="outflow", y="outflow"), riemann_solver="hllc", CFL=0.8, **lim)
    # 3D Sedov, reflective at the origin walls, outflow elsewhere
    s3 = dict(gamma=1.4, conservative_ic=True, fv_ic=True,
              bc=dict(x=("reflective", "outflow"), y=("reflective", "outflow"), z=("reflective", "outflow")))
    add("rhs", "sedov3d_p3_llf", SedovBlast(dims="xyz"), (12, 12, 12), (3, 3, 3), riemann_solver="llf",
        CFL=0.5, a_posteriori_slope_limiting=True, **s3)
    add("rhs", "sedov3d_p2_hllc", SedovBlast(dims="xyz"), (12, 12, 12), (2, 2, 2), riemann_solver="hllc",
        a_posteriori_slope_limiting=True, **s3)
    add("rhs", "sedov3d_p5_hllc", SedovBlast(dims="xyz"), (14, 13, 12), (5, 5, 5), riemann_solver="hllc",
        a_posteriori_slope_limiting=True, **s3)
    # multi-step runs
    add("steps", "sod_full", shock("x"), (256, 1, 1), (3, 0, 0), steps=-1, gamma=1.4,
        bc=dict(x="outflow"), riemann_solver="hllc", CFL=0.8, T=0.245, **lim)
    add("steps", "kh64_p5", kh((64, 64, 1)), (64, 64, 1), (5, 5, 0), steps=2, gamma=1.4,
        riemann_solver="hllc", **lim)
    add("steps", "sedov3d16_p3", SedovBlast(dims="xyz"), (16, 16, 16), (3, 3, 3), steps=2, riemann_solver="llf",
        CFL=0.5, a_posteriori_slope_limiting=True, **s3)
    add("steps", "quad48_p3", FourQuadrant(seed=11), (48, 48, 1), (3, 3, 0), steps=2, gamma=1.4,
        bc=dict(x="outflow", y="outflow"), riemann_solver="hllc", **lim)
    for integ in ("euler", "ssprk2", "rk4"):
        add("steps", f"shock_x_p2_{integ}", shock("x"), (64, 1, 1), (2, 0, 0), steps=3, integrator=integ,
            gamma=1.4, bc=dict(x="outflow"), riemann_solver="hllc", **lim)
    # Dirichlet and "ic" boundaries (values named in bc_values.py; "ic" sides use the
    # initial condition named by ic_spec)
    add("steps", "sod_ic", shock("x"), (128, 1, 1), (3, 0, 0), steps=-1, gamma=1.4, bc=dict(x="ic"),
        riemann_solver="hllc", CFL=0.8, T=0.1, ic_spec=dict(cls="Shock1D", kwargs=dict(dim="x")), **lim)
    add("rhs", "quad_p3_dirichlet", FourQuadrant(seed=5), (32, 32, 1), (3, 3, 0), gamma=1.4,
        bc=dict(x=("dirichlet", "outflow"), y=("outflow", "free"), x_value=("inflow_state", None)),
        riemann_solver="hllc", **lim)
    add("rhs", "quad_p3_ic_wall", FourQuadrant(seed=6), (32, 40, 1), (3, 3, 0), gamma=1.4,
        bc=dict(x="ic", y=("outflow", "dirichlet"), y_value=(None, "wall_y_high")), riemann_solver="hllc",
        ic_spec=dict(cls="FourQuadrant", kwargs=dict(seed=6)), **lim)
    add("steps", "kh_dirichlet_t", kh((32, 32, 1)), (32, 32, 1), (3, 3, 0), steps=3, gamma=1.4,
        bc=dict(x="periodic", y="dirichlet", y_value=("wall_y_low", "wall_y_high")), riemann_solver="hllc", **lim)
    add("rhs", "box3d_dirichlet", Sinus(dims="xyz", vx=0.5, vy=0.25, vz=-0.3), (10, 12, 14), (2, 2, 2),
        gamma=1.4, bc=dict(x=("dirichlet", "outflow"), y=("reflective", "free"), z=("ic", "dirichlet"),
                           x_value=("box_x_low", None), z_value=(None, "box_z_high")),
        riemann_solver="hllc", ic_spec=dict(cls="Sinus", kwargs=dict(dims="xyz", vx=0.5, vy=0.25, vz=-0.3)), **lim)
    # the double Mach reflection's walls: inflow on the low x side, the
    # free/reflective wall on the low y side, the moving shock on the high y side
    dmr = dict(x=("dirichlet", "outflow"), y=("special-case-double-mach-reflection-y=0", "dirichlet"),
               x_value=("dmr_inflow", None), y_value=(None, "dmr_top"))
    add("rhs", "dmr_p3", DoubleMachReflection2D(), (48, 12, 1), (3, 3, 0), gamma=1.4, bc=dmr,
        domain=((0, 4), (0, 1), (0, 1)), riemann_solver="hllc", **lim)
    add("rhs", "dmr_p7_llf", DoubleMachReflection2D(), (40, 20, 1), (7, 7, 0), gamma=1.4, bc=dmr,
        domain=((0, 4), (0, 1), (0, 1)), riemann_solver="llf", **lim)
    add("steps", "dmr_p3", DoubleMachReflection2D(), (48, 12, 1), (3, 3, 0), steps=3, gamma=1.4, bc=dmr,
        domain=((0, 4), (0, 1), (0, 1)), riemann_solver="hllc", **lim)
    # the wall in 3D (z periodic), where z ghosts are filled after it
    add("rhs", "dmr3d_p2", DoubleMachReflection2D(), (24, 12, 8), (2, 2, 2), gamma=1.4, bc=dict(dmr, z="periodic"),
        domain=((0, 2), (0, 1), (0, 0.5)), riemann_solver="hllc", **lim)
    return cases


def run_case(case, outdir):
    from fvhoe.boundary_conditions import BoundaryCondition
    from fvhoe.solver import EulerSolver

    import bc_values

    kw = dict(case["kw"])
    T = kw.pop("T", None)
    passives = kw.pop("passives", False)
    ic_spec = kw.pop("ic_spec", None)
    bc_kw = kw.pop("bc", None)
    bc_names = [[None, None], [None, None], [None, None]]
    if bc_kw is not None:
        bc_kw = dict(bc_kw)
        for a, dim in enumerate("xyz"):
            names = bc_kw.pop(f"{dim}_value", None)
            if names is None:
                continue
            names = names if isinstance(names, tuple) else (names, names)
            bc_names[a] = list(names)
            bc_kw[f"{dim}_value"] = tuple(bc_values.resolve(nm) for nm in names)
    nx, ny, nz = case["n"]
    px, py, pz = case["p"]
    domain = kw.pop("domain", ((0, 1), (0, 1), (0, 1)))
    solver_kw = dict(
        w0=case["ic"], nx=nx, ny=ny, nz=nz, px=px, py=py, pz=pz,
        x=domain[0], y=domain[1], z=domain[2], progress_bar=False,
    )
    if bc_kw is not None:
        solver_kw["bc"] = BoundaryCondition(**bc_kw)
    if passives:
        solver_kw["w0_passives"] = {
            "tracer1": lambda x, y, z: np.sin(2 * np.sin(8 * x)),
            "tracer2": lambda x, y, z: 1 + 0.5 * np.cos(2 * np.sin(8 * x)),
        }
    solver_kw.update(kw)
    solver = EulerSolver(**solver_kw)

    logged = []
    orig_log = solver.log_troubles

    def log_troubles(trouble=None, NAD_violation_magnitude=None, PAD_violation_magnitude=None, reset=False):
        if not reset:
            logged.append((np.array(trouble, dtype=np.int8), np.array(NAD_violation_magnitude),
                           np.array(PAD_violation_magnitude)))
        return orig_log(trouble, NAD_violation_magnitude, PAD_violation_magnitude, reset=reset)

    solver.log_troubles = log_troubles

    bc = solver.bc
    config = dict(
        n=[nx, ny, nz], p=[px, py, pz], h=list(solver.h),
        domain=[list(d) for d in domain],
        nvars=solver.nvars, gamma=solver.gamma, CFL=solver.CFL, fixed_dt=solver.fixed_dt,
        riemann_solver=solver.riemann_solver_name,
        bc=[list(bc.x), list(bc.y), list(bc.z)],
        a_posteriori_slope_limiting=solver.a_posteriori_slope_limiting,
        slope_limiter=solver.slope_limiter, force_trouble=solver.force_trouble,
        NAD=solver.NAD, NAD_mode=solver.NAD_mode, NAD_range=solver.NAD_range,
        NAD_vars=list(solver.NAD_vars) if solver.NAD_vars is not None else None,
        PAD=_json_pad(solver.PAD), SED=solver.SED, SED_tolerance=solver.SED_tolerance,
        convex=solver.convex, csq_floor=solver.csq_floor, integrator=case["integrator"],
        bc_values=bc_names, ic_spec=ic_spec, slab_buffer_size=solver.slab_buffer_size,
    )
    u0 = solver.am.get_numpy("u")
    out = dict(config=np.array(json.dumps(config)), u0=u0)
    if case["kind"] == "rhs":
        dt, dudt = solver.f(0.0, u0.copy())
        out.update(dt=np.array(dt), dudt=dudt)
        if logged:
            tr, nad, pad = logged[0]
            out.update(trouble=tr, nad_mag=nad, pad_mag=pad)
    else:
        stepper = getattr(solver, case["integrator"])
        if case["steps"] < 0:
            stepper(T)
        else:
            stepper(n=case["steps"])
        ts = np.array(solver.timestamps)
        out.update(u_final=solver.am.get_numpy("u"), timestamps=ts, steps=np.array(solver.step_count))
        if case["steps"] > 0 and logged:
            out.update(trouble_stages=np.stack([t for t, _, _ in logged]))
        if case["steps"] < 0:
            out.update(w_final=solver.snapshots[-1]["w"], T=np.array(T))
            if logged:
                # per-stage flag counts of the whole run (a compact fingerprint)
                out.update(trouble_counts=np.array([int(t.sum()) for t, _, _ in logged]))
                out.update(trouble_stages_first=np.stack([t for t, _, _ in logged[:9]]))
    path = os.path.join(outdir, f"{case['kind']}_{case['name']}.npz")
    np.savez_compressed(path, **out)
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FVHOE_REFERENCE"),
                    help="the FVHOE checkout to run (default: $FVHOE_REFERENCE)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.reference:
        ap.error("name the FVHOE checkout with --reference or FVHOE_REFERENCE")
    _setup(args.reference)
    _patch_dmr_free_bc()
    cases = build_cases()
    for case in cases:
        if args.only and args.only not in case["name"]:
            continue
        path = run_case(case, HERE)
        print(f"{os.path.basename(path)}: {os.path.getsize(path) / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
