"""C ABI and host-side logic without a GPU.

The library must load and export every symbol include/fvh.h declares; its
configuration checks run on the host before any device work; the Python host
classes keep the reference's interfaces and errors.
"""

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    text = open(os.path.join(ROOT, "include", "fvh.h")).read()
    return sorted(set(re.findall(r"\b(fvh_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    from fvhoe_b200 import _capi

    declared = _header_functions()
    assert len(declared) >= 12
    missing = [name for name in declared if not hasattr(_capi.lib, name)]
    assert not missing, missing
    assert set(declared) == set(_capi.EXPORTS)


def test_config_struct_layout_matches_header(tmp_path):
    from fvhoe_b200 import _capi

    src = tmp_path / "size.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fvh.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %d %d %d\\n", sizeof(fvh_config),'
                   ' offsetof(fvh_config, dmr_split), offsetof(fvh_config, pad_hi), sizeof(fvh_stats),'
                   ' sizeof(fvh_pred_stats), FVH_KK_COUNT, FVH_MLP_FEATURES, FVH_MLP_ROW);return 0;}\n')
    exe = tmp_path / "size"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()
    size, split, pad_hi, stats, pstats, kinds, feats, row = map(int, out)
    assert size == ctypes.sizeof(_capi.FvhConfig)
    assert split == _capi.FvhConfig.dmr_split.offset
    assert pad_hi == _capi.FvhConfig.pad_hi.offset
    assert stats == ctypes.sizeof(_capi.FvhStats)
    assert pstats == ctypes.sizeof(_capi.FvhPredStats)
    assert kinds == len(_capi.KERNEL_KINDS)
    assert (feats, row) == (_capi.MLP_FEATURES, _capi.MLP_ROW)


def test_predictor_entry_points_refuse_null_arguments():
    from fvhoe_b200 import _capi
    from oracle import mlp_oracle

    assert _capi.lib.fvh_mlp_param_count() == mlp_oracle.N_PARAMS
    assert _capi.lib.fvh_mlp_create(0, 0, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_mlp_destroy(None) == _capi.OK
    assert _capi.lib.fvh_mlp_get_params(None, None, 0) == _capi.ERR_ARG
    assert _capi.lib.fvh_mlp_train_step(None, None, None, 0, 0.0, 1.0, None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_mlp_logits(None, None, 0, None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_set_predictor(None, None, 0.5) == _capi.ERR_ARG
    assert _capi.lib.fvh_get_pred_stats(None, None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_pred_flags(None, None, None) == _capi.ERR_ARG


def test_ensemble_entry_points_refuse_bad_arguments():
    import ctypes

    from fvhoe_b200 import _capi

    cfg = _capi.default_config()
    out = ctypes.c_void_p()
    n = (ctypes.c_int * 1)(32)
    h = (ctypes.c_double * 1)(1 / 32)
    assert _capi.lib.fvh_ensemble_create(None, 1, n, n, h, h, ctypes.byref(out)) == _capi.ERR_ARG
    assert _capi.lib.fvh_ensemble_create(ctypes.byref(cfg), 0, n, n, h, h, ctypes.byref(out)) == _capi.ERR_ARG
    # a 1D template cannot make 2D members
    cfg.p[0], cfg.p[1], cfg.p[2] = 3, 0, 0
    st = _capi.lib.fvh_ensemble_create(ctypes.byref(cfg), 1, n, (ctypes.c_int * 1)(1), h, h, ctypes.byref(out))
    assert st == _capi.ERR_CONFIG and not out.value
    assert _capi.lib.fvh_ensemble_destroy(None) == _capi.OK
    assert _capi.lib.fvh_ensemble_state(None, 0) is None
    assert _capi.lib.fvh_ensemble_step(None, 1, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_ensemble_status(None, None, None, None, None, None) == _capi.ERR_ARG


def test_default_config_matches_reference_defaults():
    from fvhoe_b200 import _capi

    c = _capi.default_config()
    assert c.abi_version == _capi.ABI_VERSION and c.nvars == 5
    assert c.gamma == 5 / 3 and c.cfl == 0.8 and c.csq_floor == 1e-10
    assert c.riemann == _capi.RIEMANN["hllc"] and c.slope_limiter == _capi.LIMITER["minmod"]
    assert c.nad_eps == 1e-2 and c.nad_global == 1 and c.nad_relative == 1 and c.nad_var_mask == 0x1F
    assert c.pad_var == 4 and c.pad_lo == 0.0 and c.pad_hi == float("inf")
    assert c.sed == 1 and c.sed_eps == 1e-10
    assert list(c.bc[0]) == [0, 0]


@pytest.mark.parametrize(
    "change, message",
    [
        (dict(p=(9, 0, 0)), "p must be in [0, 8]"),
        (dict(n=(8, 1, 1), p=(5, 0, 0)), "fewer than the 12 ghost cells"),
        (dict(nvars=4), "nvars must be in [5, 16]"),
        (dict(riemann=7), "unknown Riemann solver"),
        (dict(bc=((1, 0), (0, 0), (0, 0))), "periodic high boundary"),
        (dict(bc=((5, 1), (0, 0), (0, 0))), "low y side only"),
        (dict(bc=((1, 1), (1, 5), (0, 0)), n=(64, 32, 1), p=(3, 3, 0)), "low y side only"),
        (dict(bc=((1, 1), (6, 1), (0, 0)), n=(64, 32, 1), p=(3, 3, 0)), "unsupported boundary kind"),
        (dict(n=(1, 1, 1), p=(0, 0, 0)), "no active axis"),
        (dict(a_posteriori=1, convex=1, n=(32, 32, 32), p=(1, 1, 1)), "3D convex"),
        (dict(pad_var=7), "pad_var"),
    ],
)
def test_create_refuses_bad_configs_before_device_work(change, message):
    from fvhoe_b200 import _capi

    c = _capi.default_config()
    c.n[0], c.p[0] = 64, 3
    for key, val in change.items():
        if key in ("n", "p"):
            for a in range(3):
                getattr(c, key)[a] = val[a]
        elif key == "bc":
            for a in range(3):
                c.bc[a][0], c.bc[a][1] = val[a]
        else:
            setattr(c, key, val)
    h = ctypes.c_void_p()
    st = _capi.lib.fvh_create(ctypes.byref(c), ctypes.byref(h))
    assert st == _capi.ERR_CONFIG
    assert message in _capi.lib.fvh_last_error(None).decode()
    assert not h.value


def test_null_arguments_are_refused():
    from fvhoe_b200 import _capi

    assert _capi.lib.fvh_create(None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_rhs(None, None, None, None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_destroy(None) == _capi.OK
    assert _capi.lib.fvh_scratch_bytes(None) == 0


def test_hydrostate_slices_like_reference():
    from fvhoe_b200 import HydroState

    hs = HydroState(passive_scalars=("a", "b"))
    assert hs.nvars == 7 and hs("rho") == (0, slice(None), slice(None), slice(None))
    assert hs(x=(1, -1))[1] == slice(1, -1)
    assert list(hs("passive_scalars")[0]) == [5, 6]
    assert HydroState(ndim=1)("P") == 4
    with pytest.raises(ValueError):
        hs("nope")
    with pytest.raises(ValueError):
        HydroState(passive_scalars=("a", "a"))


def test_boundary_condition_parsing_and_refusals():
    from fvhoe_b200 import BoundaryCondition

    bc = BoundaryCondition(x=("reflective", "outflow"), y="free")
    assert bc.x == ("reflective", "outflow") and bc.y == ("free", "free") and bc.z == ("periodic", "periodic")
    assert bc.kinds((True, True, False))[0] == ("reflective", "outflow")
    # the double-Mach-reflection wall exists on the low y side only
    dmr = "special-case-double-mach-reflection-y=0"
    assert BoundaryCondition(y=(dmr, "outflow")).kinds((True, True, False))[1] == (dmr, "outflow")
    for bad in (dict(y=dmr), dict(y=("outflow", dmr)), dict(x=(dmr, "outflow"))):
        with pytest.raises(ValueError):
            BoundaryCondition(**bad).kinds((True, True, False))
    # Dirichlet sides need a callable or an array of values (the reference raises when it applies them)
    with pytest.raises(ValueError):
        BoundaryCondition(x="dirichlet").kinds((True, False, False))
    assert BoundaryCondition(x=("ic", "dirichlet"), x_value=(None, np.ones(5))).kinds((True, False, False))[0] == (
        "ic", "dirichlet")
    with pytest.raises(ValueError):
        BoundaryCondition(x=("outflow", "periodic")).kinds((True, False, False))
    with pytest.raises(ValueError):
        BoundaryCondition(x=["outflow", "outflow"])


def test_array_manager_errors_like_reference():
    from fvhoe_b200 import ArrayManager

    am = ArrayManager()
    am.add("u", np.zeros(3))
    with pytest.raises(KeyError):
        am.add("u", np.zeros(3))
    with pytest.raises(TypeError):
        am.add("v", [1, 2, 3])
    with pytest.raises(KeyError):
        am("missing")
    assert am.to_dict()["names"] == ["u"]
    got = am.get_numpy("u")
    got[0] = 5
    assert am("u")[0] == 0
    am.remove("u")
    with pytest.raises(KeyError):
        am.get_numpy("u")


def test_timer_categories():
    from fvhoe_b200 import Timer

    t = Timer(cats=["TOTAL"])
    t.start("TOTAL")
    with pytest.raises(RuntimeError):
        t.start("TOTAL")
    t.stop("TOTAL")
    with pytest.raises(ValueError):
        t.add_cat("TOTAL")
    assert "TOTAL" in t.report()


def test_initial_conditions_match_oracle_setup():
    """The package's FV-averaged initial states equal those the fixtures were made from."""
    from fvhoe_b200.fv import fv_average, fv_uniform_meshgen
    from fvhoe_b200.hydro import HydroState, compute_conservatives
    from fvhoe_b200.initial_conditions import KelvinHelmholtzNoise2D, SedovBlast, Shock1D
    from tests.fixtures import GOLDEN, load

    hs = HydroState()
    c, d = load(os.path.join(GOLDEN, "steps_sod_full.npz"))
    X, Y, Z = fv_uniform_meshgen((256, 1, 1))
    f = Shock1D().build_ic(hs)
    u0 = fv_average(lambda x, y, z: compute_conservatives(hs, f(x, y, z), 1.4), X, Y, Z, h=tuple(c["h"]),
                    p=(3, 0, 0))
    assert np.array_equal(u0, d["u0"])
    c, d = load(os.path.join(GOLDEN, "steps_kh64_p5.npz"))
    X, Y, Z = fv_uniform_meshgen((64, 64, 1))
    f = KelvinHelmholtzNoise2D(n=(64, 64), seed=7).build_ic(hs)
    u0 = fv_average(lambda x, y, z: compute_conservatives(hs, f(x, y, z), 1.4), X, Y, Z, h=tuple(c["h"]),
                    p=(5, 5, 0))
    assert np.array_equal(u0, d["u0"])
    c, d = load(os.path.join(GOLDEN, "steps_sedov3d16_p3.npz"))
    X, Y, Z = fv_uniform_meshgen((16, 16, 16))
    assert np.array_equal(SedovBlast(dims="xyz").build_ic(hs)(X, Y, Z), d["u0"])


def test_snapshot_list_settles_before_reads_and_pickles_as_a_list():
    """Snapshots are completed lazily: every read of the list waits for the
    copies in flight first (settle), taking the length does not, and the list
    pickles as the reference's plain list."""
    import pickle

    from fvhoe_b200.ode import SnapshotList

    calls = []
    log = SnapshotList(lambda: calls.append(1))
    log.append({"t": 0.0})
    log.append({"t": 0.5})
    assert len(log) == 2 and not calls
    assert log[-1]["t"] == 0.5 and len(calls) == 1
    assert [d["t"] for d in log] == [0.0, 0.5] and len(calls) == 2
    assert log == [{"t": 0.0}, {"t": 0.5}]
    back = pickle.loads(pickle.dumps(log))
    assert type(back) is list and back == [{"t": 0.0}, {"t": 0.5}]
    assert type(log.copy()) is list
    n = len(calls)
    assert log.pop()["t"] == 0.5 and len(calls) == n + 1


@pytest.mark.parametrize("name,kw,exact", [
    ("Square", dict(dims="xy"), True),
    ("Shock1D", dict(), True),
    ("DoubleShock1D", dict(), True),
    ("ShockTube", dict(dims="xy", center=(0.5, 0.5), radius=0.3), True),
    ("ShockTube", dict(mode="cube", x_cube=(0.2, 0.6), y_cube=(0.3, 0.9)), True),
    ("FourQuadrant2D", dict(seed=7), True),
    ("DoubleMachReflection2D", dict(), True),
    ("SedovBlast", dict(mode="corner", dims="xy"), True),
    ("Sinus", dict(dims="xy"), False),
    ("ShuOsher1D", dict(), False),
    ("KelvinHelmholtz2D", dict(), False),
    ("KelvinHelmholtzNoise2D", dict(n=(24, 20), seed=3), False),
])
def test_initial_conditions_evaluate_on_torch_tensors(name, kw, exact):
    """The library's initial conditions and the FV quadrature run unchanged on
    torch tensors (the device path of EulerSolver(ic_on_device=True), here on
    CPU tensors): the same state as on numpy arrays, bit for bit unless the
    condition uses sin or exp (whose last bit may differ)."""
    import torch

    import fvhoe_b200.initial_conditions as ic
    from fvhoe_b200.fv import fv_uniform_meshgen
    from fvhoe_b200.hydro import HydroState
    from fvhoe_b200.solver import _ic_functions

    n, p = (24, 20, 1), (5, 5, 0)
    h = (1 / 24, 1 / 20, 1.0)
    cons = name == "SedovBlast"
    _, _, u0_fv = _ic_functions(getattr(ic, name)(**kw), HydroState(), None, cons, cons, 1.4, h, p)
    X, Y, Z = fv_uniform_meshgen(n)
    host = u0_fv(X, Y, Z)
    dev = u0_fv(*(torch.from_numpy(a) for a in (X, Y, Z)))
    assert isinstance(dev, torch.Tensor) and dev.dtype == torch.float64
    if exact:
        assert np.array_equal(dev.numpy(), host)
    else:
        assert np.allclose(dev.numpy(), host, rtol=1e-14, atol=1e-15)


def test_dmr_split_matches_oracle_columns():
    """The split the solver hands to the library selects the same free columns
    as the oracle's restatement of the reference's X < 1/6 mask."""
    from types import SimpleNamespace

    from fvhoe_b200.boundary_conditions import dmr_split
    from oracle import fvh_oracle as O

    for n, domain, g in (((48, 12, 1), ((0, 4), (0, 1), (0, 1)), (8, 8, 0)),
                         ((40, 20, 1), ((0, 4), (0, 1), (0, 1)), (11, 11, 0)),
                         ((30, 10, 1), ((-1, 2), (0, 1), (0, 1)), (5, 5, 0)),
                         ((16, 16, 1), ((0.2, 1.0), (0, 1), (0, 1)), (6, 6, 0)),
                         ((12, 8, 1), ((-3, -1), (0, 1), (0, 1)), (4, 4, 0))):
        buffer = (30, 30, 0)
        cfg = SimpleNamespace(n=n, domain=domain, slab_buffer_size=30, active=(True, True, False))
        cols = O._dmr_free_columns(cfg, g)
        split = dmr_split(n, *domain, buffer)
        assert np.array_equal(cols, np.arange(-g[0], n[0] + g[0]) < split)


@pytest.mark.parametrize("fixture", ["rhs_dmr_p3.npz", "rhs_dmr_p7_llf.npz"])
def test_double_mach_reflection_ic_matches_reference_state(fixture):
    """DoubleMachReflection2D gives the reference's initial conserved state
    (the fixture's u0, made by fvhoe's own DoubleMachReflection2D), bit for bit."""
    from fvhoe_b200.fv import fv_uniform_meshgen
    from fvhoe_b200.hydro import HydroState
    from fvhoe_b200.initial_conditions import DoubleMachReflection2D
    from fvhoe_b200.solver import _ic_functions
    from tests.fixtures import load

    c, d = load(os.path.join(ROOT, "tests", "golden", fixture))
    _, _, u0_fv = _ic_functions(DoubleMachReflection2D(), HydroState(), None, False, False, c["gamma"],
                                tuple(c["h"]), tuple(c["p"]))
    X, Y, Z = fv_uniform_meshgen(tuple(c["n"]), *[tuple(r) for r in c["domain"]])
    assert np.array_equal(u0_fv(X, Y, Z), d["u0"])


def test_host_state_entry_points_refuse_null_arguments():
    from fvhoe_b200 import _capi

    assert _capi.lib.fvh_step_host(None, None, 2, 0.0, 0, 0.0, None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_host_sync(None) == _capi.ERR_ARG


def _noalloc_config(**change):
    from fvhoe_b200 import _capi

    c = _capi.default_config()
    c.n[0], c.n[1], c.p[0], c.p[1] = 64, 48, 3, 3
    c.h[0], c.h[1] = 1 / 64, 1 / 48
    c.device = 0
    for key, val in change.items():
        if key == "bc":
            for a in range(3):
                c.bc[a][0], c.bc[a][1] = val[a]
        elif key in ("n", "p"):
            for a in range(3):
                getattr(c, key)[a] = val[a]
        else:
            setattr(c, key, val)
    return c


@pytest.mark.parametrize(
    "change, code, message",
    [
        (dict(bc=((4, 4), (0, 0), (0, 0))), "ERR_CONFIG", "need a handle"),
        (dict(bc=((1, 1), (5, 1), (0, 0))), "ERR_CONFIG", "need a handle"),
        (dict(device=64), "ERR_CONFIG", "device ordinal out of range"),
        (dict(device=-1), "ERR_CONFIG", "device ordinal out of range"),
        (dict(n=(1024, 1024, 1), p=(5, 5, 0)), "ERR_CONFIG", "grid too large"),
        (dict(p=(9, 3, 0)), "ERR_CONFIG", "p must be in [0, 8]"),
    ],
)
def test_noalloc_refusals_are_decided_on_the_host(change, code, message):
    """Every refusal of the allocation-free conversion comes before any CUDA call
    and before the state pointers are used, so null pointers are safe here."""
    from fvhoe_b200 import _capi

    cfg = _noalloc_config(**change)
    st = _capi.lib.fvh_primitives_noalloc(ctypes.byref(cfg), None, None, 1, None)
    assert st == getattr(_capi, code)
    assert message in _capi.lib.fvh_primitives_noalloc_error().decode()


def test_noalloc_null_arguments():
    from fvhoe_b200 import _capi

    assert _capi.lib.fvh_primitives_noalloc(None, None, None, 1, None) == _capi.ERR_ARG
    assert "null configuration" in _capi.lib.fvh_primitives_noalloc_error().decode()
    cfg = _noalloc_config()
    assert _capi.lib.fvh_primitives_noalloc(ctypes.byref(cfg), None, None, 1, None) == _capi.ERR_ARG
    assert "null state" in _capi.lib.fvh_primitives_noalloc_error().decode()


def test_stage_and_wait_limit_refuse_null_handles():
    from fvhoe_b200 import _capi

    assert _capi.lib.fvh_stage(None, None, 2, 0, 0.0, 0, 0.0, None, None) == _capi.ERR_ARG
    assert _capi.lib.fvh_ensemble_set_wait_limit(None, 1) == _capi.ERR_ARG
