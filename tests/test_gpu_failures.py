"""Failures reach the caller (GPU), without faulting or hanging the device.

* A state with a NaN in one cell: the step's read-back returns
  FVH_ERR_NONFINITE, fvh_get_stats counts the values, and EulerSolver's
  integrate raises instead of looping on a frozen time (the reference's
  integrate loop, fvhoe/ode.py:157, has no such guard).
* A state with a negative density in one cell: the status follows the
  oracle's own outcome on the same input (FVH_ERR_NONFINITE exactly when the
  reference algorithm produces NaN/Inf values), and a finite FP64 result
  equals the oracle's.
* The batched ensemble's grid-barrier waits are bounded: with the bound cut
  to one poll, blocks give up, every block returns (the stream completes) and
  fvh_ensemble_status reports FVH_ERR_TIMEOUT; after fvh_ensemble_reset with
  the default bound the ensemble steps normally again.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 64


def _kh_state(n=N, p=3):
    from fvhoe_b200 import KelvinHelmholtzNoise2D
    from fvhoe_b200.solver import initial_state

    return initial_state(KelvinHelmholtzNoise2D(n=(n, n), seed=5), n, n, 1, p, p, 0, gamma=1.4)


def _solver(u0, precision, kernel_path, n=N, p=3):
    from fvhoe_b200 import ArrayIC, EulerSolver

    return EulerSolver(w0=ArrayIC(array=u0), conservative_ic=True, fv_ic=True, nx=n, ny=n, px=p, py=p, gamma=1.4,
                       riemann_solver="hllc", CFL=0.8, a_posteriori_slope_limiting=True, NAD=1e-5,
                       progress_bar=False, precision=precision, kernel_path=kernel_path)


def _step_status(s):
    import torch

    from fvhoe_b200 import _capi

    u = s.am("u")
    dt = ctypes.c_double()
    st = _capi.lib.fvh_step(s._handle, ctypes.c_void_p(u.data_ptr()), _capi.INTEGRATOR["ssprk3"], 0.0, 0, 0.0,
                            ctypes.byref(dt), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, dt.value, _capi.lib.fvh_last_error(s._handle).decode()


@pytest.mark.parametrize("kernel_path", ["fused2d", "generic"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_nan_cell_returns_nonfinite_and_stops_integrate(precision, kernel_path):
    from fvhoe_b200 import _capi

    u0 = _kh_state()
    u0[4, 20, 33] = np.nan
    s = _solver(u0, precision, kernel_path)
    st, _, msg = _step_status(s)
    assert st == _capi.ERR_NONFINITE, (st, msg)
    assert "non-finite" in msg or "not finite" in msg
    assert s.stats()["nonfinite"] > 0
    s2 = _solver(u0, precision, kernel_path)
    with pytest.raises(FloatingPointError):
        s2.ssprk3(0.01)
    assert s2.step_count == 0 and s2.t == 0.0


def test_negative_density_follows_the_oracle():
    """FP64: the library reports a non-finite update exactly when the oracle's
    step on the same input has NaN/Inf values, and a finite result is the
    oracle's bit for bit."""
    from fvhoe_b200 import _capi
    from oracle import fvh_oracle as O

    u0 = _kh_state()
    u0[0, 40, 12] = -abs(u0[0, 40, 12])
    cfg = O.OracleConfig(n=(N, N, 1), p=(3, 3, 0), h=(1 / N, 1 / N, 1.0), gamma=1.4, riemann_solver="hllc", CFL=0.8,
                         a_posteriori_slope_limiting=True, NAD=1e-5)
    with np.errstate(all="ignore"):
        dt_ref, u_ref, _ = O.step(u0, 0.0, cfg, "ssprk3")
    ref_finite = bool(np.all(np.isfinite(u_ref))) and np.isfinite(dt_ref) and dt_ref > 0
    for kernel_path in ("fused2d", "generic"):
        s = _solver(u0, "fp64", kernel_path)
        st, dt, msg = _step_status(s)
        if ref_finite:
            assert st == _capi.OK, msg
            assert dt == dt_ref
            assert np.array_equal(s.am.get_numpy("u"), u_ref)
        else:
            assert st == _capi.ERR_NONFINITE, (st, msg)


def test_finite_states_return_ok_with_the_read_back():
    from fvhoe_b200 import _capi

    s = _solver(_kh_state(), "fp64", "fused2d")
    st, dt, msg = _step_status(s)
    assert st == _capi.OK and dt > 0, msg
    assert s.stats()["nonfinite"] == 0


def test_ensemble_barrier_wait_that_runs_out_is_reported_and_recoverable():
    import torch

    from fvhoe_b200 import BoundaryCondition, Ensemble, FourQuadrant2D, _capi

    members = [dict(w0=FourQuadrant2D(seed=q), nx=n, ny=n) for q, n in enumerate((64, 96))]
    ens = Ensemble(members, px=3, precision="fp64", gamma=1.4, riemann_solver="hllc", CFL=0.8,
                   bc=BoundaryCondition(x="outflow", y="outflow"), a_posteriori_slope_limiting=True, NAD=1e-5)
    h = ens._e
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ens.reset(0.05)
    # one poll per wait: blocks with no tile in a phase reach the barrier long
    # before the blocks with work, so their waits run out
    assert _capi.lib.fvh_ensemble_set_wait_limit(h, 1) == _capi.OK
    assert _capi.lib.fvh_ensemble_step(h, 2, stream) == _capi.OK
    torch.cuda.synchronize()  # every block returned: the launches completed
    st = _capi.lib.fvh_ensemble_status(h, None, None, None, None, stream)
    assert st == _capi.ERR_TIMEOUT
    assert "ran out" in _capi.lib.fvh_ensemble_last_error(h).decode()
    # the default bound and a reset: the ensemble advances again, with finite states
    assert _capi.lib.fvh_ensemble_set_wait_limit(h, 0) == _capi.OK
    ens.reset(0.05)
    ens.step(3)
    status = ens.status()
    assert status["nonfinite"] == 0
    assert all(k == 3 for k in status["steps"])
