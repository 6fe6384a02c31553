"""fvh_stage: one Runge-Kutta stage per call (GPU).

The reference's steppers evaluate the right-hand side once per stage and
combine (fvhoe/ode.py:245-298; SSP-RK3 at :274-280). fvh_stage exposes that
granularity on the C ABI: the stages of one step, called in order, must equal
one fvh_step call bit for bit, and a stage called out of order is refused
before any device work.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(precision, kernel_path, n=72, p=5):
    from fvhoe_b200 import ArrayIC, EulerSolver, KelvinHelmholtzNoise2D
    from fvhoe_b200.solver import initial_state

    u0 = initial_state(KelvinHelmholtzNoise2D(n=(n, n), seed=9), n, n, 1, p, p, 0, gamma=1.4)
    kw = dict(w0=ArrayIC(array=u0), conservative_ic=True, fv_ic=True, nx=n, ny=n, px=p, py=p, gamma=1.4,
              riemann_solver="hllc", CFL=0.8, a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False,
              precision=precision, kernel_path=kernel_path)
    return EulerSolver(**kw), EulerSolver(**kw)


@pytest.mark.parametrize("kernel_path", ["fused2d", "generic"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("integrator", ["ssprk3", "rk4", "ssprk2"])
def test_stages_equal_one_step(precision, kernel_path, integrator):
    import torch

    from fvhoe_b200 import _capi

    lib = _capi.lib
    a, b = _pair(precision, kernel_path)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    stages = {"ssprk2": 2, "ssprk3": 3, "rk4": 4}[integrator]
    integ = _capi.INTEGRATOR[integrator]
    t, target = 0.0, 1.5e-3  # a target inside the first step: the clamp applies
    for _ in range(2):
        ua = ctypes.c_void_p(a.am("u").data_ptr())
        ub = ctypes.c_void_p(b.am("u").data_ptr())
        dta, dtb = ctypes.c_double(), ctypes.c_double()
        _capi.check(lib.fvh_step(a._handle, ua, integ, t, 1, target, ctypes.byref(dta), stream), a._handle)
        for k in range(stages):
            _capi.check(lib.fvh_stage(b._handle, ub, integ, k, t, 1, target, ctypes.byref(dtb), stream), b._handle)
        assert dta.value == dtb.value
        assert torch.equal(a.am("u"), b.am("u"))
        assert np.array_equal(a.trouble_flags(), b.trouble_flags())
        t += dta.value


def test_stage_out_of_order_is_refused():
    import torch

    from fvhoe_b200 import _capi

    lib = _capi.lib
    a, _ = _pair("fp64", "fused2d", n=48, p=3)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ua = ctypes.c_void_p(a.am("u").data_ptr())
    ssprk3 = _capi.INTEGRATOR["ssprk3"]
    before = a.am("u").clone()
    assert lib.fvh_stage(a._handle, ua, ssprk3, 1, 0.0, 0, 0.0, None, stream) == _capi.ERR_ARG
    assert "must follow stage 0" in lib.fvh_last_error(a._handle).decode()
    assert lib.fvh_stage(a._handle, ua, ssprk3, 3, 0.0, 0, 0.0, None, stream) == _capi.ERR_ARG
    assert lib.fvh_stage(a._handle, ua, ssprk3, 0, 0.0, 0, 0.0, None, stream) == _capi.OK
    assert lib.fvh_stage(a._handle, ua, _capi.INTEGRATOR["rk4"], 1, 0.0, 0, 0.0, None, stream) == _capi.ERR_ARG
    assert lib.fvh_stage(a._handle, ua, ssprk3, 2, 0.0, 0, 0.0, None, stream) == _capi.ERR_ARG
    torch.cuda.synchronize()
    assert torch.equal(a.am("u"), before)  # stage 0 writes only the stage buffers


@pytest.mark.parametrize("kernel_path", ["fused2d", "generic"])
def test_euler_steps_equal_the_oracle(kernel_path, n=192, p=5, steps=3):
    """A one-stage step updates u in place. The fused final pass of a troubled
    tile reads the stage input two cells around the tile, cells that
    neighbouring blocks update in the same launch, so the step must read a
    copy of u: checked bit for bit against the oracle's forward Euler
    (fvhoe/ode.py:245-252) on a grid of many troubled tiles."""
    from fvhoe_b200 import ArrayIC, EulerSolver, KelvinHelmholtzNoise2D
    from fvhoe_b200.solver import initial_state
    from oracle import fvh_oracle as O

    u = initial_state(KelvinHelmholtzNoise2D(n=(n, n), seed=4), n, n, 1, p, p, 0, gamma=1.4)
    s = EulerSolver(w0=ArrayIC(array=u), conservative_ic=True, fv_ic=True, nx=n, ny=n, px=p, py=p, gamma=1.4,
                    riemann_solver="hllc", CFL=0.8, a_posteriori_slope_limiting=True, NAD=1e-5,
                    progress_bar=False, kernel_path=kernel_path)
    cfg = O.OracleConfig(n=(n, n, 1), p=(p, p, 0), h=s.h, gamma=1.4, riemann_solver="hllc",
                         a_posteriori_slope_limiting=True, NAD=1e-5)
    t = 0.0
    for _ in range(steps):
        dt, u, _ = O.step(u, t, cfg, "euler")
        t += dt
    s.euler(n=steps)
    assert s.t == t
    assert int(s.trouble_flags().sum()) > 0
    assert np.array_equal(s.am.get_numpy("u"), u)
