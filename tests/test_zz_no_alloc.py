"""The allocation-free primitive conversion against the handle-based one (GPU).

fvh_primitives_noalloc serves callers that cannot allocate device memory when
they convert conserved averages to primitives (a host application that owns
the device memory pool, or a run that has committed the whole device to its
state). It must return exactly what fvh_primitives returns, call after call,
although every call reuses the same static scratch. This file is collected
last, so a failure here leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _config(n, p, bc_kind, nvars=5):
    from fvhoe_b200 import _capi

    c = _capi.default_config()
    c.nvars = nvars
    for a in range(3):
        c.n[a], c.p[a] = n[a], p[a]
        c.h[a] = 1.0 / n[a]
        c.bc[a][0] = c.bc[a][1] = _capi.BC[bc_kind]
    c.gamma = 1.4
    c.device = 0
    return c


def _state(n, seed, nvars=5):
    """A positive-density, positive-pressure conserved state with rough structure."""
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.5 * rng.random(n)
    v = rng.uniform(-1, 1, (3,) + n)
    P = 0.5 + rng.random(n)
    u = np.empty((nvars,) + n)
    u[0] = rho
    u[1:4] = rho * v
    u[4] = P / 0.4 + 0.5 * rho * np.sum(v * v, axis=0)
    for k in range(5, nvars):
        u[k] = rho * rng.random(n)
    return u


def _with_handle(cfg, u, fv_average):
    import torch

    from fvhoe_b200 import _capi

    h = ctypes.c_void_p()
    _capi.check(_capi.lib.fvh_create(ctypes.byref(cfg), ctypes.byref(h)))
    try:
        ud = torch.from_numpy(u).cuda()
        wd = torch.empty_like(ud)
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _capi.check(_capi.lib.fvh_primitives(h, ctypes.c_void_p(ud.data_ptr()), ctypes.c_void_p(wd.data_ptr()),
                                             int(fv_average), s), h)
        return wd.cpu().numpy()
    finally:
        _capi.lib.fvh_destroy(h)


def _no_alloc(cfg, u, fv_average):
    import torch

    from fvhoe_b200 import _capi

    ud = torch.from_numpy(u).cuda()
    wd = torch.full_like(ud, float("nan"))
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = _capi.lib.fvh_primitives_noalloc(ctypes.byref(cfg), ctypes.c_void_p(ud.data_ptr()),
                                          ctypes.c_void_p(wd.data_ptr()), int(fv_average), s)
    assert st == _capi.OK, _capi.lib.fvh_primitives_noalloc_error().decode()
    return wd.cpu().numpy()


CASES = [
    ((96, 80, 1), (5, 5, 0), "periodic", 5, True),
    ((20, 18, 16), (3, 3, 3), "outflow", 5, True),
    ((256, 1, 1), (8, 0, 0), "reflective", 7, False),
]


@pytest.mark.parametrize("n, p, bc, nvars, fv", CASES)
def test_no_alloc_equals_handle_path_twice(n, p, bc, nvars, fv):
    cfg = _config(n, p, bc, nvars)
    for seed in (1, 2):  # two calls in a row on different inputs
        u = _state(n, seed, nvars)
        ref = _with_handle(cfg, u, fv)
        got = _no_alloc(cfg, u, fv)
        assert np.array_equal(got, ref)  # FP64 path: bit-exact, as everywhere else


def test_no_alloc_refuses_oversized_grids():
    """Real device arrays of the oversized grid: if the size check ever let the
    call through, it would fail as a wrong status, not as a stray access."""
    import torch

    from fvhoe_b200 import _capi

    limit = _capi.lib.fvh_primitives_noalloc_max_doubles()
    cfg = _config((1024, 1024, 1), (5, 5, 0), "periodic")
    assert 5 * (1024 + 12) ** 2 > limit
    ud = torch.ones((5, 1024, 1024), dtype=torch.float64, device="cuda")
    wd = torch.empty_like(ud)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = _capi.lib.fvh_primitives_noalloc(ctypes.byref(cfg), ctypes.c_void_p(ud.data_ptr()),
                                          ctypes.c_void_p(wd.data_ptr()), 1, s)
    assert st == _capi.ERR_CONFIG
    assert "too large" in _capi.lib.fvh_primitives_noalloc_error().decode()
