"""CUDA path against the reference-generated golden fixtures (GPU).

Each case rebuilds the fixture's problem in fvhoe_b200.EulerSolver (which
calls libfvh.so through its C ABI) from the stored initial state. In FP64
mode the update must equal the reference bit for bit: the same dt, the same
dudt / states, identical trouble flags, identical trouble logs.
"""

import os

import numpy as np
import pytest

from tests.fixtures import golden_files, load, solver_kwargs

pytestmark = pytest.mark.gpu

RHS = golden_files("rhs")
STEPS = golden_files("steps")


def _solver(c, u0, **extra):
    from fvhoe_b200 import EulerSolver

    return EulerSolver(**solver_kwargs(c, u0, **extra))


KERNEL_PATHS = ["auto", "generic"]


@pytest.mark.parametrize("kernel_path", KERNEL_PATHS)
@pytest.mark.parametrize("path", RHS, ids=[os.path.basename(p) for p in RHS])
def test_rhs_bit_exact(path, kernel_path):
    c, d = load(path)
    s = _solver(c, d["u0"], kernel_path=kernel_path)
    dt, dudt = s.f(0.0, s.am("u"))
    assert dt == float(d["dt"])
    got = dudt.cpu().numpy()
    assert np.array_equal(got, d["dudt"]), f"max |diff| {np.max(np.abs(got - d['dudt']))}"
    if "trouble" in d:
        assert np.array_equal(s.trouble_flags().astype(np.int8), d["trouble"])
        trouble, nad, pad = s._trouble_logs()
        # one evaluation after construction: the sums hold this stage's values
        assert np.array_equal(trouble[0], d["trouble"].astype(np.float64))
        assert np.array_equal(nad[0], d["nad_mag"])
        assert np.array_equal(pad[0], d["pad_mag"])


@pytest.mark.parametrize("kernel_path", KERNEL_PATHS)
@pytest.mark.parametrize("path", STEPS, ids=[os.path.basename(p) for p in STEPS])
def test_steps_bit_exact(path, kernel_path):
    c, d = load(path)
    s = _solver(c, d["u0"], kernel_path=kernel_path)
    stepper = getattr(s, c["integrator"])
    if "T" in d:
        stepper(float(d["T"]))
    else:
        stepper(n=int(d["steps"]))
    assert s.step_count == int(d["steps"])
    assert s.t == d["timestamps"][-1]
    assert np.array_equal(np.array(s.timestamps), d["timestamps"])
    u = s.am.get_numpy("u")
    assert np.array_equal(u, d["u_final"]), f"max |diff| {np.max(np.abs(u - d['u_final']))}"
    if "w_final" in d:
        assert np.array_equal(s.snapshots[-1]["w"], d["w_final"])


def test_fp32_mode_close_to_fp64():
    """FP32 reconstruction/Riemann/detection with FP64 accumulation stays close to FP64."""
    c, d = load(os.path.join(os.path.dirname(RHS[0]), "steps_kh64_p5.npz"))
    s64 = _solver(c, d["u0"])
    s32 = _solver(c, d["u0"], precision="fp32")
    s64.ssprk3(n=2)
    s32.ssprk3(n=2)
    r64 = s64.am.get_numpy("u")[0]
    r32 = s32.am.get_numpy("u")[0]
    l1 = np.mean(np.abs(r32 - r64))
    assert l1 < 1e-5, l1


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("riemann", ["hllc", "llf"])
# ragged tiles: rows that are not whole 16-byte vectors, and a last tile holding
# 1-3 cells along Y (the grid's last face then falls inside the padding columns
# of the tile before it)
@pytest.mark.parametrize("n", [(40, 36), (37, 66), (98, 35)])
def test_fused2d_equals_generic_fp64(p, riemann, n):
    """The fused 2D kernels and the generic passes give identical FP64 steps for every degree."""
    from fvhoe_b200 import BoundaryCondition, EulerSolver, FourQuadrant2D

    kw = dict(w0=FourQuadrant2D(seed=p), nx=n[0], ny=n[1], px=p, py=p, gamma=1.4, riemann_solver=riemann,
              bc=BoundaryCondition(x="outflow", y=("reflective", "outflow")), a_posteriori_slope_limiting=True,
              NAD=1e-4, progress_bar=False)
    fused = EulerSolver(kernel_path="fused2d", **kw)
    generic = EulerSolver(kernel_path="generic", **kw)
    fused.ssprk3(n=3)
    generic.ssprk3(n=3)
    assert fused.t == generic.t
    assert np.array_equal(fused.am.get_numpy("u"), generic.am.get_numpy("u"))
    assert np.array_equal(fused.trouble_flags(), generic.trouble_flags())
    assert np.array_equal(fused.snapshots[-1]["trouble"], generic.snapshots[-1]["trouble"])


@pytest.mark.parametrize("p", [3, 5, 7])
def test_fused2d_fp32_close_to_generic_fp32(p):
    from fvhoe_b200 import EulerSolver, KelvinHelmholtzNoise2D

    kw = dict(w0=KelvinHelmholtzNoise2D(n=(64, 64), seed=3), nx=64, ny=64, px=p, py=p, gamma=1.4,
              a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False, precision="fp32")
    a = EulerSolver(kernel_path="fused2d", **kw)
    b = EulerSolver(kernel_path="generic", **kw)
    dta, ka = a.f(0.0, a.am("u"))
    dtb, kb = b.f(0.0, b.am("u"))
    assert abs(dta - dtb) <= 1e-6 * dtb
    diff = (ka - kb).abs().max().item()
    scale = kb.abs().max().item()
    assert diff <= 1e-4 * scale, (diff, scale)


def test_log_division_in_the_last_stage_equals_the_separate_pass():
    """fvh_set_log_divisor makes the step's last stage divide the trouble-log sums
    (the reset branch of log_troubles); the result equals the separate division."""
    import ctypes

    import torch

    from fvhoe_b200 import EulerSolver, KelvinHelmholtzNoise2D, _capi

    kw = dict(w0=KelvinHelmholtzNoise2D(n=(48, 48), seed=5), nx=48, ny=48, px=3, py=3, gamma=1.4,
              a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False)
    logs = []
    for fused in (True, False):
        s = EulerSolver(**kw)
        h, lib = s._handle, _capi.lib
        u = ctypes.c_void_p(s.am("u").data_ptr())
        for k in range(3):
            _capi.check(lib.fvh_set_log_mode(h, 1 if k else 2), h)
            if fused:
                _capi.check(lib.fvh_set_log_divisor(h, 4.0 if k == 0 else 3.0), h)
            _capi.check(lib.fvh_step(h, u, _capi.INTEGRATOR["ssprk3"], 0.0, 0, 0.0, None, None), h)
            if not fused:
                _capi.check(lib.fvh_trouble_log(h, 4.0 if k == 0 else 3.0, None, None, None, None), h)
        torch.cuda.synchronize()
        logs.append([x.copy() for x in s._trouble_logs()])
    for a, b in zip(*logs):
        assert np.array_equal(a, b)
    assert logs[0][0].max() > 0


def test_snapshots_copied_asynchronously_equal_settled_ones(tmp_path):
    """Snapshot copies run on a separate stream and are completed when the list
    is read: a run that reads nothing until it ends records the same snapshots
    (primitives and trouble logs) as one whose helper reads each snapshot as it
    is taken, and the pickled snapshots read back unchanged."""
    from fvhoe_b200 import EulerSolver, KelvinHelmholtzNoise2D

    def make():
        return EulerSolver(w0=KelvinHelmholtzNoise2D(n=(96, 64), seed=5), nx=96, ny=64, px=5, py=5, gamma=1.4,
                           a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False)

    lazy = make()
    lazy.ssprk3(0.02, downbeats=[0.005, 0.01, 0.015], log_every_step=False)
    seen = []
    eager = make()
    eager.snapshot_helper_function = lambda s: seen.append(
        (s.snapshots[-1]["w"].copy(), s.am.get_numpy("w"), s.snapshots[-1]["trouble"].copy()))
    eager.ssprk3(0.02, downbeats=[0.005, 0.01, 0.015], log_every_step=False)
    assert len(lazy.snapshots) == len(seen) == 5
    for got, (w_eager, w_device, trouble) in zip(lazy.snapshots, seen):
        assert np.array_equal(w_eager, w_device)
        assert np.array_equal(got["w"], w_eager)
        assert np.array_equal(got["trouble"], trouble)
        assert list(got) == ["x", "y", "z", "t", "w", "trouble", "NAD violation magnitude",
                             "PAD violation magnitude"]
    assert lazy.snapshots[-1]["trouble"].max() > 0
    lazy.snapshot_dir = str(tmp_path / "snaps")
    lazy.write_snapshots(overwrite=False)
    back = make()
    back.snapshot_dir = lazy.snapshot_dir
    assert back.read_snapshots()
    assert all(np.array_equal(a["w"], b["w"]) for a, b in zip(lazy.snapshots, back.snapshots))


@pytest.mark.parametrize("ic,exact", [("FourQuadrant2D", True), ("KelvinHelmholtzNoise2D", False)])
def test_initial_state_averaged_on_the_device(ic, exact):
    """EulerSolver(ic_on_device=True) averages the initial condition on the
    device: the same state as the host path (bit for bit without sin/exp), and
    a refusal for an initial condition written for numpy arrays only."""
    import fvhoe_b200.initial_conditions as ics
    from fvhoe_b200 import EulerSolver

    n = (200, 136)
    w0 = ics.FourQuadrant2D(seed=4) if ic == "FourQuadrant2D" else ics.KelvinHelmholtzNoise2D(n=n, seed=2)
    kw = dict(w0=w0, nx=n[0], ny=n[1], px=7, py=7, gamma=1.4, a_posteriori_slope_limiting=True, progress_bar=False)
    host = EulerSolver(**kw)
    dev = EulerSolver(ic_on_device=True, **kw)
    a, b = host.am.get_numpy("u"), dev.am.get_numpy("u")
    if exact:
        assert np.array_equal(a, b)
    else:
        assert np.allclose(a, b, rtol=1e-14, atol=1e-15)
    host.ssprk3(n=2)
    dev.ssprk3(n=2)
    assert np.allclose(host.am.get_numpy("u"), dev.am.get_numpy("u"), rtol=1e-12, atol=1e-13)

    class NumpyOnly(ics.InitialCondition):
        def base_ic(self):
            return lambda x, y=None, z=None: np.stack([np.ones_like(x)] * 5)

    with pytest.raises(TypeError):
        EulerSolver(w0=NumpyOnly(), nx=16, ny=16, ic_on_device=True, progress_bar=False)


@pytest.mark.parametrize("p", [3, 7])
def test_double_mach_reflection_fused_equals_generic(p):
    """The double Mach reflection with its three walls (the inflow at x = 0, the
    free/reflective wall at y = 0, the moving shock at y = 1) on a grid larger
    than the fixtures': the fused 2D kernels equal the generic passes bit for
    bit in FP64, and the FP32 form stays close to FP64 (relative L1 of the
    density below 1e-3 after three steps through the shocks)."""
    from fvhoe_b200 import BoundaryCondition, DoubleMachReflection2D, EulerSolver
    from tests.fixtures import _bc_values_module

    vals = _bc_values_module()
    bc = BoundaryCondition(x=("dirichlet", "outflow"), y=("special-case-double-mach-reflection-y=0", "dirichlet"),
                           x_value=(vals.resolve("dmr_inflow"), None), y_value=(None, vals.resolve("dmr_top")))
    kw = dict(w0=DoubleMachReflection2D(), nx=200, ny=52, px=p, py=p, x=(0, 4), y=(0, 1), gamma=1.4, bc=bc,
              riemann_solver="hllc", a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False)
    fused = EulerSolver(kernel_path="fused2d", **kw)
    generic = EulerSolver(kernel_path="generic", **kw)
    fp32 = EulerSolver(kernel_path="fused2d", precision="fp32", **kw)
    for s in (fused, generic, fp32):
        s.ssprk3(n=3)
    assert fused.t == generic.t
    a = fused.am.get_numpy("u")
    assert np.array_equal(a, generic.am.get_numpy("u"))
    r = fp32.am.get_numpy("u")[0]
    rel = np.mean(np.abs(r - a[0])) / np.mean(np.abs(a[0]))
    print(f"dmr p={p} fp32 relative L1 {rel:.3e}")
    assert rel < 1e-3, rel


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_step_captured_in_a_cuda_graph_equals_eager_steps(precision):
    """fvh_step with dt_out = NULL makes no host synchronisation, so a whole
    SSP-RK3 step (its fifteen fused launches and the scalar resets) can be
    captured in a CUDA graph; replaying it gives the eagerly stepped states bit
    for bit (dt is computed and used on the device every replay)."""
    import ctypes

    import torch

    from fvhoe_b200 import EulerSolver, KelvinHelmholtzNoise2D, _capi

    kw = dict(w0=KelvinHelmholtzNoise2D(n=(128, 96), seed=4), nx=128, ny=96, px=5, py=5, gamma=1.4,
              riemann_solver="hllc", a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False,
              precision=precision)
    eager, graphed = EulerSolver(**kw), EulerSolver(**kw)
    lib, ssprk3 = _capi.lib, _capi.INTEGRATOR["ssprk3"]

    def step(s, stream):
        u = ctypes.c_void_p(s.am("u").data_ptr())
        _capi.check(lib.fvh_step(s._handle, u, ssprk3, 0.0, 0, 0.0, None, ctypes.c_void_p(stream)), s._handle)

    cur = torch.cuda.current_stream().cuda_stream
    for _ in range(4):
        step(eager, cur)
    step(graphed, cur)  # warm-up outside the capture (module loading, shared-memory attributes)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=side):
        step(graphed, torch.cuda.current_stream().cuda_stream)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(graphed.am.get_numpy("u"), eager.am.get_numpy("u"))
    del g


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_host_state_steps_equal_device_steps(precision):
    """fvh_step_host (state in page-locked host memory, chunked copies on two
    copy streams, one call's copy-in following the previous call's copy-out)
    gives, after every step, the state fvh_step gives on the device."""
    import ctypes

    import torch

    from fvhoe_b200 import EulerSolver, KelvinHelmholtzNoise2D, _capi

    kw = dict(w0=KelvinHelmholtzNoise2D(n=(136, 100), seed=6), nx=136, ny=100, px=5, py=5, gamma=1.4,
              riemann_solver="hllc", a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False,
              precision=precision)
    dev, host_side = EulerSolver(**kw), EulerSolver(**kw)
    lib, ssprk3 = _capi.lib, _capi.INTEGRATOR["ssprk3"]
    host = torch.empty(host_side.am("u").shape, dtype=torch.float64, pin_memory=True)
    host.copy_(host_side.am("u"))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dt_dev, dt_host = ctypes.c_double(), ctypes.c_double()
    u_dev = ctypes.c_void_p(dev.am("u").data_ptr())
    for k in range(5):
        _capi.check(lib.fvh_step(dev._handle, u_dev, ssprk3, 0.0, 0, 0.0, ctypes.byref(dt_dev), stream), dev._handle)
        _capi.check(lib.fvh_step_host(host_side._handle, ctypes.c_void_p(host.data_ptr()), ssprk3, 0.0, 0, 0.0,
                                      ctypes.byref(dt_host), stream), host_side._handle)
        assert dt_host.value == dt_dev.value
        if k in (0, 4):
            _capi.check(lib.fvh_host_sync(host_side._handle), host_side._handle)
            assert np.array_equal(host.numpy(), dev.am.get_numpy("u"))
    assert lib.fvh_host_sync(None) == _capi.ERR_ARG



@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [0, 1, 2, 3])
@pytest.mark.parametrize("n", [(20, 18, 17), (33, 16, 41)])
def test_streaming_3d_primitives_equal_generic(p, n, precision):
    """3D problems ("auto") with p <= 3 run their primitive passes as one
    streaming kernel, detect troubled cells with the sliding-window kernel and
    solve the fallback from compacted face lists; the steps equal the generic
    kernels' bit for bit on ragged grids (chunks along x cut short, tiles past
    the box) with mixed periodic, outflow and reflective sides."""
    from fvhoe_b200 import BoundaryCondition, EulerSolver, SedovBlast

    kw = dict(w0=SedovBlast(dims="xyz"), conservative_ic=True, fv_ic=True, nx=n[0], ny=n[1], nz=n[2], px=p, py=p,
              pz=p, gamma=1.4, riemann_solver="llf", CFL=0.5, precision=precision,
              bc=BoundaryCondition(x=("reflective", "outflow"), y="periodic", z=("outflow", "reflective")),
              a_posteriori_slope_limiting=True, NAD=1e-4, progress_bar=False)
    stream = EulerSolver(kernel_path="auto", **kw)
    generic = EulerSolver(kernel_path="generic", **kw)
    stream.ssprk3(n=2)
    generic.ssprk3(n=2)
    assert stream.t == generic.t
    assert np.array_equal(stream.am.get_numpy("u"), generic.am.get_numpy("u"))
    assert np.array_equal(stream.trouble_flags(), generic.trouble_flags())


_MODES_3D = {
    "local_relative": dict(NAD_mode="local", NAD_range="relative"),
    "global_absolute_nosed": dict(NAD_mode="global", NAD_range="absolute", SED=False),
    "local_absolute_vars": dict(NAD_mode="local", NAD_range="absolute", NAD_vars=("rho", "P")),
    "moncen": dict(slope_limiter="moncen"),
    "unlimited": dict(slope_limiter=None),
    "passives": dict(w0_passives={"tracer": lambda x, y, z: np.sin(6.0 * x) * np.cos(4.0 * z)}),
}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("mode", list(_MODES_3D))
def test_3d_detection_and_fallback_modes_equal_generic(mode, precision):
    """The sliding-window 3D detection, the compacting fallback and (five
    variables) the streaming primitive pass against the generic kernels under
    the detector's modes: local and absolute NAD ranges, SED off, a variable
    subset, the moncen and unlimited fallbacks, and passive scalars (which take
    the variable-count-at-run-time kernels); bit for bit, flags and logs too."""
    from fvhoe_b200 import BoundaryCondition, EulerSolver, SedovBlast

    kw = dict(w0=SedovBlast(dims="xyz"), conservative_ic=True, fv_ic=True, nx=19, ny=22, nz=17, px=2, py=2, pz=2,
              gamma=1.4, riemann_solver="hllc", CFL=0.5, precision=precision,
              bc=BoundaryCondition(x=("reflective", "outflow"), y=("outflow", "reflective"),
                                   z=("outflow", "reflective")),
              a_posteriori_slope_limiting=True, NAD=1e-4, progress_bar=False)
    kw.update(_MODES_3D[mode])
    fast = EulerSolver(kernel_path="auto", **kw)
    generic = EulerSolver(kernel_path="generic", **kw)
    fast.ssprk3(n=3)
    generic.ssprk3(n=3)
    assert fast.t == generic.t
    assert np.array_equal(fast.am.get_numpy("u"), generic.am.get_numpy("u"))
    assert np.array_equal(fast.trouble_flags(), generic.trouble_flags())
    for a, b in zip(fast._trouble_logs(), generic._trouble_logs()):
        assert np.array_equal(a, b)
