"""EulerSolver with the "cuda" array backend.

The constructor takes the arguments of fvhoe/solver.py:42-84 (plus
`backend`, `precision`, `log_troubles` and `kernel_path`), builds the mesh and the initial
condition on the host exactly as the reference does (fvhoe/solver.py:220-312),
moves the state to the GPU once, and from then on every right-hand-side
evaluation and every time step runs in the CUDA library libfvh.so through its
C ABI (include/fvh.h). Snapshots, trouble logs, timing categories and the
snapshot files keep the reference's formats (fvhoe/solver.py:794-953).

There is no CPU path: constructing the solver without a CUDA device, or
without the built library, raises.
"""

import ctypes
import inspect
import json
import os
import pickle
import shutil
import sys
from typing import Callable, Dict, Iterable, Tuple

import numpy as np

from .array_management import ArrayManager
from .boundary_conditions import DMR_Y0, BoundaryCondition
from .fv import fv_average, fv_uniform_meshgen
from .hydro import HydroState, compute_conservatives
from .initial_conditions import InitialCondition, Square
from .ode import ODE, SnapshotList

_VAR_INDEX = {"rho": 0, "vx": 1, "mx": 1, "vy": 2, "my": 2, "vz": 3, "mz": 3, "P": 4, "E": 4}
_STAGES = {"euler": 1, "ssprk2": 2, "ssprk3": 3, "rk4": 4}


def _ic_functions(w0, hs, w0_passives, conservative_ic, fv_ic, gamma, h, p):
    """(w0, u0, u0_fv) callables of an initial condition, as EulerSolver.__init__
    builds them (fvhoe/solver.py:354-399)."""
    ic_func = w0.build_ic(hs, w0_passives)
    if not {"x", "y", "z"}.issubset(inspect.signature(ic_func).parameters):
        raise ValueError("Initial condition function must accept x, y, z as arguments.")
    if conservative_ic and fv_ic:
        return NotImplemented, NotImplemented, ic_func
    if fv_ic:
        raise ValueError("Can't have finite volume averages without conservative IC.")
    if conservative_ic:
        w0f, u0 = NotImplemented, ic_func
    else:
        w0f = ic_func
        u0 = lambda x, y, z: compute_conservatives(hs, ic_func(x, y, z), gamma=gamma)  # noqa: E731
    return w0f, u0, lambda x, y, z: fv_average(u0, x, y, z, h=h, p=p)


def initial_state(w0, nx: int, ny: int, nz: int = 1, px: int = 0, py: int = 0, pz: int = 0, x=(0, 1), y=(0, 1),
                  z=(0, 1), gamma: float = 5 / 3, conservative_ic: bool = False, fv_ic: bool = False) -> np.ndarray:
    """The conserved initial state (5, nx, ny, nz) float64 an EulerSolver with
    these arguments starts from, without building the solver."""
    n = (nx, ny, nz)
    h = ((x[1] - x[0]) / nx, (y[1] - y[0]) / ny, (z[1] - z[0]) / nz)
    X, Y, Z = fv_uniform_meshgen(n, x, y, z)
    _, _, u0_fv = _ic_functions(w0, HydroState(), None, conservative_ic, fv_ic, gamma, h, (px, py, pz))
    return np.ascontiguousarray(u0_fv(X, Y, Z), dtype=np.float64)


class EulerSolver(ODE):
    def __init__(
        self,
        w0: InitialCondition = None,
        w0_passives: Dict[str, Callable] = None,
        nx: int = 1,
        ny: int = 1,
        nz: int = 1,
        px: int = 0,
        py: int = 0,
        pz: int = 0,
        x: Tuple[float, float] = (0, 1),
        y: Tuple[float, float] = (0, 1),
        z: Tuple[float, float] = (0, 1),
        CFL: float = 0.8,
        fixed_dt: float = None,
        gamma: float = 5 / 3,
        bc: BoundaryCondition = None,
        riemann_solver: str = "hllc",
        conservative_ic: bool = False,
        fv_ic: bool = False,
        fixed_primitive_variables: Iterable = None,
        a_posteriori_slope_limiting: bool = False,
        slope_limiter: str = "minmod",
        force_trouble: bool = False,
        NAD: float = 1e-2,
        NAD_mode: str = "global",
        NAD_range: str = "relative",
        NAD_vars: tuple = None,
        PAD: dict = None,
        SED: bool = True,
        SED_tolerance: float = 1e-10,
        convex: bool = False,
        density_floor: float = None,
        pressure_floor: float = None,
        csq_floor: float = 1e-10,
        progress_bar: bool = True,
        snapshots_as_fv_averages: bool = True,
        snapshot_helper_function: callable = None,
        slab_buffer_size: int = 30,
        cupy: bool = False,
        backend: str = None,
        precision: str = "fp64",
        log_troubles: bool = True,
        kernel_path: str = "auto",
        ic_on_device: bool = False,
    ):
        if backend is None:
            backend = os.environ.get("FVHOE_BACKEND", "cuda")
        if backend != "cuda":
            raise ValueError("this EulerSolver runs on the 'cuda' backend only")
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        from . import _capi  # raises when libfvh.so is missing

        self._capi = _capi
        if kernel_path not in _capi.PATH:
            raise ValueError(f"kernel_path must be one of {sorted(_capi.PATH)}")
        self.kernel_path = kernel_path
        self.backend = backend
        self.precision = precision
        self.csq_floor = csq_floor
        self.density_floor = density_floor
        self.gamma = gamma
        self.pressure_floor = pressure_floor
        self.riemann_solver_name = riemann_solver
        self.snapshot_helper_function = snapshot_helper_function
        self.snapshots_as_fv_averages = snapshots_as_fv_averages
        self.fixed_primitive_variables = fixed_primitive_variables
        self.slab_buffer_size = slab_buffer_size
        self.ic_on_device = bool(ic_on_device)
        if riemann_solver not in _capi.RIEMANN:
            raise TypeError(f"Invalid Riemann solver {riemann_solver}")
        self._init_mesh(x, y, z, nx, ny, nz, px, py, pz, CFL, fixed_dt)
        self._init_initial_conditions(w0 if w0 is not None else Square(), w0_passives, conservative_ic, fv_ic,
                                      progress_bar)
        self._init_boundary_conditions(bc)
        self._init_slope_limiting(a_posteriori_slope_limiting, slope_limiter, force_trouble, NAD, NAD_mode,
                                  NAD_range, NAD_vars, PAD, SED, SED_tolerance, convex)
        self._log_enabled = bool(log_troubles) and self.a_posteriori_slope_limiting
        self._create_handle()
        self._init_array_allocation()
        self.timer.add_cat(
            [
                "boundary conditions",
                "(high-order) hydrofluxes",
                "(high-order) riemann solver",
                "(high-order) conservative interpolation",
                "(high-order) transverse reconstruction",
                "(fallback scheme)",
                "(fallback scheme) troubled cell detection",
                "(fallback scheme) hydrofluxes",
                "(fallback scheme) riemann solver",
                "(fallback scheme) conservative interpolation",
                "(fallback scheme) transverse reconstruction",
            ]
        )

    # -- set-up (fvhoe/solver.py:220-420) ----------------------------------------
    def _init_mesh(self, x, y, z, nx, ny, nz, px, py, pz, CFL, fixed_dt):
        self.CFL = CFL
        self.fixed_dt = fixed_dt
        self.x_domain, self.y_domain, self.z_domain = x, y, z
        self.h = ((x[1] - x[0]) / nx, (y[1] - y[0]) / ny, (z[1] - z[0]) / nz)
        self.n = (nx, ny, nz)
        self.p = (px, py, pz)
        self.X, self.Y, self.Z = fv_uniform_meshgen(self.n, x, y, z)
        self.x = self.X[:, 0, 0]
        self.y = self.Y[0, :, 0]
        self.z = self.Z[0, 0, :]
        self.xdim = not (nx == 1 and px == 0)
        self.ydim = not (ny == 1 and py == 0)
        self.zdim = not (nz == 1 and pz == 0)
        self.dims = "".join(d for d, on in zip("xyz", (self.xdim, self.ydim, self.zdim)) if on)
        self.ndim = len(self.dims)

    def _init_initial_conditions(self, w0, w0_passives, conservative_ic, fv_ic, progress_bar):
        self.conservative_ic = conservative_ic
        self.fv_ic = fv_ic
        passives = tuple(w0_passives.keys()) if w0_passives is not None else ()
        self.hydro_state = HydroState(passive_scalars=passives)
        hs = self.hydro_state
        self.nvars = hs.nvars
        self.w0, self.u0, self.u0_fv = _ic_functions(w0, hs, w0_passives, conservative_ic, fv_ic, self.gamma, self.h,
                                                     self.p)
        self._ode_init(progress_bar)
        self.am = ArrayManager(backend="cuda")
        if self.ic_on_device:
            self.am.add_device("u", self._device_initial_state())
        else:
            self.am.add("u", np.ascontiguousarray(self.u0_fv(self.X, self.Y, self.Z), dtype=np.float64))
        self.f_evaluation_count = 0

    def _device_initial_state(self):
        """The FV-averaged initial state evaluated on the device: the same
        quadrature over the same mesh coordinates (uploaded from the host), with
        the initial condition's own array code running on torch tensors
        (array_ns). Library initial conditions support it; an initial condition
        written for numpy arrays only is refused."""
        import torch

        dev = torch.device(self.am.device)
        X, Y, Z = torch.meshgrid(*(torch.from_numpy(np.ascontiguousarray(c)).to(dev) for c in (self.x, self.y, self.z)),
                                 indexing="ij")
        try:
            u0 = self.u0_fv(X, Y, Z)
        except (TypeError, AttributeError, RuntimeError) as exc:
            raise TypeError("ic_on_device needs an initial condition written against fvhoe_b200.array_ns "
                            f"(the library's are); this one failed on device tensors: {exc}") from exc
        if not isinstance(u0, torch.Tensor):
            raise TypeError("ic_on_device: the initial condition returned a host array")
        return u0.to(dtype=torch.float64).contiguous()

    def _init_boundary_conditions(self, bc):
        if bc is None:
            bc = BoundaryCondition(x="periodic", y="periodic", z="periodic")
        self.bc = bc
        self._bc_kinds = bc.kinds((self.xdim, self.ydim, self.zdim))

    def _init_slope_limiting(self, a_posteriori_slope_limiting, slope_limiter, force_trouble, NAD, NAD_mode,
                             NAD_range, NAD_vars, PAD, SED, SED_tolerance, convex):
        self.a_posteriori_slope_limiting = a_posteriori_slope_limiting
        self.slope_limiter = slope_limiter
        self.force_trouble = force_trouble
        self.NAD = NAD
        self.NAD_mode = NAD_mode
        self.NAD_range = NAD_range
        self.NAD_vars = NAD_vars if isinstance(NAD_vars, tuple) or NAD_vars is None else tuple(NAD_vars)
        self.PAD = {"rho": (0.0, np.inf), "P": (0.0, np.inf)} if PAD is None else PAD
        self.SED = SED
        self.SED_tolerance = SED_tolerance
        self.convex = convex
        self.trouble_counter = 1
        if NAD_mode not in ("global", "local"):
            raise ValueError(f"Unknown mode: {NAD_mode}")
        if NAD_range not in ("relative", "absolute"):
            raise ValueError(f"Unknown range_type: {NAD_range}")
        if slope_limiter not in self._capi.LIMITER:
            raise ValueError(f"Unknown slope limiter: {slope_limiter}")

    def _config(self):
        c = self._capi
        cfg = c.default_config()
        cfg.nvars = self.nvars
        for a in range(3):
            cfg.n[a] = self.n[a]
            cfg.p[a] = self.p[a]
            cfg.h[a] = self.h[a]
            for side in range(2):
                kind = self._bc_kinds[a][side]
                if kind == "ic":
                    kind = "dirichlet"
                cfg.bc[a][side] = c.BC.get(kind, 0) if kind is not None else 0
        cfg.dmr_split = self._dmr_split() if self._bc_kinds[1][0] == DMR_Y0 else 0
        cfg.gamma = self.gamma
        cfg.cfl = self.CFL
        cfg.csq_floor = self.csq_floor
        cfg.use_fixed_dt = 0 if self.fixed_dt is None else 1
        cfg.fixed_dt = 0.0 if self.fixed_dt is None else float(self.fixed_dt)
        cfg.riemann = c.RIEMANN[self.riemann_solver_name]
        cfg.a_posteriori = int(bool(self.a_posteriori_slope_limiting))
        cfg.slope_limiter = c.LIMITER[self.slope_limiter]
        cfg.force_trouble = int(bool(self.force_trouble))
        cfg.nad_eps = float(self.NAD)
        cfg.nad_global = int(self.NAD_mode == "global")
        cfg.nad_relative = int(self.NAD_range == "relative")
        mask = 0x1F
        if self.NAD_vars is not None:
            mask = 0
            for v in self.NAD_vars:
                mask |= 1 << _VAR_INDEX[v]
        cfg.nad_var_mask = mask
        # only the last PAD entry takes effect, as in fvhoe/slope_limiting.py:229-237
        if self.PAD:
            var, (lo, hi) = list(self.PAD.items())[-1]
            cfg.pad_var = _VAR_INDEX[var]
            cfg.pad_lo = float(lo)
            cfg.pad_hi = float(hi)
        else:
            cfg.pad_var = -1
        cfg.sed = int(bool(self.SED))
        cfg.sed_eps = float(self.SED_tolerance)
        cfg.convex = int(bool(self.convex))
        cfg.precision = c.PRECISION[self.precision]
        cfg.log_troubles = int(self._log_enabled)
        cfg.device = int(self.am("u").device.index or 0)
        cfg.kernel_path = c.PATH[self.kernel_path]
        return cfg

    def _dmr_split(self) -> int:
        from .boundary_conditions import dmr_split

        active = (self.xdim, self.ydim, self.zdim)
        buffer = tuple(self.slab_buffer_size if on else 0 for on in active)
        return dmr_split(self.n, self.x_domain, self.y_domain, self.z_domain, buffer)

    def _create_handle(self):
        import torch

        c = self._capi
        self._cfg = self._config()
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.am("u").device):
            c.check(c.lib.fvh_create(ctypes.byref(self._cfg), ctypes.byref(handle)))
        self._handle = handle
        self._predictor = None
        self.pred_totals = None
        self._init_dirichlet()

    # -- Dirichlet and "ic" boundaries (fvhoe/boundary_conditions.py:18-55, 334-347) --------
    def _init_dirichlet(self):
        """Slab coordinates of every Dirichlet side, built like the reference
        (slab_buffer_size cells on the active axes, fvhoe/solver.py:318-361),
        trimmed to the ghost depth the kernels read, and the static values."""
        self._dirichlet = []
        active = (self.xdim, self.ydim, self.zdim)
        sides = [(a, s) for a in range(3) if active[a] for s in range(2)
                 if self._bc_kinds[a][s] in ("dirichlet", "ic")]
        if not sides:
            return
        from .fv import slab_meshgen, trim_slab

        c = self._capi
        # ghost layers along every active axis (the slabs span the other axes' ghost layers too)
        depth = [self.gW_depth(a) if active[a] else 0 for a in range(3)]
        for a, s in sides:
            d = ctypes.c_int()
            c.check(c.lib.fvh_boundary_layout(self._handle, a, s, ctypes.byref(d), None, None), self._handle)
            if d.value != depth[a]:
                raise RuntimeError(f"ghost depth mismatch on axis {a}: library {d.value}, host {depth[a]}")
        buffer = tuple(self.slab_buffer_size if on else 0 for on in active)
        coords = slab_meshgen(self.n, self.x_domain, self.y_domain, self.z_domain, buffer)
        for a, s in sides:
            dim, pos = "xyz"[a], "lr"[s]
            X, Y, Z = trim_slab(coords[dim + pos], buffer, tuple(depth), a, pos)
            kind = self._bc_kinds[a][s]
            value = getattr(self.bc, f"{dim}_value")[s]
            if kind == "ic":
                if self.u0 is NotImplemented:
                    raise ValueError("'ic' boundaries need a pointwise conservative initial condition")
                value = self.u0
            self._dirichlet.append(dict(axis=a, side=s, kind=kind, value=value, coords=(X, Y, Z)))
        self._dirichlet_dynamic = any(d["kind"] == "dirichlet" and callable(d["value"]) for d in self._dirichlet)
        self._upload_boundaries(force=True)

    def gW_depth(self, a: int) -> int:
        """Ghost layers the kernels read along axis a: max(gw, 3 if limiting) + 2 ceil(p_a / 2)."""
        p = [pi for pi, on in zip(self.p, (self.xdim, self.ydim, self.zdim)) if on]
        r = -(-max(p) // 2)
        gw = max(r + 1, 2 * r)
        if self.a_posteriori_slope_limiting:
            gw = max(gw, 3)
        return gw + 2 * (-(-self.p[a] // 2))

    def _upload_boundaries(self, force=False):
        if not self._dirichlet or not (force or self._dirichlet_dynamic):
            return
        c = self._capi
        for d in self._dirichlet:
            X, Y, Z = d["coords"]
            value = d["value"]
            if d["kind"] == "ic":
                if not force:
                    continue
                vals = value(x=X, y=Y, z=Z)
            elif callable(value):
                vals = value(x=X, y=Y, z=Z, t=self.t)
            else:
                vals = np.ones((self.nvars,) + X.shape) * np.asarray(value).reshape(-1, 1, 1, 1)
            vals = np.ascontiguousarray(vals, dtype=np.float64)
            count = ctypes.c_size_t()
            c.check(c.lib.fvh_boundary_layout(self._handle, d["axis"], d["side"], None, None, ctypes.byref(count)),
                    self._handle)
            if vals.size != count.value:
                raise ValueError(f"boundary values of shape {vals.shape} do not fill the {count.value} ghost values "
                                 f"of side {'xyz'[d['axis']]}{'lr'[d['side']]}")
            c.check(c.lib.fvh_set_boundary_values(self._handle, d["axis"], d["side"],
                                                  vals.ctypes.data_as(ctypes.c_void_p), self._stream()),
                    self._handle)

    # -- learned troubled-cell predictor (no counterpart in the reference) ------
    def set_predictor(self, predictor, threshold: float = 0.5, every: int = 1):
        """Attaches a TroubledCellPredictor (None detaches). Needs the fused 2D
        path, a-posteriori limiting and global NAD. Faces next to predicted
        cells take the fallback flux; the a-posteriori check still runs on every
        cell and revises the faces of cells the network missed. The network runs
        every `every` stages and its flags are reused in the stages between."""
        m = predictor._m if predictor is not None else None
        if int(every) < 1:
            raise ValueError("every must be a positive number of stages")
        self._capi.check(self._capi.lib.fvh_set_predictor(self._handle, m, float(threshold)), self._handle)
        self._capi.check(self._capi.lib.fvh_set_predictor_interval(self._handle, int(every)), self._handle)
        self._predictor = predictor
        self.pred_totals = dict(predicted=0, troubled=0, missed=0, false_alarm=0, cell_stages=0)

    def _count_predictions(self, stages):
        if self._predictor is None:
            return
        st = self._capi.FvhPredStats()
        self._capi.check(self._capi.lib.fvh_get_pred_stats(self._handle, ctypes.byref(st), self._stream()),
                         self._handle)
        for k in ("predicted", "troubled", "missed", "false_alarm", "revised_faces", "flux_fallback_faces"):
            self.pred_totals[k] = self.pred_totals.get(k, 0) + int(getattr(st, k))
        self.pred_totals["cell_stages"] += stages * int(np.prod(self.n))

    def predictor_rates(self) -> dict:
        """Miss rate (missed / troubled) and false-alarm rate (false alarms /
        untroubled) accumulated over every stage since set_predictor."""
        t = dict(self.pred_totals or {})
        if not t:
            return t
        untroubled = t["cell_stages"] - t["troubled"]
        t["miss_rate"] = t["missed"] / t["troubled"] if t["troubled"] else 0.0
        t["false_alarm_rate"] = t["false_alarm"] / untroubled if untroubled else 0.0
        return t

    def predicted_flags(self) -> np.ndarray:
        """Predicted flags (uint8, (nx, ny, nz)) of the last stage."""
        import torch

        out = torch.empty(self.n, dtype=torch.uint8, device=self.am("u").device)
        self._capi.check(
            self._capi.lib.fvh_pred_flags(self._handle, ctypes.c_void_p(out.data_ptr()), self._stream()),
            self._handle,
        )
        return out.cpu().numpy()

    def _init_array_allocation(self):
        self.am.add("w", np.zeros((self.nvars,) + self.n))
        self._dudt = None
        self._copy_stream = None  # snapshot copies to the host
        self._pending_snapshots = []

    def __del__(self):
        handle = getattr(self, "_handle", None)
        # at interpreter exit the CUDA runtime may already be torn down; the process frees everything
        if handle is not None and handle.value and not sys.is_finalizing():
            try:
                self._capi.lib.fvh_destroy(handle)
            except Exception:
                pass
            self._handle = None

    # -- device calls -------------------------------------------------------------
    def _stream(self):
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream(self.am("u").device).cuda_stream)

    def _as_device(self, u):
        import torch

        if isinstance(u, np.ndarray):
            u = torch.from_numpy(np.ascontiguousarray(u, dtype=np.float64)).to(self.am("u").device)
        if u.dtype != torch.float64 or not u.is_contiguous() or tuple(u.shape) != (self.nvars,) + self.n:
            raise ValueError(f"u must be a contiguous float64 array of shape {(self.nvars,) + self.n}")
        return u

    def _set_log_mode(self):
        if self._log_enabled:
            self._capi.check(self._capi.lib.fvh_set_log_mode(self._handle, 1 if self.trouble_counter == 0 else 2),
                             self._handle)

    def f(self, t, u):
        """One right-hand-side evaluation: (dt, dudt) (fvhoe/solver.py:422-454)."""
        import torch

        self.f_evaluation_count += 1
        u = self._as_device(u)
        dudt = torch.empty_like(u)
        dt = ctypes.c_double()
        self._upload_boundaries()
        self._set_log_mode()
        self._capi.check(
            self._capi.lib.fvh_rhs(self._handle, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(dudt.data_ptr()),
                                   ctypes.byref(dt), self._stream()),
            self._handle,
        )
        if self._log_enabled:
            self.trouble_counter += 1
        self._count_predictions(1)
        return dt.value, dudt

    def hydrodynamics(self, u):
        return self.f(self.t, u)

    def _device_step(self, integrator, target_time):
        if integrator not in _STAGES:
            raise ValueError(f"unknown integrator {integrator}")
        u = self.am("u")
        dt = ctypes.c_double()
        self._upload_boundaries()
        self._set_log_mode()
        if self._log_enabled:
            # the division step_helper_function would apply after this step, done by the step's last stage
            self._capi.check(self._capi.lib.fvh_set_log_divisor(
                self._handle, float(self.trouble_counter + _STAGES[integrator])), self._handle)
            self._logs_divided = True
        self._capi.check(
            self._capi.lib.fvh_step(
                self._handle, ctypes.c_void_p(u.data_ptr()), self._capi.INTEGRATOR[integrator], float(self.t),
                0 if target_time is None else 1, 0.0 if target_time is None else float(target_time),
                ctypes.byref(dt), self._stream()),
            self._handle,
        )
        self.f_evaluation_count += _STAGES[integrator]
        if self._log_enabled:
            self.trouble_counter += _STAGES[integrator]
        self._count_predictions(_STAGES[integrator])
        return dt.value

    def step_helper_function(self):
        # log_troubles(reset=True) of fvhoe/solver.py:809-820
        if self._log_enabled and self.trouble_counter > 0:
            if not getattr(self, "_logs_divided", False):
                self._capi.check(
                    self._capi.lib.fvh_trouble_log(self._handle, float(self.trouble_counter), None, None, None,
                                                   self._stream()),
                    self._handle,
                )
            self._logs_divided = False
            self.trouble_counter = 0

    def trouble_flags(self) -> np.ndarray:
        """Trouble flags (uint8, (nx, ny, nz)) of the last stage."""
        import torch

        out = torch.empty(self.n, dtype=torch.uint8, device=self.am("u").device)
        self._capi.check(
            self._capi.lib.fvh_trouble_flags(self._handle, ctypes.c_void_p(out.data_ptr()), self._stream()),
            self._handle,
        )
        return out.cpu().numpy()

    def stats(self) -> dict:
        st = self._capi.FvhStats()
        self._capi.check(self._capi.lib.fvh_get_stats(self._handle, ctypes.byref(st), self._stream()), self._handle)
        return dict(dt_stage=st.dt_stage, dt_step=st.dt_step, troubled=st.troubled, nonfinite=st.nonfinite)

    def primitives(self, u=None, fv_average: bool = True):
        """FV-averaged (or cell-centre) primitives of u as a device tensor (fvhoe/solver.py:753-792)."""
        import torch

        u = self.am("u") if u is None else self._as_device(u)
        w = torch.empty_like(u)
        self._capi.check(
            self._capi.lib.fvh_primitives(self._handle, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                                          int(fv_average), self._stream()),
            self._handle,
        )
        return w

    def _trouble_logs_device(self):
        """The trouble logs of the run so far (trouble count, NAD and PAD
        magnitudes) as a new (3,) + n device tensor."""
        import torch

        t = torch.empty((3,) + self.n, dtype=torch.float64, device=self.am("u").device)
        self._capi.check(
            self._capi.lib.fvh_trouble_log(self._handle, 0.0, ctypes.c_void_p(t[0].data_ptr()),
                                           ctypes.c_void_p(t[1].data_ptr()), ctypes.c_void_p(t[2].data_ptr()),
                                           self._stream()),
            self._handle,
        )
        return t

    def _trouble_logs(self):
        """The trouble logs as three (5,) + n host arrays (synchronous)."""
        host = self._trouble_logs_device().cpu().numpy()
        return [np.broadcast_to(host[i], (5,) + self.n).copy() for i in range(3)]

    def _host_copy(self, t):
        """Enqueues the copy of device tensor t into pinned host memory on the
        snapshot copy stream, after the work queued so far on the solver's
        stream, and returns the host tensor (complete once the copy is)."""
        import torch

        main = torch.cuda.current_stream(t.device)
        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream(device=t.device)
        cs = self._copy_stream
        cs.wait_stream(main)
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        with torch.cuda.stream(cs):
            h.copy_(t, non_blocking=True)
        t.record_stream(cs)
        return h

    # -- snapshots (fvhoe/solver.py:835-953) -----------------------------------------
    def snapshot(self):
        """Records the snapshot dict of the reference (x, y, z, t, w and, with
        limiting, the trouble logs). The primitives and logs are computed on the
        device and copied to pinned host memory on a separate stream, so the
        copies overlap the following steps; reading `snapshots` (or calling the
        snapshot helper) first waits for the copies still in flight."""
        w = self.primitives(fv_average=self.snapshots_as_fv_averages)
        self.am("w").copy_(w)
        log = {"x": self.x, "y": self.y, "z": self.z, "t": self.t, "w": None}
        host_w = self._host_copy(w)
        apost = self.a_posteriori_slope_limiting
        host_logs = self._host_copy(self._trouble_logs_device()) if apost and self._log_enabled else None
        event = self._copy_stream.record_event()
        n = self.n

        def finish():
            log["w"] = host_w.numpy()
            if apost:
                if host_logs is not None:
                    host = host_logs.numpy()
                    trouble, nad, pad = [np.broadcast_to(host[i], (5,) + n).copy() for i in range(3)]
                else:
                    trouble = nad = pad = np.zeros((5,) + n)
                log["trouble"] = trouble
                log["NAD violation magnitude"] = nad
                log["PAD violation magnitude"] = pad

        self._pending_snapshots.append((event, finish))
        self.snapshots.append(log)
        self.snapshot_times.append(self.t)
        if self.snapshot_helper_function is not None:
            self._settle_snapshots()
            self.snapshot_helper_function(self)

    def _settle_snapshots(self):
        """Waits for the snapshot copies in flight and completes their entries."""
        pending = getattr(self, "_pending_snapshots", None)
        if not pending:
            return
        self._pending_snapshots = []
        for event, finish in pending:
            event.synchronize()
            finish()

    def read_snapshots(self) -> bool:
        if os.path.exists(self.snapshot_dir):
            with open(os.path.join(self.snapshot_dir, "arrs.pkl"), "rb") as fh:
                self.snapshots = SnapshotList(self._settle_snapshots, pickle.load(fh))
            print(f"Read from snapshot directory {self.snapshot_dir}")
            return True
        return False

    def write_snapshots(self, overwrite: bool):
        d = self.snapshot_dir
        if os.path.exists(d) and not overwrite:
            raise FileExistsError(f"Snapshot directory {d} already exists.")
        if os.path.exists(d) and overwrite:
            shutil.rmtree(d)
            print(f"Clearing out snapshot directory {d}")
        os.makedirs(d)
        with open(os.path.join(d, "arrs.pkl"), "wb") as fh:
            pickle.dump(self.snapshots, fh)
        attrs = {}
        for k, v in self.__dict__.items():
            if k == "w0":
                attrs[k] = getattr(v, "__name__", "__name__ not found")
                continue
            if k.startswith("_") or (callable(v) and k != "am") or isinstance(v, np.ndarray) or k in (
                    "progress_bar", "timestamps", "snapshots", "w0_cell_centers_cache", "hydro_state"):
                continue
            if k in ("am", "bc", "timer"):
                attrs[k] = v.to_dict()
                continue
            if k == "PAD":
                attrs[k] = {key: [{np.inf: "inf", -np.inf: "-inf"}.get(i, i) for i in val] for key, val in v.items()}
                continue
            try:
                json.dumps(v)
            except TypeError:
                continue
            attrs[k] = v
        attrs = {key: attrs[key] for key in sorted(attrs, key=lambda s: (s.lower(), s))}
        with open(os.path.join(d, "attrs.json"), "w") as fh:
            json.dump(attrs, fh, indent=4)
        with open(os.path.join(d, "timing.txt"), "w") as fh:
            fh.write(self.timer.report())
        print(f"Wrote to snapshot directory {d}")

    def run(self, *args, **kwargs):
        """Runge-Kutta order from the degree, up to RK4 (fvhoe/solver.py:955-974)."""
        q = min(max(self.p), 3)
        return (self.euler, self.ssprk2, self.ssprk3, self.rk4)[q](*args, **kwargs)

    def plot_1d_slice(self, *args, **kwargs):
        raise NotImplementedError("plotting needs matplotlib, which this package does not use")

    plot_2d_slice = plot_1d_slice
    plot_fields = plot_1d_slice
