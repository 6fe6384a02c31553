"""Benchmark: Mcell-updates/s of FVHOE's per-stage update on B200.

Workload: 2D Kelvin-Helmholtz, periodic unit square, 2048^2 cells, gamma 1.4,
p = 5, HLLC, SSP-RK3, CFL 0.8, a-posteriori NAD (1e-5, global relative) + PAD
with SED and the MUSCL/minmod fallback; the initial state is the seeded
synthetic KH band with per-cell vy noise of amplitude 1e-3. One bench step is
one SSP-RK3 step (3 stages), i.e. 3 * 2048^2 cell-updates, the reference's
own unit (cells x RK stages / time).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32]
  python bench.py --impl reference ...   # the reference algorithm on the host cores

With N > 1 (launched by torch.distributed.run) every rank advances its own
replica (a different noise seed); there is no data-path collective, the
timing is the maximum over ranks and `value` counts the cells of all ranks.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mcell-updates/s on 1 B200: chosen form vs plain FP64 at stated L1 error"
UNIT = "Mcell-updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"],
                    help="the chosen form; fp32 is also compared against the plain fp64 path")
    ap.add_argument("--accuracy-time", type=float, default=1.0,
                    help="common time at which the L1 density error against fp64 is taken (the config's t_end)")
    ap.add_argument("--accuracy-series", default="0.01,0.1,0.5",
                    help="earlier times at which the L1 density error is also stated (comma-separated)")
    ap.add_argument("--start-time", type=float, default=0.01,
                    help="time both forms are advanced to before the timed steps")
    ap.add_argument("--n", type=int, default=2048, help="cells per side")
    ap.add_argument("--p", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-sample", type=int, default=512, help="side of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain fp64 comparison (profiling runs)")
    ap.add_argument("--no-predictor", action="store_true", help="skip the learned-predictor leg")
    ap.add_argument("--pred-n", type=int, default=4096, help="cells per side of the learned-predictor leg")
    ap.add_argument("--pred-p", type=int, default=7)
    ap.add_argument("--pred-steps", type=int, default=10, help="timed steps of each form in the predictor leg")
    ap.add_argument("--pred-train-n", type=int, default=1024, help="side of the training runs")
    ap.add_argument("--pred-snapshots", type=int, default=16, help="stages sampled per training run")
    ap.add_argument("--pred-epochs", type=int, default=2)
    ap.add_argument("--pred-accuracy-time", type=float, default=0.02)
    ap.add_argument("--pred-every", type=int, default=3,
                    help="stages between predictions of the second learned form (3: once per SSP-RK3 step)")
    ap.add_argument("--no-sedov", action="store_true", help="skip the 3D Sedov leg")
    ap.add_argument("--sedov-n", type=int, default=256, help="cells per side of the 3D Sedov leg")
    ap.add_argument("--sedov-steps", type=int, default=5, help="timed steps of each form in the Sedov leg")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--ens-members", type=int, default=256)
    ap.add_argument("--ens-steps", type=int, default=10, help="timed ensemble steps")
    ap.add_argument("--ens-singles", type=int, default=16, help="members also timed one at a time")
    return ap.parse_args()


def workload_config(args, n=None):
    n = args.n if n is None else n
    return {
        "workload": f"2D Kelvin-Helmholtz {n}x{n}, p={args.p}, HLLC, SSP-RK3, CFL 0.8, "
                    "a-posteriori NAD 1e-5 + PAD + SED, MUSCL-minmod fallback, periodic",
        "cells": n * n,
        "p": args.p,
        "riemann": "hllc",
        "integrator": "ssprk3",
        "precision": args.precision,
        "step": "SSP-RK3 step: 3 cell-updates per cell",
        "l2": "inputs larger than L2 (FP64 state 40 n^2 bytes)",
    }


def solver_kwargs(n, p, seed):
    """The KH workload; its initial state is averaged on the device (every
    solver of a comparison starts from the same state)."""
    from fvhoe_b200 import KelvinHelmholtzNoise2D

    return dict(w0=KelvinHelmholtzNoise2D(n=(n, n), seed=seed), nx=n, ny=n, px=p, py=p, gamma=1.4,
                riemann_solver="hllc", CFL=0.8, a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False,
                ic_on_device=True)


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        if args.impl == "reference":
            return rank, world, local, None
        import torch

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        return rank, world, local, dist
    return rank, world, local, None


def max_over_ranks(x, dist):
    """The maximum of x over the ranks (on the GPU with NCCL, on the host with gloo)."""
    if dist is None:
        return x
    import torch

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, ms_local, dist, world):
    """Whole-job Mcell-updates/s of `world` replicas that each did units_per_rank
    cell-updates: all units over the slowest rank's time. Returns (value, max ms)."""
    ms = max_over_ranks(ms_local, dist)
    return world * units_per_rank / (ms / 1e3) / 1e6, ms


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"fvh_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kind, n, p, precision):
    """DRAM bytes per launch of `kind` from the committed ncu summaries (lines
    `traffic <precision>_p<p> <kind> cells=C bytes=B`), scaled to n^2 cells."""
    import glob

    key = f"{precision}_p{p}"
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as fh:
            for line in fh:
                f = line.split()
                if len(f) == 5 and f[0] == "traffic" and f[1] == key and f[2] == kind:
                    cells = int(f[3].split("=")[1])
                    return int(f[4].split("=")[1]) * (n * n) / cells
    return None


def ncu_stage_traffic(n, p, precision):
    """DRAM bytes of one whole stage (every launch of the stage) from the line
    `traffic <precision>_p<p> stage cells=C bytes=B` of the ncu summaries,
    scaled to n^2 cells."""
    return ncu_traffic("stage", n, p, precision)


# FP64 pipe of a B200: 64 FP64 add / mul / fma per clock per SM, 148 SMs, 1.965 GHz
FP64_PEAK_OPS = 64 * 148 * 1.965e9


def fp64_ops_per_cell(p):
    """FP64 operations per cell-update of the plain path, counted by ncu from the
    kernels' executed DADD / DMUL / DFMA instructions (lines
    `fp64ops fp64_p<p> cells=C ops=O` of the ncu summaries: one stage of C cells)."""
    import glob

    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as fh:
            for line in fh:
                f = line.split()
                if len(f) == 4 and f[0] == "fp64ops" and f[1] == f"fp64_p{p}":
                    return int(f[3].split("=")[1]) / int(f[2].split("=")[1])
    return None


# ---------------------------------------------------------------------------
# CPU baselines (the oracle port of the reference algorithm)
# ---------------------------------------------------------------------------
def _oracle_sample(job):
    """One SSP-RK3 step of the KH workload on an n x n sample with the oracle; returns seconds."""
    n, p, seed = job
    import numpy as np

    sys.path.insert(0, ROOT)
    from fvhoe_b200.fv import fv_average, fv_uniform_meshgen
    from fvhoe_b200.hydro import HydroState, compute_conservatives
    from fvhoe_b200.initial_conditions import KelvinHelmholtzNoise2D
    from oracle import fvh_oracle as O

    hs = HydroState()
    f = KelvinHelmholtzNoise2D(n=(n, n), seed=seed).build_ic(hs)
    X, Y, Z = fv_uniform_meshgen((n, n, 1))
    h = (1 / n, 1 / n, 1.0)
    u0 = fv_average(lambda x, y, z: compute_conservatives(hs, f(x, y, z), 1.4), X, Y, Z, h=h, p=(p, p, 0))
    cfg = O.OracleConfig(n=(n, n, 1), p=(p, p, 0), h=h, gamma=1.4, riemann_solver="hllc", CFL=0.8,
                         a_posteriori_slope_limiting=True, NAD=1e-5)
    t0 = time.perf_counter()
    O.step(np.ascontiguousarray(u0), 0.0, cfg, "ssprk3")
    return time.perf_counter() - t0


def cpu_baseline_port(args):
    n = args.cpu_sample
    sec = _oracle_sample((n, args.p, 0))
    return {"value": 3 * n * n / sec / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one SSP-RK3 step of the same KH workload at {n}x{n} (p={args.p}) with the NumPy "
                      f"oracle (single-threaded NumPy, 1 core of {os.cpu_count()}); {sec:.1f} s"}


def run_reference(args):
    """The reference algorithm (the oracle port; the reference is pure Python and cannot be
    installed on the GPU host) on all host cores: each bench step runs one SSP-RK3 step of
    independent KH samples in parallel processes."""
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    side = 128 if args.steps > 30 else 192
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        for _ in range(args.warmup):
            pool.map(_oracle_sample, [(side, args.p, i) for i in range(cores)])
        t0 = time.perf_counter()
        for k in range(args.steps):
            pool.map(_oracle_sample, [(side, args.p, k * cores + i) for i in range(cores)])
        wall = time.perf_counter() - t0
    cell_updates = 3 * side * side * cores * args.steps
    value = cell_updates / wall / 1e6
    sample = (f"per bench step: {cores} processes each run one SSP-RK3 step of the KH workload at "
              f"{side}x{side} (p={args.p}) with the NumPy oracle port of the reference")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _time_steps(lib, _capi, h, uptr, sp, stream, steps):
    """CUDA-event time of `steps` SSP-RK3 steps issued as EulerSolver.take_step issues them,
    minus the dt read-back: the trouble log restarts, three stages accumulate into it, and
    the step's last stage divides it by 3."""
    import torch

    ssprk3 = _capi.INTEGRATOR["ssprk3"]

    def step():
        _capi.check(lib.fvh_set_log_mode(h, 1), h)
        _capi.check(lib.fvh_set_log_divisor(h, 3.0), h)
        _capi.check(lib.fvh_step(h, uptr, ssprk3, 0.0, 0, 0.0, None, sp), h)

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), step


def predictor_leg(args, stream, sp):
    """The learned troubled-cell predictor on KH at pred_n^2, p = pred_p, FP32 fused.

    1. Training rows from the plain FP64 solver: KH runs of two seeds and a
       four-quadrant Riemann run at pred_train_n^2, one right-hand-side
       evaluation every other step (features of every cell + its a-posteriori flag).
    2. Training on the GPU by the library's tensor-core kernels (Adam, BCE with
       positives weighted by the class ratio), held-out rates on a KH run of
       another seed.
    3. The same initial state advanced to a common time by the plain FP64 path,
       the FP32 fused path and the FP32 fused path with the predictor: L1 density
       errors against FP64, miss and false-alarm rates over those steps.
    4. Timed steps of each form (CUDA events, device-resident state)."""
    import ctypes

    import torch

    from fvhoe_b200 import (BoundaryCondition, EulerSolver, FourQuadrant2D, TroubledCellPredictor, _capi,
                            collect_training_data)

    lib = _capi.lib
    nt = args.pred_train_n
    every = 2
    steps = args.pred_snapshots * every
    t0 = time.perf_counter()
    runs = [EulerSolver(**solver_kwargs(nt, args.pred_p, seed=101)),
            EulerSolver(**solver_kwargs(nt, args.pred_p, seed=102)),
            EulerSolver(w0=FourQuadrant2D(seed=103), nx=nt, ny=nt, px=args.pred_p, py=args.pred_p, gamma=1.4,
                        riemann_solver="hllc", CFL=0.8, bc=BoundaryCondition(x="outflow", y="outflow"),
                        a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False, ic_on_device=True)]
    X, y = collect_training_data(runs, steps=steps, every=every)
    del runs
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = TroubledCellPredictor(device=torch.cuda.current_device(), seed=7)
    t0 = time.perf_counter()
    hist = net.fit(X, y, epochs=args.pred_epochs, batch=65536, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    rows = int(X.shape[0])
    positives = float(y.float().mean().item())
    del X, y
    held = EulerSolver(**solver_kwargs(nt, args.pred_p, seed=104))
    Xh, yh = collect_training_data([held], steps=8, every=4)
    held_rates = net.evaluate(Xh, yh, threshold=0.5)
    del Xh, yh, held

    n, p = args.pred_n, args.pred_p
    cells = n * n

    def make(precision, every=0):
        s = EulerSolver(precision=precision, **solver_kwargs(n, p, seed=0))
        if every:
            s.set_predictor(net, threshold=0.5, every=every)
        return s

    k = args.pred_every
    plain = make("fp64")
    fused = make("fp32")
    learned = make("fp32", every=1)
    learned_k = make("fp32", every=k)
    t_acc = args.pred_accuracy_time
    for s in (plain, fused, learned, learned_k):
        s.ssprk3(t_acc)
    rho = plain.am("u")[0]
    l1_fused = float(torch.mean(torch.abs(fused.am("u")[0] - rho)).item())
    l1_learned = float(torch.mean(torch.abs(learned.am("u")[0] - rho)).item())
    l1_learned_k = float(torch.mean(torch.abs(learned_k.am("u")[0] - rho)).item())
    rates = learned.predictor_rates()
    rates_k = learned_k.predictor_rates()

    def timed(s):
        h = s._handle
        up = ctypes.c_void_p(s.am("u").data_ptr())
        _time_steps(lib, _capi, h, up, sp, stream, args.warmup)
        ms, _ = _time_steps(lib, _capi, h, up, sp, stream, args.pred_steps)
        return 3 * cells * args.pred_steps / (ms / 1e3) / 1e6, ms / args.pred_steps

    v_plain, ms_plain = timed(plain)
    v_fused, ms_fused = timed(fused)
    v_learned, ms_learned = timed(learned)
    v_learned_k, ms_learned_k = timed(learned_k)
    lk = f"fp32_fused_learned_every{k}"

    def kind_ms(s, steps=2):
        """Per-kind milliseconds per step (CUDA events around each launch)."""
        h = s._handle
        _capi.check(lib.fvh_profile_enable(h, 1), h)
        up = ctypes.c_void_p(s.am("u").data_ptr())
        _time_steps(lib, _capi, h, up, sp, stream, steps)
        K = len(_capi.KERNEL_KINDS)
        pms = (ctypes.c_double * K)()
        plaunch = (ctypes.c_uint64 * K)()
        _capi.check(lib.fvh_profile_read(h, pms, None, plaunch, sp), h)
        _capi.check(lib.fvh_profile_enable(h, 0), h)
        return {nm: pms[i] / steps for i, nm in enumerate(_capi.KERNEL_KINDS) if plaunch[i]}

    # where the time goes: the predictor saves final-pass revisions and costs
    # inference plus fallback fluxes in the flux pass
    km_fused, km_learned, km_k = kind_ms(fused), kind_ms(learned), kind_ms(learned_k)
    shares = {nm: v / sum(km_learned.values()) for nm, v in km_learned.items()}

    def balance(km):
        saved = km_fused.get("final", 0.0) - km.get("final", 0.0)
        flux_added = km.get("face", 0.0) - km_fused.get("face", 0.0)
        infer = km.get("predict", 0.0)
        return {"final_pass_saved_ms_per_step": saved, "flux_pass_added_ms_per_step": flux_added,
                "inference_ms_per_step": infer, "net_ms_per_step": infer + flux_added - saved,
                "net_without_inference_ms_per_step": flux_added - saved}

    errors = net.errors()
    return {
        "config": f"2D Kelvin-Helmholtz {n}x{n}, p={p}, HLLC, SSP-RK3, CFL 0.8, NAD 1e-5 + PAD + SED, periodic",
        "network": "100 -> 64 -> 64 -> 1 GELU, BF16 tensor-core operands (tcgen05), FP32 accumulation",
        "training": {"rows": rows, "positive_fraction": positives, "epochs": args.pred_epochs,
                     "loss_per_epoch": hist, "data_seconds": t_data, "train_seconds": t_train,
                     "source": f"plain FP64 solver, KH seeds 101/102 and a four-quadrant run at {nt}^2, "
                               f"p={args.pred_p}, one stage every {every} steps over {steps} steps",
                     "held_out": held_rates},
        "prediction_interval": {"fp32_fused_learned": "every stage",
                                lk: f"every {k} stages, flags reused in between"},
        "mcell_updates_per_s": {"plain_fp64": v_plain, "fp32_fused": v_fused, "fp32_fused_learned": v_learned,
                                lk: v_learned_k},
        "ms_per_step": {"plain_fp64": ms_plain, "fp32_fused": ms_fused, "fp32_fused_learned": ms_learned,
                        lk: ms_learned_k},
        "speedup_vs_plain_fp64": {"fp32_fused": v_fused / v_plain, "fp32_fused_learned": v_learned / v_plain,
                                  lk: v_learned_k / v_plain},
        "l1_density_error_vs_fp64": {"t": t_acc, "steps": plain.step_count, "fp32_fused": l1_fused,
                                     "fp32_fused_learned": l1_learned, lk: l1_learned_k},
        "rates_over_l1_run": rates,
        "rates_over_l1_run_every": {lk: rates_k},
        "kernel_shares_learned": shares,
        "kernel_ms_per_step": {"fp32_fused": km_fused, "fp32_fused_learned": km_learned, lk: km_k},
        "balance_vs_fp32_fused": {"fp32_fused_learned": balance(km_learned), lk: balance(km_k)},
        "tensor_core_wait_errors": errors,
    }


def ensemble_members(count, seed=2024, side=None):
    """The batched-ensemble workload: square grids of side drawn uniformly from
    {128, 192, ..., 1024} (or all of one side), each a four-quadrant Riemann
    problem with its own seeded split point and states."""
    import numpy as np

    from fvhoe_b200 import FourQuadrant2D

    rng = np.random.default_rng(seed)
    sides = rng.choice(np.arange(128, 1025, 64), size=count) if side is None else np.full(count, side)
    return [dict(w0=FourQuadrant2D(seed=1000 + q), nx=int(s), ny=int(s)) for q, s in enumerate(sides)]


ENSEMBLE_KW = dict(gamma=1.4, riemann_solver="hllc", CFL=0.8, a_posteriori_slope_limiting=True, NAD=1e-5)


def sedov_leg(args, stream, sp):
    """The 3D Sedov configuration on the N-D kernels (the streaming primitive
    pass in FP32, the sliding-window detection, the compacting fallback, the
    generic sweeps for the rest): sedov_n^3 cells of
    [0,1]^3, p = 3, LLF, SSP-RK3, CFL 0.5, reflective at the x = 0, y = 0, z = 0
    faces and outflow elsewhere, a-posteriori MUSCL with NAD and PAD, the blast
    energy in the corner cell. Timed steps (CUDA events, state on the device) of
    the plain FP64 path and of the FP32 form, and the L1 density difference
    between the two after the same steps."""
    import ctypes

    import torch

    from fvhoe_b200 import BoundaryCondition, EulerSolver, SedovBlast, _capi

    lib = _capi.lib
    n = args.sedov_n
    cells = n ** 3
    bc = BoundaryCondition(x=("reflective", "outflow"), y=("reflective", "outflow"), z=("reflective", "outflow"))

    def make(precision):
        return EulerSolver(w0=SedovBlast(dims="xyz"), conservative_ic=True, fv_ic=True, nx=n, ny=n, nz=n, px=3,
                           py=3, pz=3, gamma=1.4, riemann_solver="llf", CFL=0.5, bc=bc,
                           a_posteriori_slope_limiting=True, progress_bar=False, precision=precision,
                           ic_on_device=True)

    out = {"config": f"3D Sedov {n}^3, p=3, LLF, SSP-RK3, CFL 0.5, reflective origin faces, outflow elsewhere, "
                     "a-posteriori MUSCL with NAD + PAD; N-D kernels", "cells": cells}
    rho = {}
    for precision in ("fp64", "fp32"):
        s = make(precision)
        up = ctypes.c_void_p(s.am("u").data_ptr())
        _time_steps(lib, _capi, s._handle, up, sp, stream, args.warmup)
        ms, _ = _time_steps(lib, _capi, s._handle, up, sp, stream, args.sedov_steps)
        out[precision] = {"mcell_updates_per_s": 3 * cells * args.sedov_steps / (ms / 1e3) / 1e6,
                          "ms_per_step": ms / args.sedov_steps, "scratch_bytes": lib.fvh_scratch_bytes(s._handle),
                          "nonfinite": s.stats()["nonfinite"]}
        # per-kind device time of one more step (CUDA events around each launch)
        h = s._handle
        _capi.check(lib.fvh_profile_enable(h, 1), h)
        _time_steps(lib, _capi, h, up, sp, stream, 1)
        K = len(_capi.KERNEL_KINDS)
        pms = (ctypes.c_double * K)()
        plaunch = (ctypes.c_uint64 * K)()
        _capi.check(lib.fvh_profile_read(h, pms, None, plaunch, sp), h)
        _capi.check(lib.fvh_profile_enable(h, 0), h)
        out[precision]["kernels_ms_per_step"] = {nm: round(pms[i], 3) for i, nm in enumerate(_capi.KERNEL_KINDS)
                                                 if plaunch[i]}
        out[precision]["launches_per_step"] = int(sum(plaunch))
        rho[precision] = s.am("u")[0].double().clone()
        del s
        torch.cuda.empty_cache()
    out["speedup_fp32_vs_fp64"] = out["fp32"]["mcell_updates_per_s"] / out["fp64"]["mcell_updates_per_s"]
    steps = args.warmup + args.sedov_steps
    out["l1_density_difference_fp32_vs_fp64"] = (rho["fp32"] - rho["fp64"]).abs().mean().item()
    out["note"] = f"both forms advanced {steps} steps from the same state, each with its own CFL dt"
    return out


def ensemble_leg(args, stream, members=None, label=None):
    """256 independent four-quadrant problems (p=3, HLLC, SSP-RK3, CFL 0.8,
    outflow, a-posteriori NAD 1e-5 + PAD + SED, FP32 with FP64 stage
    accumulation), target t_end = 0.2 each: autotuned tile shape and blocks per
    SM, CUDA-event time of ens_steps graph-replayed steps of the whole
    ensemble; then a sample of the members timed one at a time through the
    single-problem fused path, for the batching gain."""
    import torch

    from fvhoe_b200 import BoundaryCondition, Ensemble, EulerSolver

    if members is None:
        members = ensemble_members(args.ens_members)
        label = "square sides uniform in {128..1024 step 64}"
    kw = dict(ENSEMBLE_KW, bc=BoundaryCondition(x="outflow", y="outflow"))
    t0 = time.perf_counter()
    ens = Ensemble(members, px=3, precision="fp32", **kw)
    t_setup = time.perf_counter() - t0
    ens.reset(0.2)
    tune = ens.autotune(steps=2)
    ens.reset(0.2)
    ens.step(args.warmup)
    torch.cuda.synchronize()
    before = ens.status()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ens.step(args.ens_steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    after = ens.status()
    updates = after["cell_updates"] - before["cell_updates"]
    value = updates / (ms / 1e3) / 1e6
    graph = ens.graph_info()
    cells = int(sum(m["nx"] * m["ny"] for m in members))
    nbytes = ens.nbytes()
    del ens
    torch.cuda.empty_cache()
    # the same members one at a time (sampled): one fvh_step per member per step
    import numpy as np

    rng = np.random.default_rng(7)
    pick = sorted(rng.choice(len(members), size=min(args.ens_singles, len(members)), replace=False).tolist())
    single_updates = 0
    single_ms = 0.0
    for q in pick:
        m = members[q]
        s = EulerSolver(w0=m["w0"], nx=m["nx"], ny=m["ny"], px=3, py=3, precision="fp32", progress_bar=False,
                        log_troubles=False, **kw)
        # the stepper alone, like the ensemble (integrate() would add two snapshots per call)
        s.integrator = "ssprk3"
        for _ in range(args.warmup):
            s.take_step()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.ens_steps):
            s.take_step()
        b.record(stream)
        torch.cuda.synchronize()
        single_ms += a.elapsed_time(b)
        single_updates += 3 * args.ens_steps * m["nx"] * m["ny"]
        del s
    single_value = single_updates / (single_ms / 1e3) / 1e6
    return {
        "config": f"{len(members)} four-quadrant Riemann problems, {label} "
                  f"({cells} cells), p=3, HLLC, SSP-RK3, CFL 0.8, outflow, NAD 1e-5 + PAD + SED, FP32 with FP64 "
                  "stage accumulation, t_end = 0.2 each",
        "value": value, "unit": UNIT, "steps": args.ens_steps, "ms_per_step": ms / args.ens_steps,
        "cell_updates": int(updates), "active_after": after["active"], "nonfinite": after["nonfinite"],
        "autotune": tune, "graph": graph, "device_bytes": nbytes, "setup_seconds": t_setup,
        "one_at_a_time": {"members": len(pick), "value": single_value,
                          "path": "EulerSolver.take_step (SSP-RK3), one fused-path step per member and step, "
                                  "dt read back"},
        "batching_gain": value / single_value,
    }


def kernel_profile(lib, _capi, h, step, sp, args, value, precision=None):
    """Per-kind CUDA-event times of a few steps (each launch bracketed by an event
    pair) and the roofline of the dominant kind: its algorithmic bytes per
    launch over its measured duration, against the measured HBM peak; the
    whole-step fraction of the 120 B per cell-update model; the DRAM traffic per
    launch and per stage from the committed ncu summaries."""
    import ctypes

    precision = precision or args.precision
    _capi.check(lib.fvh_profile_enable(h, 1), h)
    prof_steps = 3
    for _ in range(prof_steps):
        step()
    K = len(_capi.KERNEL_KINDS)
    pms = (ctypes.c_double * K)()
    pbytes = (ctypes.c_double * K)()
    plaunch = (ctypes.c_uint64 * K)()
    _capi.check(lib.fvh_profile_read(h, pms, pbytes, plaunch, sp), h)
    _capi.check(lib.fvh_profile_enable(h, 0), h)
    total_ms = sum(pms)
    kinds = {}
    for i, name in enumerate(_capi.KERNEL_KINDS):
        if plaunch[i]:
            kinds[name] = {"ms_per_step": pms[i] / prof_steps, "share": pms[i] / total_ms,
                           "launches_per_step": plaunch[i] / prof_steps,
                           "gb_s": pbytes[i] / (pms[i] / 1e3) / 1e9 if pms[i] > 0 else None}
    dom = max(range(K), key=lambda i: pms[i])
    dom_name = _capi.KERNEL_KINDS[dom]
    per_launch_bytes = pbytes[dom] / plaunch[dom]
    per_launch_s = pms[dom] / plaunch[dom] / 1e3
    achieved = per_launch_bytes / per_launch_s / 1e9
    peak, peak_src = hbm_peak()
    traffic = ncu_traffic(dom_name, args.n, args.p, precision)
    step_gbs = 120 * value * 1e6 / 1e9
    stage = ncu_stage_traffic(args.n, args.p, precision)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": dom_name, "peak_source": f"{peak_src} HBM copy bandwidth",
                "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_s * 1e3,
                "step_frac": step_gbs / peak,
                "stage_model": {"bytes_per_cell_update": 120, "achieved_gb_s": step_gbs},
                "dram_bytes_per_stage": stage,
                "dram_over_algorithmic": stage / (120.0 * args.n * args.n) if stage else None}
    fp64 = fp64_ops_per_cell(args.p) if precision == "fp64" else None
    if fp64:
        rate = fp64 * value * 1e6  # FP64 operations per second at this throughput
        roofline["fp64"] = {"ops_per_cell_update": fp64, "achieved_tops": rate / 1e12,
                            "peak_tops": FP64_PEAK_OPS / 1e12, "frac": rate / FP64_PEAK_OPS,
                            "peak_model": "64 FP64 add/mul/fma per clock per SM x 148 SMs x 1.965 GHz "
                                          "(the FP64 pipe; no FMA contraction in the plain path)"}
    return kinds, roofline


def e2e_leg(lib, _capi, h, u, sp, stream, args, cells, world, dist):
    """End to end through the C ABI with the state in pinned host memory: every
    step copies the whole state in, steps it (dt read back) and copies it out.
    fvh_step_host pipelines the copies in chunks (a step's copy-out overlaps the
    next step's copy-in); the serial form (copy in, step, copy out, wait) is
    timed too for comparison."""
    import ctypes

    import torch

    host = torch.empty(u.shape, dtype=torch.float64, pin_memory=True)
    host.copy_(u)
    torch.cuda.synchronize()
    nbytes = u.numel() * 8
    dt = ctypes.c_double()
    ssprk3 = _capi.INTEGRATOR["ssprk3"]
    hptr = ctypes.c_void_p(host.data_ptr())
    uptr = ctypes.c_void_p(u.data_ptr())
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        _capi.check(lib.fvh_set_log_mode(h, 1), h)
        _capi.check(lib.fvh_set_log_divisor(h, 3.0), h)
        _capi.check(lib.fvh_step_host(h, hptr, ssprk3, 0.0, 0, 0.0, ctypes.byref(dt), sp), h)
    _capi.check(lib.fvh_host_sync(h), h)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        u.copy_(host, non_blocking=True)
        _capi.check(lib.fvh_set_log_mode(h, 1), h)
        _capi.check(lib.fvh_set_log_divisor(h, 3.0), h)
        _capi.check(lib.fvh_step(h, uptr, ssprk3, 0.0, 0, 0.0, ctypes.byref(dt), sp), h)
        host.copy_(u, non_blocking=True)
        stream.synchronize()
    serial_s = max_over_ranks(time.perf_counter() - t0, dist)
    return {"value": world * 3 * cells * args.e2e_steps / e2e_s / 1e6, "unit": UNIT,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": args.e2e_steps,
            "path": "fvh_step_host (C ABI), pinned host state copied in and out every step",
            "serial_value": world * 3 * cells * args.e2e_steps / serial_s / 1e6}


def accuracy_run(args, series, seed, stream):
    """The chosen form and plain FP64 from the same initial state to each time of
    `series` in turn (EulerSolver.ssprk3 with exact target hits, as the
    reference's integrate does): the L1 density error at every time, and each
    form's whole-run throughput (CUDA events around each segment, host loop
    and dt read-backs included)."""
    import torch

    from fvhoe_b200 import EulerSolver

    cells = args.n * args.n
    out = {"t": series[-1], "definition": "mean |rho_chosen - rho_fp64| over the grid at time t, same initial "
                                          "state, each form with its own CFL steps and exact target hits",
           "series": []}
    solvers = {"chosen": EulerSolver(precision=args.precision, **solver_kwargs(args.n, args.p, seed=seed)),
               "fp64": EulerSolver(precision="fp64", **solver_kwargs(args.n, args.p, seed=seed)),
               # the chaos floor: plain FP64 from the same state with every density moved by one ulp
               "fp64_ulp": EulerSolver(precision="fp64", **solver_kwargs(args.n, args.p, seed=seed))}
    rho = solvers["fp64_ulp"].am("u")[0]
    rho.copy_(torch.nextafter(rho, torch.full_like(rho, float("inf"))))
    run_ms = {k: 0.0 for k in solvers}
    for t in series:
        for name, sv in solvers.items():
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            sv.ssprk3(t)
            b.record(stream)
            torch.cuda.synchronize()
            run_ms[name] += a.elapsed_time(b)
        rho_c = solvers["chosen"].am("u")[0]
        rho_p = solvers["fp64"].am("u")[0]
        rho_u = solvers["fp64_ulp"].am("u")[0]
        out["series"].append({"t": t, "l1": float(torch.mean(torch.abs(rho_c - rho_p)).item()),
                              "l1_fp64_one_ulp": float(torch.mean(torch.abs(rho_u - rho_p)).item()),
                              "steps_chosen": solvers["chosen"].step_count,
                              "steps_fp64": solvers["fp64"].step_count})
    out["value"] = out["series"][-1]["l1"]
    out["chaos_floor"] = ("l1_fp64_one_ulp: the same plain FP64 run started from densities moved by one ulp; "
                          "KH amplifies any round-off difference, so no form can stay closer to FP64 than that")
    out["whole_run"] = {name: {"mcell_updates_per_s": 3 * cells * sv.step_count / (run_ms[name] / 1e3) / 1e6,
                               "steps": sv.step_count, "seconds": run_ms[name] / 1e3}
                        for name, sv in solvers.items() if name != "fp64_ulp"}
    out["whole_run"]["speedup_of_chosen"] = (out["whole_run"]["chosen"]["mcell_updates_per_s"] /
                                             out["whole_run"]["fp64"]["mcell_updates_per_s"])
    del solvers
    torch.cuda.empty_cache()
    return out


def leg_summary(legs):
    """The few figures of each leg that the headline line repeats (the legs
    are printed in full on their own lines before it)."""
    out = {}
    lp = legs.get("learned_predictor")
    if lp:
        out["learned_predictor"] = ({k: {f: round(x, 3) for f, x in lp[k].items()}
                                     for k in ("mcell_updates_per_s", "speedup_vs_plain_fp64")}
                                    if "error" not in lp else lp)
    sd = legs.get("sedov_3d")
    if sd:
        out["sedov_3d"] = ({k: sd[k]["mcell_updates_per_s"] for k in ("fp64", "fp32")} if "error" not in sd else sd)
    be = legs.get("batched_ensemble")
    if be:
        out["batched_ensemble"] = ({"value": be["value"], "batching_gain": be["batching_gain"],
                                    "small_members_gain": be.get("small_members", {}).get("batching_gain")}
                                   if "error" not in be else be)
    return out


def l1_summary(l1):
    """The headline's L1 figures: the error at t_end, and per time of the series
    [t, L1 of the chosen form, L1 of FP64 moved by one ulp (the chaos floor)]."""
    if l1 is None:
        return None
    return {"t": l1["t"], "value": l1["value"],
            "series": [[x["t"], x["l1"], x["l1_fp64_one_ulp"]] for x in l1["series"]],
            "series_columns": ["t", "l1", "l1_fp64_one_ulp"],
            "whole_run_speedup": l1["whole_run"]["speedup_of_chosen"]}


def run_ours(args):
    import ctypes

    import numpy as np
    import torch

    rank, world, local, dist = dist_setup(args)
    torch.cuda.set_device(local)
    from fvhoe_b200 import EulerSolver, _capi

    lib = _capi.lib
    cells = args.n * args.n
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    # the chosen form and the plain FP64 path on the same initial state, both first
    # advanced to t = 0.01 with the reference's stepper (the state the timed steps start from)
    t_start = args.start_time
    chosen = EulerSolver(precision=args.precision, **solver_kwargs(args.n, args.p, seed=rank))
    chosen.ssprk3(t_start)
    plain = None
    if args.precision != "fp64" and not args.no_plain:
        plain = EulerSolver(precision="fp64", **solver_kwargs(args.n, args.p, seed=rank))
        plain.ssprk3(t_start)

    h = chosen._handle
    u = chosen.am("u")
    uptr = ctypes.c_void_p(u.data_ptr())
    _, step = _time_steps(lib, _capi, h, uptr, sp, stream, args.warmup)

    # timed region of the chosen form (device-resident state)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = lib.fvh_kernel_launches()
    ms, _ = _time_steps(lib, _capi, h, uptr, sp, stream, args.steps)
    launches = lib.fvh_kernel_launches() - l0
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    value, ms = replica_throughput(3 * cells * args.steps, ms, dist, world)

    plain_line = None
    if plain is not None:
        hp = plain._handle
        up = ctypes.c_void_p(plain.am("u").data_ptr())
        _time_steps(lib, _capi, hp, up, sp, stream, args.warmup)
        if dist is not None:
            dist.barrier()
        msp, _ = _time_steps(lib, _capi, hp, up, sp, stream, args.steps)
        pv, msp = replica_throughput(3 * cells * args.steps, msp, dist, world)
        plain_line = {"value": pv, "ms_per_step": msp / args.steps, "speedup_of_chosen": value / pv}

    # per-kernel timing of a few steps for the roofline of the dominant kernel
    kinds, roofline = kernel_profile(lib, _capi, h, step, sp, args, value / world)
    if plain is not None:
        _, pstep = _time_steps(lib, _capi, hp, up, sp, stream, 0)
        pkinds, proof = kernel_profile(lib, _capi, hp, pstep, sp, args, plain_line["value"] / world, precision="fp64")
        plain_line["roofline"] = {k: proof[k] for k in ("kernel", "frac", "step_frac", "dram_over_algorithmic")}
        if "fp64" in proof:
            plain_line["roofline"]["fp64"] = {k: proof["fp64"][k] for k in ("ops_per_cell_update", "achieved_tops",
                                                                              "frac")}

    # end to end through the C ABI with the state in pinned host memory
    e2e = e2e_leg(lib, _capi, h, u, sp, stream, args, cells, world, dist)
    if plain is not None:
        pe = e2e_leg(lib, _capi, hp, plain.am("u"), sp, stream, args, cells, world, dist)
        plain_line["e2e"] = {k: pe[k] for k in ("value", "unit", "serial_value")}
        del plain
    stats = chosen.stats()
    del chosen
    torch.cuda.empty_cache()

    # L1 density error of the chosen form against plain FP64 at the config's t_end
    # (fresh solvers, the same stepper and targets), with the whole-run throughput
    l1 = None
    if args.precision != "fp64" and not args.no_plain and world == 1:
        series = [float(x) for x in args.accuracy_series.split(",") if x] + [args.accuracy_time]
        l1 = accuracy_run(args, series, seed=rank, stream=stream)

    if rank == 0:
        form = {"fp32": "FP32 reconstruction, Riemann fluxes and detection; FP64 stage accumulation",
                "fp64": "plain FP64, bit-exact with the reference"}[args.precision]
        legs = {}
        if world == 1 and not args.no_predictor:
            torch.cuda.empty_cache()
            try:
                legs["learned_predictor"] = predictor_leg(args, stream, sp)
            except Exception as exc:  # the headline line is printed whatever this leg does
                legs["learned_predictor"] = {"error": f"{type(exc).__name__}: {exc}"}
        if world == 1 and not args.no_sedov:
            torch.cuda.empty_cache()
            try:
                legs["sedov_3d"] = sedov_leg(args, stream, sp)
            except Exception as exc:
                legs["sedov_3d"] = {"error": f"{type(exc).__name__}: {exc}"}
        if world == 1 and not args.no_ensemble:
            torch.cuda.empty_cache()
            try:
                legs["batched_ensemble"] = ensemble_leg(args, stream)
                # where batching pays: many small members, launch- and host-bound one at a time
                legs["batched_ensemble"]["small_members"] = ensemble_leg(
                    args, stream, ensemble_members(args.ens_members, side=128), "all of side 128")
            except Exception as exc:
                legs["batched_ensemble"] = {"error": f"{type(exc).__name__}: {exc}"}
        # every leg in full on its own line, then the headline line last (compact)
        if l1 is not None:
            print("leg accuracy " + json.dumps(l1), flush=True)
        for name, leg in legs.items():
            print(f"leg {name} " + json.dumps(leg), flush=True)
        if kinds:
            print("leg kernels " + json.dumps(kinds), flush=True)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32", "data": "synthetic",
            "plain_fp64": plain_line, "l1_density_error_vs_fp64": l1_summary(l1),
            "config": dict(workload_config(args), parallelism=f"replicas x{world}" if world > 1 else "single",
                           timed_from=f"t = {t_start} (both forms advanced there first)"),
            "chosen_form": form, "roofline": roofline, "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
            "troubled_cells_last_stage": stats["troubled"], "nonfinite": stats["nonfinite"],
            "legs": leg_summary(legs),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_port(args)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    import faulthandler

    faulthandler.enable()
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
