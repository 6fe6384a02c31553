"""Learned troubled-cell predictor on the GPU.

* the tensor-core forward pass and gradients against the CPU oracle with the
  same BF16 operand rounding (tolerances below);
* features and labels extracted from a solver stage against the oracle's
  primitives and flags;
* the stage with a predictor attached equals, bit for bit in FP64, the
  oracle's stage with the fallback applied on (troubled | predicted) cells,
  with the a-posteriori flags unchanged;
* training: the network trained by the project's kernels on KH / four-quadrant
  runs predicts held-out flags far better than the untrained network, and,
  against the same run without a predictor, the final pass (the revision
  sweep) revises far fewer faces: the faces of predicted cells take their
  fallback flux in the flux pass instead.
"""

import os

import numpy as np
import pytest

from oracle import fvh_oracle as O
from oracle import mlp_oracle as mo
from tests.fixtures import golden_files, load, oracle_config, solver_kwargs

pytestmark = pytest.mark.gpu


def _rows(rng, n, scale=1.0):
    import torch

    X = np.zeros((n, mo.N_ROW), dtype=np.float32)
    X[:, :mo.N_IN] = np.clip(rng.normal(0, 0.5 * scale, (n, mo.N_IN)), -1, 1)
    Xb = mo.bf16(X)
    Xt = torch.from_numpy(mo.bf16_bits(X).view(np.int16)).view(torch.bfloat16).cuda()
    return Xb, Xt


def _net(seed=0):
    from fvhoe_b200 import TroubledCellPredictor

    return TroubledCellPredictor(device=0, seed=seed)


def test_logits_match_oracle():
    rng = np.random.default_rng(0)
    net = _net(1)
    Xb, Xt = _rows(rng, 1000)
    got = net.logits(Xt).cpu().numpy()
    ref = mo.forward(net.get_params(), Xb, bf16_operands=True)
    # FP32 accumulation order and erff / expf differences, amplified by at most one BF16 rounding of h1
    assert np.max(np.abs(got - ref)) <= 2e-2 * max(1.0, np.max(np.abs(ref))), np.max(np.abs(got - ref))
    assert np.corrcoef(got, ref)[0, 1] > 0.9999
    assert net.errors() == 0


@pytest.mark.parametrize("n", [128, 1000, 5000])
def test_gradients_match_oracle(n):
    import torch

    rng = np.random.default_rng(n)
    net = _net(2)
    p = net.get_params().copy()
    p[mo.B1:mo.W2] = rng.normal(0, 0.1, 64)
    p[mo.B2:mo.W3] = rng.normal(0, 0.1, 64)
    p[mo.B3] = -0.3
    net.set_params(p)
    Xb, Xt = _rows(rng, n)
    y = (rng.uniform(size=n) < 0.35).astype(np.uint8)
    g, loss = net.gradients(Xt, torch.from_numpy(y).cuda(), pos_weight=2.0)
    gr, lr = mo.gradients(p, Xb, y, 2.0, bf16_operands=True)
    assert abs(loss - lr) <= 1e-4 * abs(lr) + 1e-6
    for name, a, b in (("W1", mo.W1, mo.B1), ("b1", mo.B1, mo.W2), ("W2", mo.W2, mo.B2), ("b2", mo.B2, mo.W3),
                       ("w3", mo.W3, mo.B3), ("b3", mo.B3, mo.N_PARAMS)):
        d = np.abs(g[a:b] - gr[a:b])
        scale = np.max(np.abs(gr[a:b]))
        # relative to the block's largest entry; BF16 roundings of dz may flip between FP32 and FP64
        assert np.max(d) <= 2e-2 * scale + 1e-7, (name, np.max(d), scale)
        assert np.linalg.norm(d) <= 5e-3 * np.linalg.norm(gr[a:b]) + 1e-7, name
    assert net.errors() == 0


def test_train_step_reduces_loss():
    import torch

    rng = np.random.default_rng(5)
    net = _net(3)
    Xb, Xt = _rows(rng, 8192)
    # a learnable rule: flag rows whose first feature is large
    y = torch.from_numpy((Xb[:, 0] > 0.3).astype(np.uint8)).cuda()
    first = net.train_step(Xt, y, lr=3e-3, want_loss=True)
    for _ in range(150):
        last = net.train_step(Xt, y, lr=3e-3, want_loss=True)
    assert last < 0.5 * first, (first, last)
    assert net.errors() == 0


def _kh_solver(n, seed, p=3, **extra):
    from fvhoe_b200 import EulerSolver, KelvinHelmholtzNoise2D

    return EulerSolver(w0=KelvinHelmholtzNoise2D(n=(n, n), seed=seed), nx=n, ny=n, px=p, py=p, gamma=1.4,
                       a_posteriori_slope_limiting=True, NAD=1e-5, progress_bar=False, **extra)


def test_features_and_labels_match_oracle():
    import torch

    from fvhoe_b200 import _capi

    path = os.path.join(os.path.dirname(golden_files("rhs")[0]), "rhs_kh_p3.npz")
    c, d = load(path)
    from fvhoe_b200 import EulerSolver

    s = EulerSolver(**solver_kwargs(c, d["u0"]))
    s.f(0.0, s.am("u"))
    n = int(np.prod(s.n))
    X = torch.empty((n, mo.N_ROW), dtype=torch.bfloat16, device="cuda")
    y = torch.empty(n, dtype=torch.uint8, device="cuda")
    _capi.check(_capi.lib.fvh_mlp_features(s._handle, X.data_ptr(), y.data_ptr(), None), s._handle)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy().reshape(s.n), d["trouble"].astype(np.uint8))
    cfg = oracle_config(c)
    w = O.fv_primitives(d["u0"], cfg, cfg.p, [3, 3, 0])[:, :, :, 0]
    ranges = [w[v].max() - w[v].min() for v in (0, 1, 2, 4)]
    ref = mo.bf16(mo.features(w, (0, 1, 2, 4), ranges, ghosts=3).astype(np.float32))
    got = X.view(torch.int16).cpu().numpy().view(np.uint16)
    got = mo.from_bf16_bits(got)[:, :mo.N_IN]
    assert np.all(mo.from_bf16_bits(X.view(torch.int16).cpu().numpy().view(np.uint16))[:, mo.N_IN:] == 0)
    # one BF16 ulp (2^-8 relative) from float log1p against FP64
    assert np.all(np.abs(got - ref) <= 2 ** -7 * np.abs(ref) + 1e-6)


@pytest.mark.parametrize("name", ["rhs_kh_p3.npz", "rhs_kh_p5.npz", "rhs_quad_p3.npz"])
def test_predicted_stage_equals_oracle_blend(name):
    """FP64: faces of predicted cells take the fallback flux in the flux pass,
    missed cells are revised in the final pass; the result equals the oracle's
    stage with the fallback on (troubled | predicted), bit for bit."""
    from fvhoe_b200 import EulerSolver

    c, d = load(os.path.join(os.path.dirname(golden_files("rhs")[0]), name))
    s = EulerSolver(**solver_kwargs(c, d["u0"]))
    net = _net(7)
    # a threshold that flags a sizeable, imperfect subset
    s.set_predictor(net, threshold=0.5)
    dt, dudt = s.f(0.0, s.am("u"))
    pred = s.predicted_flags().astype(bool)
    trouble = s.trouble_flags().astype(bool)
    assert np.array_equal(trouble, d["trouble"].astype(bool))
    cfg = oracle_config(c)
    dt_ref, dudt_ref, _ = O.rhs(d["u0"], cfg, predicted=pred)
    assert dt == dt_ref
    assert np.array_equal(dudt.cpu().numpy(), dudt_ref)
    r = s.predictor_rates()
    assert r["predicted"] == int(pred.sum())
    assert r["troubled"] == int(trouble.sum())
    assert r["missed"] == int((trouble & ~pred).sum())
    assert r["false_alarm"] == int((pred & ~trouble).sum())
    assert 0 < r["predicted"] < pred.size
    assert net.errors() == 0


def test_trained_predictor_gains_over_untrained():
    """Train on KH runs of two seeds and a four-quadrant run; evaluate on a KH
    run of another seed. The trained network misses few troubled cells, far
    fewer than the untrained one at the same false-alarm budget, so the final
    pass revises only a small fraction of the troubled cells."""
    from fvhoe_b200 import BoundaryCondition, EulerSolver, FourQuadrant2D, collect_training_data

    train = [_kh_solver(128, 1), _kh_solver(128, 2),
             EulerSolver(w0=FourQuadrant2D(seed=4), nx=128, ny=128, px=3, py=3, gamma=1.4,
                         bc=BoundaryCondition(x="outflow", y="outflow"), a_posteriori_slope_limiting=True, NAD=1e-5,
                         progress_bar=False)]
    X, y = collect_training_data(train, steps=40, every=2)
    net = _net(11)
    untrained = _net(11)
    hist = net.fit(X, y, epochs=6, batch=8192, lr=3e-3)
    assert hist[-1] < hist[0]
    test = _kh_solver(128, 9)
    Xt, yt = collect_training_data([test], steps=40, every=4)
    thr = 0.5
    got = net.evaluate(Xt, yt, threshold=thr)
    base = untrained.evaluate(Xt, yt, threshold=thr)
    print("trained", got, "untrained", base)
    assert got["miss_rate"] < 0.2, got
    assert got["false_alarm_rate"] < 0.2, got
    assert got["miss_rate"] + got["false_alarm_rate"] < 0.5 * (base["miss_rate"] + base["false_alarm_rate"])
    # attached to a solver: the revision pass handles only the misses
    run = _kh_solver(128, 9)
    run.set_predictor(net, threshold=thr)
    run.ssprk3(n=10)
    r = run.predictor_rates()
    print("attached", r)
    assert r["missed"] < 0.2 * r["troubled"]
    assert net.errors() == 0
    # against the method without the predictor, on the same run: the final
    # pass (the revision sweep) revises far fewer faces, because the faces of
    # predicted cells took their fallback flux in the flux pass already
    import ctypes

    from fvhoe_b200 import _capi

    plain = _kh_solver(128, 9)
    plain.integrator = "ssprk3"
    revised_plain = 0
    for _ in range(10):
        plain.take_step()
        st = _capi.FvhPredStats()
        _capi.check(_capi.lib.fvh_get_pred_stats(plain._handle, ctypes.byref(st), plain._stream()), plain._handle)
        revised_plain += st.revised_faces
        assert st.flux_fallback_faces == 0
    print("final-pass revisions: plain", revised_plain, "with the predictor", r["revised_faces"],
          "flux-pass fallback faces", r["flux_fallback_faces"])
    assert revised_plain > 0
    assert r["revised_faces"] < 0.3 * revised_plain
    assert r["flux_fallback_faces"] > 0.5 * revised_plain


@pytest.mark.parametrize("every,launches", [(1, 6), (2, 3), (3, 2)])
def test_prediction_interval(every, launches):
    """With an interval of k stages the network runs on stages 0, k, 2k, ... and
    the stages between reuse its flags; the a-posteriori check still judges
    every stage, so the predictor counts cover all of them."""
    import ctypes

    from fvhoe_b200 import _capi

    n = 64
    s = _kh_solver(n, 1)
    s.set_predictor(_net(3), threshold=0.5, every=every)
    lib, h = _capi.lib, s._handle
    _capi.check(lib.fvh_profile_enable(h, 1), h)
    s.ssprk3(n=2)
    K = len(_capi.KERNEL_KINDS)
    ms = (ctypes.c_double * K)()
    count = (ctypes.c_uint64 * K)()
    _capi.check(lib.fvh_profile_read(h, ms, None, count, s._stream()), h)
    _capi.check(lib.fvh_profile_enable(h, 0), h)
    assert count[_capi.KERNEL_KINDS.index("predict")] == launches
    r = s.predictor_rates()
    assert r["cell_stages"] == 6 * n * n
    assert 0 <= r["missed"] <= r["troubled"]
    with pytest.raises(ValueError):
        s.set_predictor(_net(3), every=0)
