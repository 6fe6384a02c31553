"""Batched ensemble on the GPU.

In FP64 every member of an ensemble equals the same problem advanced alone by
EulerSolver.ssprk3(t_end) — same step count, same final time, identical state
— for every tile variant that fits, with and without the CUDA graph. The
autotuner leaves the states as it found them.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T_END = 0.02


def _kw():
    from fvhoe_b200 import BoundaryCondition

    return dict(gamma=1.4, riemann_solver="hllc", CFL=0.8, bc=BoundaryCondition(x="outflow", y="outflow"),
                a_posteriori_slope_limiting=True, NAD=1e-4)


def _members():
    from fvhoe_b200 import FourQuadrant2D

    sizes = [(32, 32), (48, 40), (64, 64), (40, 56), (24, 72)]
    return [dict(w0=FourQuadrant2D(seed=10 + i), nx=a, ny=b) for i, (a, b) in enumerate(sizes)]


def _single(m, precision, p=3):
    from fvhoe_b200 import EulerSolver

    s = EulerSolver(w0=m["w0"], nx=m["nx"], ny=m["ny"], px=p, py=p, precision=precision, progress_bar=False,
                    **_kw())
    s.ssprk3(T_END)
    return s


@pytest.fixture(scope="module")
def singles64():
    return [_single(m, "fp64") for m in _members()]


def _ensemble(precision, p=3, use_graph=True):
    from fvhoe_b200 import Ensemble

    return Ensemble(_members(), px=p, precision=precision, use_graph=use_graph, **_kw())


def test_fp64_members_equal_single_runs_every_variant(singles64):
    variants = _ensemble("fp64").variants()
    tried = 0
    for info in variants:
        if info["max_blocks_per_sm"] <= 0:
            continue
        e2 = _ensemble("fp64")
        e2.configure(info["variant"])
        st = e2.run(T_END)
        assert st["active"] == 0 and st["nonfinite"] == 0
        for q, s in enumerate(singles64):
            assert st["steps"][q] == s.step_count, (info, q)
            assert st["t"][q] == s.t, (info, q)
            assert np.array_equal(e2.state(q), s.am.get_numpy("u")), (info, q)
        tried += 1
    assert tried >= 2


def test_graph_and_direct_launches_agree(singles64):
    a = _ensemble("fp64", use_graph=True)
    b = _ensemble("fp64", use_graph=False)
    sa = a.run(T_END)
    sb = b.run(T_END)
    assert a.graph_info()["graph"], a.graph_info()
    assert not b.graph_info()["graph"]
    assert np.array_equal(sa["steps"], sb["steps"])
    for q in range(len(a)):
        assert np.array_equal(a.state(q), b.state(q))
    assert sa["cell_updates"] == 3 * sum(int(s) * m["nx"] * m["ny"] for s, m in zip(sa["steps"], _members()))


def test_fp32_members_close_to_single_fp32_runs():
    ens = _ensemble("fp32")
    st = ens.run(T_END)
    for q, m in enumerate(_members()):
        s = _single(m, "fp32")
        assert st["steps"][q] == s.step_count
        assert abs(st["t"][q] - s.t) <= 1e-12
        u = s.am.get_numpy("u")
        d = np.max(np.abs(ens.state(q) - u))
        assert d <= 1e-9 * np.max(np.abs(u)), (q, d)


def test_autotune_keeps_states_and_picks_a_fitting_variant():
    ens = _ensemble("fp32")
    ens.reset(T_END)
    before = [ens.state(q) for q in range(len(ens))]
    choice = ens.autotune(steps=2)
    fits = {v["variant"] for v in ens.variants() if v["max_blocks_per_sm"] > 0}
    assert choice["variant"] in fits and choice["blocks_per_sm"] >= 1 and choice["ms_per_step"] > 0
    for q in range(len(ens)):
        assert np.array_equal(ens.state(q), before[q])
    st = ens.status()
    assert np.all(st["t"] == 0.0) and np.all(st["steps"] == 0)
