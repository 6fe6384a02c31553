"""Properties of the reference algorithm itself, shown on the oracle (CPU).

With a-posteriori limiting on a periodic domain the reference's update is not
conservative: its simple face broadcast (fvhoe/slope_limiting.py:364-380)
gives the face at x = 0 the weight of cell 0 only and the face at x = n that of
cell n-1 only, although on a periodic domain they are the same face, so the
two copies of a boundary face can blend different fluxes. The totals then
change by exactly the mismatch of the two copies; the interior faces
telescope. The CUDA path equals the oracle bit for bit (tests/test_gpu_golden.py,
tests/test_gpu_fullsize.py), so it has the same property; conservation to
round-off is checked where the scheme has it (no limiting, or walls).
"""

import numpy as np

from oracle import fvh_oracle as O


def _kh(n, p, seed=3):
    from fvhoe_b200 import KelvinHelmholtzNoise2D
    from fvhoe_b200.solver import initial_state

    return initial_state(KelvinHelmholtzNoise2D(n=(n, n), seed=seed), n, n, 1, p, p, 0, gamma=1.4)


def test_limited_periodic_update_changes_totals_by_the_boundary_face_mismatch(n=64, p=3):
    u0 = _kh(n, p)
    cfg = O.OracleConfig(n=(n, n, 1), p=(p, p, 0), h=(1 / n, 1 / n, 1.0), gamma=1.4, riemann_solver="hllc",
                         a_posteriori_slope_limiting=True, NAD=1e-5)
    _, dudt, info = O.rhs(u0, cfg)
    F, G, _ = info["fluxes"]
    assert info["trouble"].any()
    for v in range(5):
        # sum of -(F[i+1] - F[i]) / h over the cells: only the boundary copies remain
        expected = -n * (F[v, n, :, 0] - F[v, 0, :, 0]).sum() - n * (G[v, :, n, 0] - G[v, :, 0, 0]).sum()
        total = dudt[v].sum()
        scale = np.abs(dudt[v]).sum() + 1e-300
        assert abs(total - expected) <= 1e-12 * scale, (v, total, expected)
    # the mismatch is real: the copies of some boundary faces differ
    assert not (np.array_equal(F[:, n], F[:, 0]) and np.array_equal(G[:, :, n], G[:, :, 0]))


def test_unlimited_periodic_update_conserves(n=64, p=3):
    u0 = _kh(n, p)
    cfg = O.OracleConfig(n=(n, n, 1), p=(p, p, 0), h=(1 / n, 1 / n, 1.0), gamma=1.4, riemann_solver="hllc")
    _, dudt, info = O.rhs(u0, cfg)
    F, G, _ = info["fluxes"]
    assert np.array_equal(F[:, n], F[:, 0]) and np.array_equal(G[:, :, n], G[:, :, 0])
    for v in range(5):
        assert abs(dudt[v].sum()) <= 1e-12 * (np.abs(dudt[v]).sum() + 1e-300)
