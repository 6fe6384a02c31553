"""The oracle against the reference-generated golden fixtures (CPU).

Every fixture was produced by running jpalafou/FVHOE itself
(tests/golden/make_golden.py). The oracle must reproduce each one exactly:
the same dt, bit-identical dudt and states, identical trouble flags and
NAD/PAD magnitudes.
"""

import os

import numpy as np
import pytest

from oracle import fvh_oracle as O
from tests.fixtures import golden_files, load, oracle_config

RHS = golden_files("rhs")
STEPS = golden_files("steps")


def test_fixture_set_present():
    assert len(RHS) >= 30 and len(STEPS) >= 5


@pytest.mark.parametrize("path", RHS, ids=[os.path.basename(p) for p in RHS])
def test_rhs_matches_reference(path):
    c, d = load(path)
    dt, dudt, info = O.rhs(d["u0"], oracle_config(c))
    assert dt == float(d["dt"])
    assert np.array_equal(dudt, d["dudt"])
    if "trouble" in d:
        assert np.array_equal(np.asarray(info["trouble"], dtype=np.int8), d["trouble"])
        assert np.array_equal(info["nad_mag"], d["nad_mag"])
        assert np.array_equal(info["pad_mag"], d["pad_mag"])


@pytest.mark.parametrize("path", STEPS, ids=[os.path.basename(p) for p in STEPS])
def test_steps_match_reference(path):
    c, d = load(path)
    cfg = oracle_config(c)
    u = d["u0"].copy()
    t = 0.0
    T = float(d["T"]) if "T" in d else None
    flags = []
    for _ in range(int(d["steps"])):
        dt, u, infos = O.step(u, t, cfg, c["integrator"], target=T)
        t += dt
        flags.extend(np.asarray(i["trouble"], dtype=np.int8) for i in infos if "trouble" in i)
    assert np.array_equal(u, d["u_final"])
    assert t == d["timestamps"][-1]
    if "trouble_stages" in d:
        assert np.array_equal(np.stack(flags), d["trouble_stages"])
    if "trouble_counts" in d:
        assert [int(f.sum()) for f in flags] == list(d["trouble_counts"])


def test_stencil_rules_are_consistent():
    for p in range(9):
        for kind in "lcrt":
            w = O.stencil_weights(p, kind)
            assert len(w) == 2 * O.stencil_radius(p) + 1
            assert abs(w.sum() - 1.0) < 1e-15
        assert np.array_equal(O.stencil_weights(p, "r"), O.stencil_weights(p, "l")[::-1])
    assert np.array_equal(O.stencil_weights(1, "c"), [0.0, 1.0, 0.0])
    assert np.array_equal(O.stencil_weights(1, "t"), [0.0, 1.0, 0.0])
