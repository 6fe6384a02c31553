"""CPU oracle for the FVHOE per-stage update.

TEST INFRASTRUCTURE ONLY. This package is a plain-NumPy restatement of the
reference's algorithm (jpalafou/FVHOE, `fvhoe/`), used to check the CUDA path.
Only `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline leg
import it, and only as the checker; the product package `fvhoe_b200` never
imports, calls or falls back to anything here.

Parity of this oracle is pinned against golden vectors produced by the
reference itself (`tests/golden/make_golden.py`, run where the reference is
importable) and, in this container, against the live reference.
"""

from .fvh_oracle import *  # noqa: F401,F403
