"""The CPU oracle against the reference's own CUDA kernels (golden fixtures).

The fixtures were produced by tests/golden/make_golden.py, which runs the
reference's src/*.cu compiled unmodified for sm_100a on a B200.  The reference
stores populations in FP32 and spreads with float atomics; the oracle is FP64
and deterministic, so the comparison is a tolerance check whose bounds come
from the reference's own FP32 round-off (the FP32 mode of the oracle shows the
same size of difference).
"""
import os

import numpy as np
import pytest

from cases import CASES, build, collect
from oracle.pyoracle import Oracle
from parity import rel_l2

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# relative L2 bounds, oracle (FP64) vs reference (FP32 fluid, FP64 gel)
TOL = {
    "u": 2e-3, "Ul": 1e-3, "Fdrag": 1e-4, "pop": 1e-5, "rho": 1e-5, "c1": 1e-5,
    "Dl": 1e-5, "Sl": 1e-4, "Cl": 1e-4, "Frep": 1e-4, "lag": 1e-7, "Vl": 1e-6,
    "un_robin": 1e-4,  # = -Sl, an FP32 quantity of the fluid side
}
GEL_TOL = 1e-6  # gel fields are FP64 on both sides; T1 is round-off sized and checked absolutely


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("fp32", [False, True])
def test_oracle_matches_reference_fixture(case, fp32):
    path = os.path.join(HERE, f"{case}.npz")
    gold = np.load(path)
    sim = build(Oracle, case, fp32=fp32)
    sim.run(0, CASES[case]["iters"])
    got = collect(sim, case)
    sim.close()
    bad = []
    for k in gold.files:
        if k.endswith("_T1"):
            continue
        name = k.split("_", 1)[1] if k.startswith("g") and "_" in k else k
        tol = TOL.get(name, GEL_TOL if k.startswith("g") else 1e-4)
        err = rel_l2(got[k], gold[k])
        if not err <= tol:
            bad.append((k, err, tol))
    assert not bad, bad


def test_fixture_shapes():
    for case, c in CASES.items():
        g = np.load(os.path.join(HERE, f"{case}.npz"))
        n = int(np.prod(c["dims"]))
        assert g["u"].size == 3 * n and g["c1"].size == n
        assert g["g0_um"].size > 0
