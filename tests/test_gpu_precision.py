"""FP16 / BF16 population storage (deviations f_q - w_q, FP32 collision and
moments) against the FP64 oracle on the golden cases.

FP16 stores the deviations scaled by 2^20 (its normal range then covers
deviations from 6e-11 to 0.06 with 11-bit precision), rounded to nearest or
("f16c") with the mass- and momentum-conserving rounding; BF16 stores them
unscaled with 8-bit precision.  The tolerances below are relative L2 errors.
"""
import numpy as np
import pytest

from cases import CASES, build, collect
from oracle.pyoracle import Oracle
from parity import rel_l2

pytestmark = pytest.mark.gpu

TOL = {
    "f16": {"u": 2e-3, "Ul": 2e-3, "pop": 1e-5, "c1": 1e-4, "rn": 1e-7, "um": 1e-7},
    "bf16": {"u": 3e-2, "Ul": 3e-2, "pop": 1e-4, "c1": 1e-3, "rn": 1e-6, "um": 1e-6},
}
TOL["f16c"] = TOL["f16c2"] = TOL["f16"]  # FP16 storage with the conserving rounding


@pytest.mark.parametrize("storage", ["f16", "f16c", "f16c2", "bf16"])
@pytest.mark.parametrize("case", list(CASES))
def test_low_precision_storage_vs_oracle(gpu, storage, case):
    from glsm_fluid_3d_b200 import System

    sim = build(System, case, storage=storage)
    sim.run(0, CASES[case]["iters"])
    got = collect(sim, case)
    sim.close()
    ref = build(Oracle, case)
    ref.run(0, CASES[case]["iters"])
    want = collect(ref, case)
    ref.close()
    bad = []
    for name, tol in TOL[storage].items():
        keys = [k for k in want if k == name or k.endswith("_" + name)]
        for k in keys:
            e = rel_l2(got[k], want[k])
            print(f"{storage} {case} {k} rel_l2={e:.2e}")
            if not e <= tol:
                bad.append((k, e, tol))
    assert not bad, bad
