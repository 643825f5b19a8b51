"""The bounded device waits end with an error status, not a hang.

A force-region tile of the substep kernel waits for the IBM tasks of its
substep (wait_ibm in csrc/lbm.cu) with an iteration limit.  The test aid
glsm_test_ibm_wait_extra makes every tile wait for IBM tasks that never run, so
each wait runs out: the launch completes, the next glsm_fluid_sync reports
GLSM_ERR_DEVICE with "IBM wait timed out", and the same process then runs a
normal system correctly (the context stays usable).  No fault, trap or endless
loop is involved: the wait gives up after a fraction of a second.
"""
import time

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from parity import rel_l2

pytestmark = pytest.mark.gpu


def _make(cls):
    s = cls(24, 24, 24, nsub=2)
    s.add_gel((6, 6, 6), (5.75, 5.75, 5.75), 1, 1)
    s.gel_noise(0, 12345, 1e-3)
    s.set_params(beta=1.0, ramp_steps=0.0)
    s.finalize()
    return s


def test_ibm_wait_runs_out_and_is_reported(gpu):
    from glsm_fluid_3d_b200 import GlsmError, System

    s = _make(System)
    s.fluid.run(0, 1)
    s.fluid.sync()  # a normal iteration reports nothing
    s.fluid.test_ibm_wait_extra(1)
    t0 = time.perf_counter()
    s.fluid.run(1, 1)
    with pytest.raises(GlsmError, match="IBM wait timed out"):
        s.fluid.sync()
    elapsed = time.perf_counter() - t0
    print(f"iteration with the wait running out: {elapsed:.2f} s")
    assert elapsed < 30.0
    # the flag was read and cleared: a normal iteration reports nothing again
    s.fluid.test_ibm_wait_extra(0)
    s.fluid.run(2, 1)
    s.fluid.sync()
    s.close()

    # the same process then runs a fresh system correctly
    gpu_sys, cpu = _make(System), _make(Oracle)
    gpu_sys.run(0, 10)
    cpu.run(0, 10)
    for fid, name, tol in ((2, "u", 1e-4), (0, "pop", 1e-6), (20, "rn", 1e-9)):
        e = rel_l2(gpu_sys.get(fid), cpu.get(fid))
        assert e < tol, (name, e)
    assert np.isfinite(gpu_sys.get(2)).all()
    gpu_sys.close()
    cpu.close()
