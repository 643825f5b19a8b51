"""The conserving FP16 rounding (storage "f16c" on every substep, "f16c2" on
odd substeps; glsm_fluid_set_f16_rounding).

* the device rounding reproduces its float32 restatement in the oracle module
  bit for bit, on values of every magnitude FP16 storage meets;
* over a long run its velocity error against the FP32 solver stays well below
  that of round-to-nearest, which accumulates long-wavelength noise.
"""
import ctypes

import numpy as np
import pytest

from oracle.pyoracle import conserve_round_f16
from parity import rel_l2

pytestmark = pytest.mark.gpu


def device_round(v):
    from glsm_fluid_3d_b200 import lib

    L = lib()
    v = np.ascontiguousarray(v, dtype=np.float32)
    out = np.empty_like(v)
    rc = L.glsm_f16_conserve_round(v.ctypes.data, out.ctypes.data, v.shape[0])
    assert rc == 0, L.glsm_last_error()
    return out


def test_conserving_rounding_matches_restatement(gpu):
    rng = np.random.default_rng(7)
    n = 200_000
    mag = 10.0 ** rng.uniform(-9, 4, size=(n, 1))  # scaled deviations: subnormal FP16 to 1e4
    v = (rng.standard_normal((n, 19)) * mag).astype(np.float32)
    v[:1000] = 0.0                                  # exact zeros
    v[1000:2000] = np.float32(2.0) ** rng.integers(-20, 12, size=(1000, 19)).astype(np.float32)  # powers of two
    v[2000:3000] *= np.float32(1 + 2.0 ** -12)       # just off FP16 numbers
    got = device_round(v)
    want = conserve_round_f16(v)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    # every output is an FP16 number within 1.5 spacings of its input
    assert np.array_equal(got.astype(np.float16).astype(np.float32), got)


def _run(storage, iters):
    from glsm_fluid_3d_b200 import System

    # deterministic spreads: the comparison repeats bit for bit
    s = System(32, 32, 32, nsub=25, storage=storage, deterministic=True)
    s.add_gel((4, 4, 4), (7.75, 7.75, 7.75), 1, 1)
    s.gel_noise(0, 5, 1e-3)
    s.set_params(beta=1.0, ramp_steps=0.0)
    s.finalize()
    s.run(0, iters)
    u = s.fluid.read("u")
    s.close()
    return u


def test_conserving_rounding_keeps_long_run_error_low(gpu):
    iters = 2000  # 50,000 substeps
    ref = _run("f32", iters)
    e_near = rel_l2(_run("f16", iters), ref)
    e_cons = rel_l2(_run("f16c", iters), ref)
    e_odd = rel_l2(_run("f16c2", iters), ref)
    print(f"u rel L2 vs FP32 after {iters} iterations: nearest {e_near:.3e}, conserving {e_cons:.3e}, "
          f"conserving on odd substeps {e_odd:.3e}")
    assert e_cons < 0.3 * e_near, (e_cons, e_near)
    assert e_odd < e_near, (e_odd, e_near)
