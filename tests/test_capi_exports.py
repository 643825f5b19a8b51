"""The C-ABI library loads without a GPU and exports every entry point that
include/glsm_b200.h declares (no compute calls are made here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(glsm_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared("glsm_b200.h")
    for must in ("glsm_gel_create", "glsm_coupler_create", "glsm_fluid_create", "glsm_fluid_run",
                 "glsm_fluid_step_velocity", "glsm_fluid_step_concentration", "glsm_gel_step_elasticity",
                 "glsm_gel_step_chemistry", "glsm_coupler_pack", "glsm_coupler_scatter",
                 "glsm_coupler_repulsion"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from glsm_fluid_3d_b200 import build

    lib = ctypes.CDLL(build.build())
    missing = [n for n in declared("glsm_b200.h") if not hasattr(lib, n)]
    assert not missing, missing


def test_argument_errors_without_gpu():
    """Argument checks run before any CUDA call and report through glsm_last_error."""
    from glsm_fluid_3d_b200 import lib

    L = lib()
    h = ctypes.c_void_p()
    assert L.glsm_gel_create(0, 6, 6, 0.0, 0.0, 0.0, 1, 1, ctypes.byref(h)) == -1
    assert b"gel size" in L.glsm_last_error()
    assert L.glsm_gel_create(6, 6, 6, 0.0, 0.0, 0.0, 3, 1, ctypes.byref(h)) == -1
    assert L.glsm_fluid_run(None, 0, 1) == -1


def test_fluid_desc_defaults_match_reference_constants():
    """tau, h, beta, ramp and the derived Nsub = llround(dt/dt_fluid) = 25 (src/fluid.cu:167-201)."""
    from glsm_fluid_3d_b200 import FluidDesc, lib

    d = FluidDesc()
    env = {k: os.environ.pop(k) for k in ("IBM_BETA", "IBM_RAMP_STEPS") if k in os.environ}
    try:
        assert lib().glsm_fluid_desc_default(ctypes.byref(d), 101, 101, 101) == 0
    finally:
        os.environ.update(env)
    assert d.nsub == 25
    assert abs(d.tau - 0.8) < 1e-7 and abs(d.h - 0.5) < 1e-7
    assert d.beta == 1.0 and d.ramp_steps == 20000.0
    assert d.storage == 0


def test_copy_bandwidth_rejects_bad_sizes():
    """Arguments are checked before any CUDA call, so this runs without a GPU."""
    import ctypes

    from glsm_fluid_3d_b200 import lib

    L = lib()
    out = ctypes.c_double(0.0)
    for nbytes, reps in ((0, 1), (17, 1), (1 << 20, 0), (1 << 20, 100001), ((8 << 30) + 16, 1)):
        assert L.glsm_copy_bandwidth(nbytes, reps, ctypes.byref(out)) == -1, (nbytes, reps)
    assert b"multiple of 16" in L.glsm_copy_bandwidth_error()
