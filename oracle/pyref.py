"""ctypes binding for the reference's own CUDA build (oracle/_ref/libglsm_ref.so).

TEST INFRASTRUCTURE ONLY: the checker for parity against the reference kernels
(lasite/gLSM_fluid_3D src/*.cu compiled unmodified for sm_100a through
oracle/ref_harness.cu) and the timed reference arm of bench.py.  Same method
names and field ids as pyoracle.Oracle.  Needs a GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libglsm_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: build it with `make -f oracle/Makefile ref`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        L.ref_create.restype = vp
        L.ref_create.argtypes = [i, i, i, i]
        L.ref_add_gel.argtypes = [vp, i, i, i, d, d, d, i, i]
        L.ref_gel_noise.argtypes = [vp, i, ctypes.c_ulonglong, d]
        L.ref_gel_control.argtypes = [vp, i, i, d]
        L.ref_set_beta.argtypes = [vp, d]
        L.ref_finalize.argtypes = [vp]
        L.ref_run.argtypes = [vp, i, i]
        L.ref_time.restype = d
        L.ref_time.argtypes = [vp, i, i]
        L.ref_info.argtypes = [vp, ctypes.POINTER(ll)]
        L.ref_field.restype = ll
        L.ref_field.argtypes = [vp, i, i, ctypes.POINTER(d), ll]
        L.ref_destroy.argtypes = [vp]
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_record_center.argtypes = [vp, i]
        L.ref_write_files.argtypes = [vp, i]
        L.ref_set_start_time.argtypes = [vp, i]
        _lib = L
    return _lib


class Reference:
    """One coupled system run by the reference's CUDA code on cuda:0."""

    def __init__(self, nx, ny, nz, nsub=25):
        self.L = lib()
        self.h = self.L.ref_create(nx, ny, nz, nsub)
        if not self.h:
            raise RuntimeError("ref_create failed (no GPU?)")
        self.n_gels = 0

    def _chk(self, r, what):
        if r != 0:
            raise RuntimeError(f"{what}: {self.L.ref_last_error().decode()}")

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def set_start_time(self, t):
        """Gels added afterwards and the fluid restart from the .dat files of
        time t in the current directory (the reference's setGoonValue)."""
        self._chk(self.L.ref_set_start_time(self.h, int(t)), "start time")

    def set_params(self, beta=1.0, ramp_steps=20000.0):
        # Fluid::stepVelocity reads IBM_RAMP_STEPS on every call (src/fluid.cu:265-268)
        os.environ["IBM_RAMP_STEPS"] = repr(float(ramp_steps))
        self.L.ref_set_beta(self.h, beta)

    def add_gel(self, size, pos, gel_type=1, gel_id=None):
        gid = self.n_gels + 1 if gel_id is None else gel_id
        r = self.L.ref_add_gel(self.h, *size, *pos, gel_type, gid)
        if r < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        self.n_gels += 1
        return r

    def gel_noise(self, gel, seed, amp):
        self._chk(self.L.ref_gel_noise(self.h, gel, seed, amp), "noise")

    def reset_quiescent(self, gel):
        self._chk(self.L.ref_gel_control(self.h, gel, 0, 0.0), "reset")

    def fire_pulse(self, gel):
        self._chk(self.L.ref_gel_control(self.h, gel, 1, 0.0), "pulse")

    def set_anchor(self, gel, z):
        self._chk(self.L.ref_gel_control(self.h, gel, 2, z), "anchor")

    def set_active_from(self, gel, it):
        self._chk(self.L.ref_gel_control(self.h, gel, 3, float(it)), "active")

    def build_tube_mask(self, gel, wall_thickness, circular=False):
        self._chk(self.L.ref_gel_control(self.h, gel, 5 if circular else 4, float(wall_thickness)), "tube")

    def record_center(self, iter):
        """Gel::recordCenter(iter) of every gel (src/gel.cu:706-712)."""
        self._chk(self.L.ref_record_center(self.h, iter), "recordCenter")

    def write_files(self, iter):
        """Gel::writeFiles(iter) of every gel and Fluid::writeFiles(iter)
        (src/gel.cu:543-553, src/fluid.cu:140-150) into the current directory;
        the writer threads are joined before this returns."""
        self._chk(self.L.ref_write_files(self.h, iter), "writeFiles")

    def finalize(self):
        self._chk(self.L.ref_finalize(self.h), "finalize")

    def run(self, iter0, n):
        self._chk(self.L.ref_run(self.h, iter0, n), "run")

    def time(self, iter0, n) -> float:
        ms = self.L.ref_time(self.h, iter0, n)
        if ms < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return ms

    def info(self):
        out = (ctypes.c_longlong * 4)()
        self.L.ref_info(self.h, out)
        return dict(N=out[0], M=out[1], n_gels=out[2], nsub=out[3])

    def get(self, field, gel=0):
        n = self.L.ref_field(self.h, field, gel, None, 0)
        if n < 0:
            raise KeyError(field)
        buf = np.empty(n, dtype=np.float64)
        r = self.L.ref_field(self.h, field, gel, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        if r != n:
            raise RuntimeError(self.L.ref_last_error().decode())
        return buf
