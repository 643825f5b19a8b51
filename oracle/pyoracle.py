"""ctypes binding for the CPU oracle (oracle/_build/libglsm_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker.  The product (glsm_fluid_3d_b200)
never imports this module.

The oracle restates the coupled gel-fluid step of lasite/gLSM_fluid_3D
(src/sim.cpp:97-112 call order; kernels in src/fluid_kernels.cu,
src/gel_kernels.cu, src/coupling_kernels.cu) in FP64 (or FP32 "reference-like"
mode).  Field ids match glsm_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libglsm_oracle.so")

F_POP, F_RHO, F_U, F_C1, F_FIBM = 0, 1, 2, 3, 4
M_LAG, M_UL, M_VL, M_FDRAG, M_FREP, M_CL, M_DL, M_SL = 10, 11, 12, 13, 14, 15, 16, 17
G_RN, G_VELN, G_VELS, G_FN, G_UM, G_VM, G_WM = 20, 21, 22, 23, 24, 25, 26
G_UN_NORM, G_VN_NORM, G_T0, G_T1, G_T2, G_RM, G_NMSM = 27, 28, 29, 30, 31, 32, 33
G_VOLM, G_PREM, G_UN_ROBIN, G_UM_NORM, G_VM_NORM, G_WMP, G_FN_ROBIN = 34, 35, 36, 37, 38, 39, 40

_lib = None


def build() -> str:
    """Compile the oracle with the committed Makefile (g++/OpenMP, no GPU)."""
    subprocess.check_call(["make", "-s", "-f", os.path.join(HERE, "Makefile"), LIB_PATH])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i, i, i, i, i]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_params.argtypes = [vp, d, d, d, d, d, i, i, i]
        L.orc_add_gel.argtypes = [vp, i, i, i, d, d, d, i, i]
        L.orc_gel_noise.argtypes = [vp, i, ctypes.c_ulonglong, d]
        L.orc_gel_control.argtypes = [vp, i, i, d]
        L.orc_finalize.argtypes = [vp]
        L.orc_info.argtypes = [vp, ctypes.POINTER(ll)]
        L.orc_gel_info.argtypes = [vp, i, ctypes.POINTER(ll)]
        L.orc_gel_steady.argtypes = [vp, i, ctypes.POINTER(d)]
        L.orc_units.argtypes = [vp, ctypes.POINTER(d)]
        L.orc_run.argtypes = [vp, i, i]
        L.orc_phase.argtypes = [vp, i, i]
        L.orc_field.restype = ll
        L.orc_field.argtypes = [vp, i, i, ctypes.POINTER(d), ll, i]
        L.orc_threads.argtypes = [i]
        L.orc_threads.restype = i
        L.orc_noise.restype = d
        L.orc_noise.argtypes = [ctypes.c_ulonglong] * 4
        _lib = L
    return _lib


def threads(n: int = 0) -> int:
    return lib().orc_threads(n)


class Oracle:
    """One coupled system (fluid lattice + gels) on the CPU."""

    def __init__(self, nx, ny, nz, nsub=25, fp32=False):
        self.L = lib()
        self.h = self.L.orc_create(nx, ny, nz, nsub, 1 if fp32 else 0)
        if not self.h:
            raise ValueError("invalid oracle dims")
        self.dims = (nx, ny, nz)
        self.nsub = nsub
        self.n_gels = 0

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, beta=1.0, ramp_steps=20000.0, force=(0.0, 0.0, 0.0), periodic=(0, 0, 0)):
        self.L.orc_set_params(self.h, beta, ramp_steps, *force, *periodic)

    def add_gel(self, size, pos, gel_type=1, gel_id=None):
        gid = self.n_gels + 1 if gel_id is None else gel_id
        r = self.L.orc_add_gel(self.h, *size, *pos, gel_type, gid)
        if r < 0:
            raise RuntimeError("add_gel failed")
        self.n_gels += 1
        return r

    def gel_noise(self, gel, seed, amp):
        assert self.L.orc_gel_noise(self.h, gel, seed, amp) == 0

    def reset_quiescent(self, gel):
        assert self.L.orc_gel_control(self.h, gel, 0, 0.0) == 0

    def fire_pulse(self, gel):
        assert self.L.orc_gel_control(self.h, gel, 1, 0.0) == 0

    def set_anchor(self, gel, z):
        assert self.L.orc_gel_control(self.h, gel, 2, z) == 0

    def set_active_from(self, gel, it):
        assert self.L.orc_gel_control(self.h, gel, 3, float(it)) == 0

    def build_tube_mask(self, gel, wall_thickness, circular=False):
        assert self.L.orc_gel_control(self.h, gel, 5 if circular else 4, float(wall_thickness)) == 0

    def finalize(self):
        assert self.L.orc_finalize(self.h) == 0

    def info(self):
        out = (ctypes.c_longlong * 4)()
        self.L.orc_info(self.h, out)
        return dict(N=out[0], M=out[1], n_gels=out[2], nsub=out[3])

    def gel_info(self, g):
        out = (ctypes.c_longlong * 7)()
        assert self.L.orc_gel_info(self.h, g, out) == 0
        return dict(LX=out[0], LY=out[1], LZ=out[2], nE=out[3], nN=out[4], M=out[5], offset=out[6])

    def steady(self, g):
        out = (ctypes.c_double * 3)()
        self.L.orc_gel_steady(self.h, g, out)
        return tuple(out)

    def units(self):
        out = (ctypes.c_double * 2)()
        self.L.orc_units(self.h, out)
        return tuple(out)

    def run(self, iter0, n):
        assert self.L.orc_run(self.h, iter0, n) == 0

    def phase(self, phase, it=0):
        assert self.L.orc_phase(self.h, phase, it) == 0

    def get(self, field, gel=0):
        n = self.L.orc_field(self.h, field, gel, None, 0, 0)
        if n < 0:
            raise KeyError(field)
        buf = np.empty(n, dtype=np.float64)
        r = self.L.orc_field(self.h, field, gel, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n, 0)
        assert r == n
        return buf

    def set(self, field, values, gel=0):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        r = self.L.orc_field(self.h, field, gel, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), v.size, 1)
        if r < 0:
            raise KeyError(field)


def noise(seed, gel_id, slot, field):
    return lib().orc_noise(seed, gel_id, slot, field)


def iso_crossing(A, B, C, D, E, F, G, H, viso=0.15, eps=1e-12):
    """solveBilinear (src/gel_kernels.cu:165-212): the point (x, y) of the unit
    square where the bilinear interpolants of u (corners A B / C D) and v
    (E F / G H) both equal viso, or None."""
    import math

    a00, a10, a01, a11 = A - viso, B - A, C - A, A - B + D - C
    b00, b10, b01, b11 = E - viso, F - E, G - E, E - F + H - G
    c2 = b10 * a11 - b11 * a10
    c1 = b00 * a11 + b10 * a01 - b01 * a10 - b11 * a00
    c0 = b00 * a01 - b01 * a00
    if abs(c2) < eps:
        if abs(c1) < eps:
            return None
        roots = [-c0 / c1]
    else:
        disc = c1 * c1 - 4.0 * c2 * c0
        if disc < 0.0:
            return None
        s = math.sqrt(disc)
        roots = [(-c1 + s) / (2.0 * c2), (-c1 - s) / (2.0 * c2)]
    for x in roots:
        if x < -eps or x > 1.0 + eps:
            continue
        den = a01 + a11 * x
        if abs(den) < eps:
            continue
        y = -(a00 + a10 * x) / den
        if y < -eps or y > 1.0 + eps:
            continue
        return min(max(x, 0.0), 1.0), min(max(y, 0.0), 1.0)
    return None


def filament(un_norm, vn_norm, LX, LY, LZ, viso=0.15):
    """calFilamentD (src/gel_kernels.cu:837-866): for every node face (xi, yi, zi),
    xi in [1, LX-1], yi in [1, LY-1], zi in [1, LZ-1], the crossing of the
    u_norm = viso and v_norm = viso contours as (xi + xb, yi + yb, zi); faces in
    x-fastest order.  Nodal fields over (LX+2)(LY+2)(LZ+2) slots."""
    sx, sxy = LX + 2, (LX + 2) * (LY + 2)
    out = []
    for zi in range(1, LZ):
        for yi in range(1, LY):
            for xi in range(1, LX):
                n00 = xi + yi * sx + zi * sxy
                n10, n01, n11 = n00 + 1, n00 + sx, n00 + sx + 1
                r = iso_crossing(un_norm[n00], un_norm[n10], un_norm[n01], un_norm[n11],
                                 vn_norm[n00], vn_norm[n10], vn_norm[n01], vn_norm[n11], viso)
                if r is not None:
                    out.append((xi + r[0], yi + r[1], float(zi)))
    return np.array(out, dtype=np.float64).reshape(-1, 3)


# D3Q19 velocities in the reference's direction order (src/fluid.cu:202-215)
D3Q19_C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                    [1, 1, 0], [-1, 1, 0], [-1, -1, 0], [1, -1, 0], [1, 0, 1], [-1, 0, 1], [-1, 0, -1],
                    [1, 0, -1], [0, 1, 1], [0, 1, -1], [0, -1, -1], [0, -1, 1]])


def conserve_round_f16(v):
    """float32 restatement of the library's conserving FP16 rounding (FP16
    storage option; the reference stores FP32, so this has no reference
    counterpart).  v: (n, 19) float32 scaled post-collision values of n cells.
    Every value is rounded to nearest FP16; then for q = 1..18 in order a value
    moves one FP16 spacing towards its exact value when that lowers M^2 + |P|^2
    (the cell's summed mass and momentum rounding errors so far): when the
    projection t = M + c_q . P has the sign of the value's rounding error and
    |t| exceeds one spacing (a face direction) or 1.5 (a diagonal).  Returns the
    float32 values of the chosen FP16 numbers.  All arithmetic is float32 with
    one rounding per operation, in the kernel's order."""
    f32 = np.float32
    v = np.asarray(v, dtype=f32)
    h = v.astype(np.float16).astype(f32)
    e = (v - h).astype(f32)
    n = v.shape[0]
    M = np.zeros(n, f32)
    P = np.zeros((3, n), f32)
    for q in range(19):
        M = (M + e[:, q]).astype(f32)
        for a in range(3):
            c = D3Q19_C[q, a]
            if c:
                P[a] = (P[a] + e[:, q] if c > 0 else P[a] - e[:, q]).astype(f32)
    for q in range(1, 19):
        c = D3Q19_C[q]
        bits = h[:, q].view(np.int32) & np.int32(0x7F800000)
        ulp = np.maximum((bits - np.int32(10 << 23)).view(f32), f32(2.0 ** -24))
        de = np.copysign(ulp, -e[:, q]).astype(f32)
        t = M.copy()
        for a in range(3):
            if c[a]:
                t = (t + P[a] if c[a] > 0 else t - P[a]).astype(f32)
        # M^2 + |P|^2 falls exactly when t has the sign of e and |t| exceeds
        # (1 + |c|^2) / 2 spacings
        thr = (f32(1.5) * ulp).astype(f32) if int((c * c).sum()) == 2 else ulp
        same_sign = (t.view(np.int32) ^ e[:, q].view(np.int32)) >= 0
        move = (np.abs(t) > thr) & same_sign
        h[:, q] = np.where(move, (h[:, q] - de).astype(f32), h[:, q])
        M = np.where(move, (M + de).astype(f32), M)
        for a in range(3):
            if c[a]:
                P[a] = np.where(move, (P[a] + de if c[a] > 0 else P[a] - de).astype(f32), P[a])
    return h
