"""glsm_fluid_3d_b200 -- the coupled gel-fluid step of lasite/gLSM_fluid_3D on B200.

Python face of libglsm_b200.so (C ABI in include/glsm_b200.h).  The classes
keep the reference's names and methods (src/gel.h Gel, src/coupling.h Coupler,
src/fluid.h Fluid), so a driver written against the reference reads the same:

    g1 = Gel((6, 6, 6), (16.67, 25.0, 25.0), 1, 1)
    g2 = Gel((6, 6, 6), (33.33, 25.0, 25.0), 1, 2)
    coupler = Coupler([g1, g2])
    fluid = Fluid((101, 101, 101), coupler)            # dims in lattice cells
    for it in range(n):                                 # src/sim.cpp:97-112
        for g in (g1, g2):
            g.stepElasticity(it); g.stepChemistry(it)
        coupler.packFromGels()
        fluid.stepVelocity(it); fluid.stepConcentration(it)
        coupler.applyGelRepulsion(); coupler.scatterToGels()

or, the same iterations fused and graph-captured: ``fluid.run(0, n)``.
All compute runs in hand-written sm_100a kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import FluidDesc, GlsmError, check, lib

__all__ = ["Gel", "Coupler", "Fluid", "System", "Batch", "GlsmError", "STORAGE", "lib", "copy_bandwidth",
           "pattern_bandwidth", "l2_reset_persisting", "l2_persisting_setaside"]

STORAGE = {"f32": 0, "fp32": 0, "f16": 1, "fp16": 1, "bf16": 2, "f16c": 1, "f16c2": 1}
# FP16 rounding modes (glsm_fluid_set_f16_rounding); storage "f16c" is FP16
# storage with the conserving rounding on every substep, "f16c2" on every
# second (odd) substep
F16_ROUNDING = {"nearest": 0, "conserving": 1, "conserving_odd": 2}
_STORAGE_ROUNDING = {"f16c": "conserving", "f16c2": "conserving_odd"}

GEL_FIELDS = {
    "rn": 0, "Veln": 1, "Vels": 2, "Fn": 3, "um": 4, "vm": 5, "wm": 6, "un_norm": 7, "vn_norm": 8,
    "T0": 9, "T1": 10, "T2": 11, "rm": 12, "nmSm": 13, "Volm": 14, "Prem": 15, "un_robin": 16,
    "um_norm": 17, "vm_norm": 18, "wmp": 19, "Fn_robin": 20, "rm_loc": 21,
}
FLUID_FIELDS = {"pop": 0, "rho": 1, "u": 2, "c1": 3}
MARKER_FIELDS = {"lag": 0, "Ul": 1, "Vl": 2, "Fdrag": 3, "Frep": 4, "Cl": 5, "Dl": 6, "Sl": 7}


def l2_reset_persisting():
    """Turn every persisting L2 line back into a normal one (glsm_l2_reset_persisting);
    call with the GPU idle, before flushing L2 between timed steps."""
    check(lib().glsm_l2_reset_persisting(), "l2_reset_persisting")


def l2_persisting_setaside() -> int:
    """The context's persisting L2 set-aside in bytes (glsm_l2_persisting_setaside)."""
    out = ctypes.c_size_t(0)
    check(lib().glsm_l2_persisting_setaside(ctypes.byref(out)), "l2_persisting_setaside")
    return out.value


def copy_bandwidth(nbytes: int, reps: int) -> float:
    """Measured copy bandwidth in GB/s (read + write bytes): a buffer of nbytes
    copied back and forth reps times in one launch through L2 only.  With
    2 x nbytes well below the 126 MB L2 this is the L2 copy bandwidth, well
    above it the HBM copy bandwidth (glsm_copy_bandwidth)."""
    L = lib()
    out = ctypes.c_double(0.0)
    rc = L.glsm_copy_bandwidth(int(nbytes), int(reps), ctypes.byref(out))
    if rc != 0:
        raise GlsmError(f"copy_bandwidth: {L.glsm_copy_bandwidth_error().decode()}")
    return out.value


def pattern_bandwidth(dims, storage="f32", reps: int = 20):
    """(even, odd) GB/s of the substep kernel's access pattern without the
    collision on a lattice of `dims` in the kernel's layout and element size:
    every cell reads its 19 populations and writes them back, in the even AA
    form (own slots) and the odd form (neighbours' slots) (glsm_pattern_bandwidth)."""
    L = lib()
    ge, go = ctypes.c_double(0.0), ctypes.c_double(0.0)
    st = STORAGE[storage] if isinstance(storage, str) else int(storage)
    rc = L.glsm_pattern_bandwidth(int(dims[0]), int(dims[1]), int(dims[2]), st, int(reps), ctypes.byref(ge),
                                  ctypes.byref(go))
    if rc != 0:
        raise GlsmError(f"pattern_bandwidth: {L.glsm_copy_bandwidth_error().decode()}")
    return ge.value, go.value


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Gel:
    """Gel(gelSize, gelPosition, gelType, gel_id) -- src/gel.h:35, src/gel.cu:555-663."""

    def __init__(self, size, position, gel_type=1, gel_id=1):
        self.L = lib()
        h = ctypes.c_void_p()
        check(self.L.glsm_gel_create(int(size[0]), int(size[1]), int(size[2]), float(position[0]),
                                     float(position[1]), float(position[2]), int(gel_type), int(gel_id),
                                     ctypes.byref(h)), "Gel")
        self.h = h
        info = (ctypes.c_int64 * 8)()
        check(self.L.glsm_gel_info(self.h, info), "Gel info")
        self.LX, self.LY, self.LZ, self.nE, self.nN, self.M, self.gel_id, self.gel_type = (int(v) for v in info)
        self.coupler = None

    # reference-named members -------------------------------------------------
    @property
    def m_numGelNodes(self):
        return self.nN

    @property
    def m_numGelElements(self):
        return self.nE

    @property
    def m_boundaryCount(self):
        return self.M

    def stepElasticity(self, it):
        check(self.L.glsm_gel_step_elasticity(self.h, int(it)), "stepElasticity")

    def stepChemistry(self, it):
        check(self.L.glsm_gel_step_chemistry(self.h, int(it)), "stepChemistry")

    def recordCenter(self, it):
        check(self.L.glsm_gel_record_center(self.h, int(it)), "recordCenter")

    def resetToQuiescent(self):
        check(self.L.glsm_gel_reset_quiescent(self.h), "resetToQuiescent")

    def fireExcitationPulse(self):
        check(self.L.glsm_gel_fire_pulse(self.h), "fireExcitationPulse")

    def setAnchorZ(self, z):
        check(self.L.glsm_gel_set_anchor_z(self.h, float(z)), "setAnchorZ")

    def buildTubeMask(self, wall_thickness, circular=False):
        check(self.L.glsm_gel_build_tube_mask(self.h, int(wall_thickness), 1 if circular else 0), "buildTubeMask")

    # extensions ---------------------------------------------------------------
    def set_active_from(self, it):
        check(self.L.glsm_gel_set_active_from(self.h, int(it)), "set_active_from")

    def set_bz_f(self, f):
        """GelParams::f; recomputes the steady state and restarts the chemistry from it."""
        check(self.L.glsm_gel_set_bz_f(self.h, float(f)), "set_bz_f")

    def add_noise(self, seed, amplitude):
        check(self.L.glsm_gel_add_noise(self.h, int(seed), float(amplitude)), "add_noise")

    def steady_state(self):
        out = (ctypes.c_double * 3)()
        check(self.L.glsm_gel_steady_state(self.h, out), "steady_state")
        return tuple(out)

    def filament(self, max_points=None):
        """calFilamentD: the u_norm = v_norm = 0.15 crossing points, (n, 3) array
        in node units (glsm_gel_filament)."""
        n = ctypes.c_size_t()
        check(self.L.glsm_gel_filament(self.h, None, 0, ctypes.byref(n)), "filament")
        cap = n.value if max_points is None else min(n.value, int(max_points))
        out = np.zeros(3 * max(cap, 1), dtype=np.float64)
        check(self.L.glsm_gel_filament(self.h, _dptr(out), cap, ctypes.byref(n)), "filament")
        return out[:3 * cap].reshape(-1, 3)

    def series_config(self, every, capacity):
        check(self.L.glsm_gel_series_config(self.h, int(every), int(capacity)), "series_config")
        self._series_cap = int(capacity)

    def series(self):
        cap = getattr(self, "_series_cap", 1000)
        buf = np.zeros(12 * cap)
        check(self.L.glsm_gel_series_read(self.h, _dptr(buf), buf.size), "series")
        return buf.reshape(cap, 12)

    def read(self, field):
        fid = GEL_FIELDS[field] if isinstance(field, str) else int(field)
        n = self.L.glsm_gel_field_size(self.h, fid)
        if n == 0:
            raise KeyError(field)
        buf = np.empty(n, dtype=np.float64)
        check(self.L.glsm_gel_read(self.h, fid, _dptr(buf), n), f"read {field}")
        return buf

    def read_into(self, field, buf):
        """Read a field into a caller-owned float64 array (e.g. pinned host memory)."""
        fid = GEL_FIELDS[field] if isinstance(field, str) else int(field)
        check(self.L.glsm_gel_read(self.h, fid, _dptr(buf), buf.size), f"read {field}")

    def snapshot(self, fields, bufs):
        """Output snapshot (glsm_gel_snapshot): the fields as they are behind the
        queued work go to the float64 buffers (page-locked, one per field, left
        untouched until snapshot_wait) on a copy stream; returns at once."""
        ids = (ctypes.c_int * len(fields))(*[GEL_FIELDS[f] if isinstance(f, str) else int(f) for f in fields])
        for f, b in zip(fields, bufs):
            fid = GEL_FIELDS[f] if isinstance(f, str) else int(f)
            if b.dtype != np.float64 or not b.flags.c_contiguous or b.size != self.L.glsm_gel_field_size(self.h, fid):
                raise ValueError(f"snapshot buffer for {f}: contiguous float64 of the field's size")
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(bufs))(*[_dptr(b) for b in bufs])
        check(self.L.glsm_gel_snapshot(self.h, len(fields), ids, ptrs), "snapshot")

    def snapshot_wait(self):
        check(self.L.glsm_gel_snapshot_wait(self.h), "snapshot_wait")

    def write(self, field, values):
        fid = GEL_FIELDS[field] if isinstance(field, str) else int(field)
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(self.L.glsm_gel_write(self.h, fid, _dptr(v), v.size), f"write {field}")

    def device_ptr(self, field):
        fid = GEL_FIELDS[field] if isinstance(field, str) else int(field)
        return self.L.glsm_gel_device_ptr(self.h, fid)

    def close(self):
        if getattr(self, "h", None):
            check(self.L.glsm_gel_destroy(self.h), "Gel destroy")
            self.h = None


class Coupler:
    """Coupler(gels) -- src/coupling.h:16, src/coupling.cu:50-80."""

    def __init__(self, gels):
        self.L = lib()
        self.gels = list(gels)
        arr = (ctypes.c_void_p * max(1, len(self.gels)))(*[g.h for g in self.gels])
        h = ctypes.c_void_p()
        check(self.L.glsm_coupler_create(arr, len(self.gels), ctypes.byref(h)), "Coupler")
        self.h = h
        self.M = self.L.glsm_coupler_markers(self.h)
        for g in self.gels:
            g.coupler = self
        self.fluid = None

    @property
    def sumGelBoundaryCount(self):
        return self.M

    def packFromGels(self):
        check(self.L.glsm_coupler_pack(self.h), "packFromGels")

    def scatterToGels(self):
        check(self.L.glsm_coupler_scatter(self.h), "scatterToGels")

    def applyGelRepulsion(self):
        check(self.L.glsm_coupler_repulsion(self.h), "applyGelRepulsion")

    def read(self, field):
        fid = MARKER_FIELDS[field] if isinstance(field, str) else int(field)
        n = (3 if fid <= 4 else 1) * self.M
        buf = np.empty(max(n, 1), dtype=np.float32)
        check(self.L.glsm_coupler_read(self.h, fid, _fptr(buf), buf.size), f"read {field}")
        return buf[:n]

    def stream(self):
        return self.L.glsm_coupler_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            check(self.L.glsm_coupler_destroy(self.h), "Coupler destroy")
            self.h = None
            for g in self.gels:
                g.coupler = None


class Fluid:
    """Fluid(dims, coupler) -- src/fluid.h:26, src/fluid.cu:152-232.

    `dims` are lattice cells per axis (the reference derives 2*s+1 from a
    physical size s; any size is accepted here).  Keyword overrides: nsub,
    storage ("f32" | "f16" | "bf16" | "f16c" | "f16c2": FP16 with the
    conserving rounding on every / every second substep), tau, beta, ramp_steps, force, periodic, fp16_scale, h;
    deterministic=True spreads by fixed-order gathers (a run repeats bit for
    bit) instead of float atomics.
    """

    def __init__(self, dims, coupler, deterministic=False, **kw):
        rounding = _STORAGE_ROUNDING.get(kw.get("storage"))
        self.L = lib()
        d = FluidDesc()
        check(self.L.glsm_fluid_desc_default(ctypes.byref(d), int(dims[0]), int(dims[1]), int(dims[2])), "desc")
        for k, v in kw.items():
            if v is None:
                continue
            if k == "storage":
                d.storage = STORAGE[v] if isinstance(v, str) else int(v)
            elif k in ("force", "periodic"):
                arr = getattr(d, k)
                for j in range(3):
                    arr[j] = v[j]
            else:
                setattr(d, k, v)
        self.desc = d
        h = ctypes.c_void_p()
        check(self.L.glsm_fluid_create(ctypes.byref(d), coupler.h, ctypes.byref(h)), "Fluid")
        self.h = h
        self.coupler = coupler
        coupler.fluid = self
        info = (ctypes.c_int64 * 8)()
        check(self.L.glsm_fluid_info(self.h, info), "info")
        self.nx, self.ny, self.nz, self.N, self.Nsub, self.storage, self.device_bytes, _ = (int(v) for v in info)
        if deterministic:
            self.set_deterministic(True)
        if rounding:
            self.set_f16_rounding(rounding)

    def set_l2_persisting(self, on=True):
        """Keep the population array in the persisting part of L2 across the
        substeps (off by default; for one system alone on the GPU;
        glsm_fluid_set_l2_persisting)."""
        check(self.L.glsm_fluid_set_l2_persisting(self.h, 1 if on else 0), "set_l2_persisting")

    def set_f16_rounding(self, mode="conserving"):
        """Rounding of FP16 storage: "nearest", "conserving" (each cell's
        mass and momentum rounding errors nearly cancel) or "conserving_odd"
        (conserving on odd substeps only); glsm_fluid_set_f16_rounding."""
        check(self.L.glsm_fluid_set_f16_rounding(self.h, F16_ROUNDING[mode]), "set_f16_rounding")

    def set_deterministic(self, on=True):
        """Spreads as fixed-order gathers (glsm_fluid_set_deterministic)."""
        check(self.L.glsm_fluid_set_deterministic(self.h, 1 if on else 0), "set_deterministic")

    def stepVelocity(self, it):
        check(self.L.glsm_fluid_step_velocity(self.h, int(it)), "stepVelocity")

    def stepConcentration(self, it):
        check(self.L.glsm_fluid_step_concentration(self.h, int(it)), "stepConcentration")

    def run(self, iter0, n):
        """n fused, graph-captured coupled iterations starting at iter0 (asynchronous)."""
        check(self.L.glsm_fluid_run(self.h, int(iter0), int(n)), "run")

    def save_checkpoint(self, path=None):
        """Exact-restart checkpoint of the whole system (fluid, coupler, gels):
        returned as bytes, and written to `path` when given."""
        n = ctypes.c_size_t()
        check(self.L.glsm_checkpoint_bytes(self.h, ctypes.byref(n)), "checkpoint size")
        buf = np.empty(n.value, dtype=np.uint8)
        check(self.L.glsm_checkpoint_save(self.h, buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes), "checkpoint")
        if path is not None:
            buf.tofile(path)
        return buf.tobytes()

    def load_checkpoint(self, data):
        """Restore a checkpoint (bytes, or the path of a file written by
        save_checkpoint) into this system, built with the same lattice and gels."""
        if isinstance(data, (str, os.PathLike)):
            buf = np.fromfile(data, dtype=np.uint8)
        else:
            buf = np.frombuffer(data, dtype=np.uint8)
        check(self.L.glsm_checkpoint_load(self.h, buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes), "load checkpoint")

    def sync(self):
        check(self.L.glsm_fluid_sync(self.h), "sync")

    def profile_velocity(self, it):
        """stepVelocity(it) with per-substep CUDA-event timings (ms) on the system stream."""
        ms = np.zeros(self.Nsub, dtype=np.float32)
        check(self.L.glsm_fluid_profile_velocity(self.h, int(it), _fptr(ms)), "profile_velocity")
        return ms

    def profile_substeps(self, it, n_steps=1):
        """n_steps calls of stepVelocity(it + j) as one captured graph of their
        substep launches; the time (ms) of the whole graph on the system stream."""
        out = ctypes.c_float()
        check(self.L.glsm_fluid_profile_substeps_n(self.h, int(it), int(n_steps), ctypes.byref(out)),
              "profile_substeps")
        return float(out.value)

    def test_ibm_wait_extra(self, extra):
        """Test aid: make the force-region tiles wait for `extra` IBM tasks that
        never run, so the bounded wait gives up (glsm_test_ibm_wait_extra)."""
        check(self.L.glsm_test_ibm_wait_extra(self.h, int(extra)), "test_ibm_wait_extra")

    def conservation(self):
        """(mass, px, py, pz): sum of rho and of c_q f_q over the lattice, reduced
        in FP64 on the device."""
        out = (ctypes.c_double * 4)()
        check(self.L.glsm_fluid_conservation(self.h, out), "conservation")
        return tuple(out)

    def units(self):
        out = (ctypes.c_float * 2)()
        check(self.L.glsm_fluid_units(self.h, out), "units")
        return tuple(out)

    def read(self, field):
        fid = FLUID_FIELDS[field] if isinstance(field, str) else int(field)
        n = {0: 19, 1: 1, 2: 3, 3: 1}[fid] * self.N
        buf = np.empty(n, dtype=np.float32)
        check(self.L.glsm_fluid_read(self.h, fid, _fptr(buf), n), f"read {field}")
        return buf

    def read_into(self, field, buf):
        fid = FLUID_FIELDS[field] if isinstance(field, str) else int(field)
        check(self.L.glsm_fluid_read(self.h, fid, _fptr(buf), buf.size), f"read {field}")

    def snapshot(self, u_buf, c_buf):
        """Output snapshot (glsm_fluid_snapshot): u (3 N float32) and the current
        c1 (N float32) behind the queued work, transferred to the page-locked
        buffers on a copy stream; returns at once (see snapshot_wait)."""
        if u_buf.dtype != np.float32 or c_buf.dtype != np.float32 or u_buf.size != 3 * self.N or c_buf.size != self.N:
            raise ValueError("snapshot buffers: float32, 3 N and N values")
        check(self.L.glsm_fluid_snapshot(self.h, _fptr(u_buf), _fptr(c_buf)), "snapshot")

    def snapshot_wait(self):
        check(self.L.glsm_fluid_snapshot_wait(self.h), "snapshot_wait")

    def write(self, field, values):
        fid = FLUID_FIELDS[field] if isinstance(field, str) else int(field)
        v = np.ascontiguousarray(values, dtype=np.float32).ravel()
        check(self.L.glsm_fluid_write(self.h, fid, _fptr(v), v.size), f"write {field}")

    def info(self):
        out = (ctypes.c_int64 * 8)()
        check(self.L.glsm_fluid_info(self.h, out), "info")
        return dict(nx=out[0], ny=out[1], nz=out[2], N=out[3], nsub=out[4], storage=out[5], device_bytes=out[6],
                    substeps=out[7])

    def close(self):
        if getattr(self, "h", None):
            check(self.L.glsm_fluid_destroy(self.h), "Fluid destroy")
            self.h = None
            self.coupler.fluid = None


class Batch:
    """Several systems advanced together by batched launches (include/glsm_b200.h glsm_batch_*)."""

    def __init__(self):
        self.L = lib()
        h = ctypes.c_void_p()
        check(self.L.glsm_batch_create(ctypes.byref(h)), "Batch")
        self.h = h
        self.members = []

    def add(self, fluid, iter0=0, n_iters=0):
        """fluid joins at iteration iter0 and runs n_iters iterations (0: no limit)."""
        check(self.L.glsm_batch_add(self.h, fluid.h, int(iter0), int(n_iters)), "batch add")
        self.members.append(fluid)

    def remaining(self, fluid):
        return self.L.glsm_batch_remaining(self.h, fluid.h)

    def remove(self, fluid):
        check(self.L.glsm_batch_remove(self.h, fluid.h), "batch remove")
        self.members.remove(fluid)

    def run(self, n):
        check(self.L.glsm_batch_run(self.h, int(n)), "batch run")

    def sync(self):
        check(self.L.glsm_batch_sync(self.h), "batch sync")

    def __len__(self):
        return self.L.glsm_batch_size(self.h)

    def close(self):
        if getattr(self, "h", None):
            check(self.L.glsm_batch_destroy(self.h), "Batch destroy")
            self.h = None
            self.members = []


class System:
    """One coupled system with the same construction interface as the CPU
    oracle and the reference harness used by the tests (add_gel, gel_noise,
    set_params, finalize, run, get with the oracle's field ids)."""

    def __init__(self, nx, ny, nz, nsub=25, storage="f32", fp16_scale=None, methods=False, deterministic=False):
        self.dims = (nx, ny, nz)
        self.deterministic = deterministic
        self.nsub = nsub
        self.storage = storage
        self.fp16_scale = fp16_scale
        self.methods = methods  # run() through the per-method calls instead of the fused graph
        self.gels = []
        self.params = dict(beta=1.0, ramp_steps=20000.0, force=(0.0, 0.0, 0.0), periodic=(0, 0, 0))
        self.coupler = None
        self.fluid = None
        self.active_from = {}

    def add_gel(self, size, pos, gel_type=1, gel_id=None):
        gid = len(self.gels) + 1 if gel_id is None else gel_id
        self.gels.append(Gel(size, pos, gel_type, gid))
        return len(self.gels) - 1

    def gel_noise(self, g, seed, amp):
        self.gels[g].add_noise(seed, amp)

    def reset_quiescent(self, g):
        self.gels[g].resetToQuiescent()

    def fire_pulse(self, g):
        self.gels[g].fireExcitationPulse()

    def set_anchor(self, g, z):
        self.gels[g].setAnchorZ(z)

    def set_active_from(self, g, it):
        self.active_from[g] = int(it)
        self.gels[g].set_active_from(it)

    def set_params(self, beta=1.0, ramp_steps=20000.0, force=(0.0, 0.0, 0.0), periodic=(0, 0, 0)):
        self.params = dict(beta=beta, ramp_steps=ramp_steps, force=force, periodic=periodic)

    def finalize(self):
        self.coupler = Coupler(self.gels)
        self.fluid = Fluid(self.dims, self.coupler, nsub=self.nsub, storage=self.storage,
                           fp16_scale=self.fp16_scale, deterministic=self.deterministic, **self.params)

    def run(self, iter0, n):
        if not self.methods:
            self.fluid.run(iter0, n)
            self.fluid.sync()
            return
        # the reference driver loop, method by method (src/sim.cpp:97-112)
        for it in range(iter0, iter0 + n):
            for k, g in enumerate(self.gels):
                af = self.active_from.get(k, 0)
                if af > 0 and it == af:
                    g.fireExcitationPulse()
            for k, g in enumerate(self.gels):
                af = self.active_from.get(k, 0)
                if af > 0 and it < af:
                    continue
                g.stepElasticity(it)
                g.stepChemistry(it)
            self.coupler.packFromGels()
            self.fluid.stepVelocity(it)
            self.fluid.stepConcentration(it)
            self.coupler.applyGelRepulsion()
            self.coupler.scatterToGels()
        self.fluid.sync()

    def info(self):
        return dict(N=self.fluid.N, M=self.coupler.M, n_gels=len(self.gels), nsub=self.fluid.Nsub)

    # oracle field ids: 0-4 lattice, 10-17 markers, 20-40 gel
    def get(self, fid, gel=0):
        if fid < 10:
            if fid == 4:
                return np.zeros(3 * self.fluid.N)
            return self.fluid.read(fid).astype(np.float64)
        if fid < 20:
            return self.coupler.read(fid - 10).astype(np.float64)
        return self.gels[gel].read(fid - 20)

    def close(self):
        if self.fluid:
            self.fluid.close()
        if self.coupler:
            self.coupler.close()
        for g in self.gels:
            g.close()
        self.fluid = self.coupler = None
        self.gels = []
