"""Loads libglsm_b200.so (built in-tree by build.py) and declares its C ABI.

There is no fallback: if the CUDA library cannot be found or built, importing
the package fails with the reason.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_lib = None


class GlsmError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path) or _build.needs_build():
        try:
            _build.build()
        except Exception as e:  # noqa: BLE001
            if not os.path.exists(path):
                raise ImportError(f"libglsm_b200.so is missing and could not be built: {e}") from e
    L = ctypes.CDLL(path)
    vp, i, d, f, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_uint64
    P = ctypes.POINTER
    L.glsm_last_error.restype = ctypes.c_char_p
    L.glsm_version.restype = i
    sig = {
        "glsm_gel_create": [i, i, i, d, d, d, i, i, P(vp)],
        "glsm_gel_destroy": [vp],
        "glsm_gel_info": [vp, P(ctypes.c_int64)],
        "glsm_gel_steady_state": [vp, P(d)],
        "glsm_gel_step_elasticity": [vp, i],
        "glsm_gel_step_chemistry": [vp, i],
        "glsm_gel_record_center": [vp, i],
        "glsm_gel_series_config": [vp, i, i],
        "glsm_gel_series_read": [vp, P(d), ctypes.c_size_t],
        "glsm_gel_reset_quiescent": [vp],
        "glsm_gel_fire_pulse": [vp],
        "glsm_gel_set_anchor_z": [vp, d],
        "glsm_gel_build_tube_mask": [vp, i, i],
        "glsm_gel_set_active_from": [vp, i],
        "glsm_gel_add_noise": [vp, u64, d],
        "glsm_gel_read": [vp, i, P(d), ctypes.c_size_t],
        "glsm_gel_write": [vp, i, P(d), ctypes.c_size_t],
        "glsm_gel_snapshot": [vp, i, P(i), P(P(d))],
        "glsm_gel_snapshot_wait": [vp],
        "glsm_coupler_create": [P(vp), i, P(vp)],
        "glsm_coupler_destroy": [vp],
        "glsm_coupler_pack": [vp],
        "glsm_coupler_scatter": [vp],
        "glsm_coupler_repulsion": [vp],
        "glsm_coupler_markers": [vp],
        "glsm_coupler_read": [vp, i, P(f), ctypes.c_size_t],
        "glsm_fluid_desc_default": [vp, i, i, i],
        "glsm_fluid_create": [vp, vp, P(vp)],
        "glsm_fluid_destroy": [vp],
        "glsm_fluid_step_velocity": [vp, i],
        "glsm_fluid_step_concentration": [vp, i],
        "glsm_fluid_run": [vp, i, i],
        "glsm_fluid_sync": [vp],
        "glsm_fluid_read": [vp, i, P(f), ctypes.c_size_t],
        "glsm_fluid_snapshot": [vp, P(f), P(f)],
        "glsm_fluid_snapshot_wait": [vp],
        "glsm_fluid_write": [vp, i, P(f), ctypes.c_size_t],
        "glsm_fluid_info": [vp, P(ctypes.c_int64)],
        "glsm_fluid_units": [vp, P(f)],
        "glsm_fluid_profile_velocity": [vp, i, P(f)],
        "glsm_fluid_conservation": [vp, P(d)],
        "glsm_fluid_set_deterministic": [vp, i],
        "glsm_gel_filament": [vp, P(d), ctypes.c_size_t, P(ctypes.c_size_t)],
        "glsm_fluid_profile_substeps": [vp, i, P(f)],
        "glsm_fluid_profile_substeps_n": [vp, i, i, P(f)],
        "glsm_test_ibm_wait_extra": [vp, i],
        "glsm_gel_set_bz_f": [vp, d],
        "glsm_checkpoint_bytes": [vp, P(ctypes.c_size_t)],
        "glsm_checkpoint_save": [vp, vp, ctypes.c_size_t],
        "glsm_checkpoint_load": [vp, vp, ctypes.c_size_t],
        "glsm_batch_create": [P(vp)],
        "glsm_batch_destroy": [vp],
        "glsm_batch_add": [vp, vp, i, i],
        "glsm_batch_remove": [vp, vp],
        "glsm_batch_size": [vp],
        "glsm_batch_run": [vp, i],
        "glsm_batch_sync": [vp],
        "glsm_fluid_set_f16_rounding": [vp, i],
        "glsm_fluid_set_l2_persisting": [vp, i],
        "glsm_l2_reset_persisting": [],
        "glsm_l2_persisting_setaside": [P(ctypes.c_size_t)],
        "glsm_f16_conserve_round": [vp, vp, ctypes.c_size_t],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i
    L.glsm_gel_field_size.argtypes = [vp, i]
    L.glsm_gel_field_size.restype = ctypes.c_size_t
    L.glsm_gel_device_ptr.argtypes = [vp, i]
    L.glsm_gel_device_ptr.restype = vp
    L.glsm_batch_remaining.argtypes = [vp, vp]
    L.glsm_batch_remaining.restype = ctypes.c_longlong
    L.glsm_coupler_stream.argtypes = [vp]
    L.glsm_coupler_stream.restype = vp
    L.glsm_copy_bandwidth.argtypes = [ctypes.c_size_t, i, P(d)]
    L.glsm_pattern_bandwidth.argtypes = [i, i, i, i, i, P(d), P(d)]
    L.glsm_copy_bandwidth.restype = i
    L.glsm_copy_bandwidth_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = lib().glsm_last_error().decode(errors="replace")
        raise GlsmError(f"{what}: status {rc}: {msg}")


class FluidDesc(ctypes.Structure):
    """glsm_fluid_desc (include/glsm_b200.h)."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nsub", ctypes.c_int), ("storage", ctypes.c_int),
        ("tau", ctypes.c_float), ("beta", ctypes.c_float), ("ramp_steps", ctypes.c_float),
        ("force", ctypes.c_float * 3), ("periodic", ctypes.c_int * 3),
        ("fp16_scale", ctypes.c_float), ("h", ctypes.c_float),
    ]
