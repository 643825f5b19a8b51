"""Comparison helpers shared by the parity tests."""
import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    if den == 0.0:
        return float(np.linalg.norm(a - b))
    return float(np.linalg.norm(a - b) / den)


def max_abs(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.abs(a - b).max()) if a.size else 0.0


def report(got: dict, want: dict, keys=None):
    """{field: (rel_l2, max_abs, scale)} for the fields present in both."""
    keys = keys or [k for k in want if k in got]
    return {k: (rel_l2(got[k], want[k]), max_abs(got[k], want[k]), float(np.abs(want[k]).max())) for k in keys}


def tolerance_for(name: str, tol: dict, default: float) -> float:
    for prefix, t in tol.items():
        if name == prefix or name.endswith("_" + prefix):
            return t
    return default
