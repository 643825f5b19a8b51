"""Exact-restart checkpoint (glsm_checkpoint_*).

A checkpoint taken mid-run and loaded into a freshly built system reproduces
the saved state byte for byte (a second checkpoint of the restored system is
identical to the first), including the mutable gel settings and an odd AA
layout of the populations.  Continuing both systems gives the same results up
to the ordering of floating-point atomics in the spreads, which also separates
two uninterrupted runs.
"""
import numpy as np
import pytest

from glsm_fluid_3d_b200 import GlsmError, System
from parity import rel_l2

pytestmark = pytest.mark.gpu

DIMS, NSUB = (24, 20, 28), 3


def _build(with_settings=True, dims=DIMS):
    s = System(*dims, nsub=NSUB)
    s.add_gel((3, 3, 3), (3.75, 4.75, 6.75), 1, 1)
    s.add_gel((3, 3, 3), (8.25, 4.75, 6.75), 2, 2)
    s.gel_noise(0, 5, 1e-3)
    s.gel_noise(1, 6, 1e-3)
    if with_settings:
        s.reset_quiescent(1)
        s.set_active_from(1, 7)
    s.set_params(beta=1.0, ramp_steps=0.0)
    s.finalize()
    return s


def _state(s):
    out = {"u": s.get(2), "c1": s.get(3)}
    for g in range(2):
        for name, fid in (("rn", 20), ("um", 24), ("vm", 25), ("veln", 21)):
            out[f"g{g}_{name}"] = s.get(fid, g)
    return out


def test_checkpoint_roundtrip_and_continuation(gpu, tmp_path):
    a = _build()
    a.run(0, 5)  # 15 substeps: the populations are in the reversed (odd) layout
    path = tmp_path / "sys.ckpt"
    c1 = a.fluid.save_checkpoint(str(path))

    b = _build(with_settings=False)  # activation comes from the checkpoint
    b.fluid.load_checkpoint(str(path))
    c2 = b.fluid.save_checkpoint()
    assert c1 == c2

    # the methods path honours the host-side activation bookkeeping of System
    b.active_from = dict(a.active_from)
    a.run(5, 8)
    b.run(5, 8)
    sa, sb = _state(a), _state(b)
    rows = []
    for k in sa:
        e = rel_l2(sb[k], sa[k])
        t = 1e-5 if k in ("u", "c1") else 1e-9
        rows.append((k, e, t))
    print("\n".join(f"{k:10s} rel_l2={e:.2e} tol={t:.0e}" for k, e, t in rows))
    assert all(e <= t for _, e, t in rows), rows
    a.close()
    b.close()


def test_checkpoint_rejects_other_systems(gpu):
    a = _build()
    a.run(0, 2)
    data = a.fluid.save_checkpoint()
    other = _build(dims=(24, 20, 26))
    with pytest.raises(GlsmError):
        other.fluid.load_checkpoint(data)
    with pytest.raises(GlsmError):
        a.fluid.load_checkpoint(data[:100])
    with pytest.raises(GlsmError):
        a.fluid.load_checkpoint(b"x" * len(data))
    a.fluid.load_checkpoint(data)  # the intact checkpoint still loads
    a.close()
    other.close()
