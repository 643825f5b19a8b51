"""Output snapshots through the Python binding (glsm_gel_snapshot,
glsm_fluid_snapshot): each snapshot holds the fields as they were behind the
work queued before it, while later iterations run on; compared bit for bit
with synchronous reads of a second, identical system stopped at the same
iteration (deterministic spreads)."""
import numpy as np
import pytest
import torch

from cases import build

pytestmark = pytest.mark.gpu


def _pinned(n, dtype):
    return torch.empty(n, dtype=dtype, pin_memory=True).numpy()


def _system():
    from glsm_fluid_3d_b200 import System

    return build(System, "pair", deterministic=True)


def test_snapshots_match_synchronous_reads(gpu):
    a = _system()
    g0 = a.gels[0]
    nN = g0.read("Veln").size
    N = a.fluid.N
    vel = [_pinned(nN, torch.float64) for _ in range(4)]
    um = [_pinned(g0.read("um").size, torch.float64) for _ in range(4)]
    u = _pinned(3 * N, torch.float32)
    c = _pinned(N, torch.float32)
    # four iterations queued back to back, a gel snapshot after each; the
    # fluid snapshot after the third
    for k in range(4):
        a.fluid.run(k, 1)
        g0.snapshot(["Veln", "um"], [vel[k], um[k]])
        if k == 2:
            a.fluid.snapshot(u, c)
    g0.snapshot_wait()
    a.fluid.snapshot_wait()
    a.fluid.sync()
    for k in range(4):
        b = _system()
        b.fluid.run(0, k + 1)
        b.fluid.sync()
        assert np.array_equal(vel[k], b.gels[0].read("Veln")), k
        assert np.array_equal(um[k], b.gels[0].read("um")), k
        if k == 2:
            assert np.array_equal(u, b.fluid.read("u")), "u"
            assert np.array_equal(c, b.fluid.read("c1")), "c1"
        b.close()
    a.close()


def test_snapshot_rejects_wrong_buffers(gpu):
    a = _system()
    with pytest.raises(ValueError):
        a.gels[0].snapshot(["Veln"], [np.zeros(3, dtype=np.float64)])
    with pytest.raises(ValueError):
        a.fluid.snapshot(np.zeros(3, dtype=np.float32), np.zeros(3, dtype=np.float32))
    a.close()
