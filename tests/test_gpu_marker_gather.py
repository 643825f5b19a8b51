"""The fused iteration gathers the gels' surface markers (Coupler::packFromGels,
src/coupling.cu:82-98, kernel k_gather_boundary, src/coupling_kernels.cu:42)
only when they can have changed: after the mechanics moved the nodes (every
5th iteration), or first in a run call after the host changed a gel (fields,
parameters, per-method steps, checkpoints, batches) or handed out one of its
device pointers.  Between those the marker arrays are a function of unchanged
node fields, so skipping the gather is exact; these tests check that, and that
each kind of change reaches the markers of the next iteration.
"""
import ctypes

import numpy as np
import pytest

from cases import CASES, build, collect

pytestmark = pytest.mark.gpu

SHIFT = 0.0625  # exact in float32 and float64


def _system(case, **kw):
    from glsm_fluid_3d_b200 import System

    return build(System, case, deterministic=True, **kw)


def _run_split(sim, iters):
    """One run call per iteration, a host read between calls."""
    for it in range(iters):
        sim.fluid.run(it, 1)
        sim.gels[0].read("rn")
    sim.fluid.sync()


@pytest.mark.parametrize("case", ["pair", "rod"])
def test_skipped_gathers_are_exact(gpu, case):
    """A run whose non-mechanics iterations reuse the markers equals, bit for
    bit, runs that gather every iteration (a device pointer is out, so each
    run call gathers afresh)."""
    iters = CASES[case]["iters"]
    a = _system(case)
    a.run(0, iters)
    got_one_call = collect(a, case)
    a.close()

    b = _system(case)
    _run_split(b, iters)
    got_split = collect(b, case)
    b.close()

    c = _system(case)
    c.gels[0].device_ptr("rn")  # from here on every run call gathers
    _run_split(c, iters)
    always = collect(c, case)
    c.close()

    for k in always:
        assert np.array_equal(got_one_call[k], always[k]), k
        assert np.array_equal(got_split[k], always[k]), k


def _lag(sim):
    return sim.coupler.read("lag").reshape(-1, 3)


def _shifted_markers_after(sim, change):
    """Run to iteration 3, apply change(sim) (which moves every node of gel 0
    by SHIFT in x), run iteration 3 (no mechanics): the markers of gel 0 must
    have moved by SHIFT."""
    sim.fluid.run(0, 3)
    sim.fluid.sync()
    before = _lag(sim).copy()
    change(sim)
    sim.fluid.run(3, 1)
    sim.fluid.sync()
    after = _lag(sim)
    m0 = sim.gels[0].m_boundaryCount
    return after[:m0] - before[:m0]


def _host_write(sim):
    g = sim.gels[0]
    rn = g.read("rn").reshape(-1, 3)
    rn[:, 0] += SHIFT
    g.write("rn", rn)


def _device_write(sim):
    import torch

    g = sim.gels[0]
    n = g.read("rn").size
    ptr = g.device_ptr("rn")

    class View:
        __cuda_array_interface__ = {"shape": (n // 3, 3), "typestr": "<f8", "data": (ptr, False), "version": 3}

    t = torch.as_tensor(View(), device="cuda")
    t[:, 0] += SHIFT
    torch.cuda.synchronize()


@pytest.mark.parametrize("change", [_host_write, _device_write], ids=["field_write", "device_pointer"])
def test_node_changes_between_calls_reach_the_markers(gpu, change):
    sim = _system("single")
    d = _shifted_markers_after(sim, change)
    sim.close()
    # float32 positions of float64 nodes moved by an exact shift
    assert np.allclose(d[:, 0], SHIFT, atol=4e-6), (d[:, 0].min(), d[:, 0].max())
    assert np.abs(d[:, 1:]).max() == 0.0


def test_checkpoint_load_reaches_the_markers(gpu):
    """A checkpoint taken before the nodes were shifted, loaded after a run of
    the shifted gel, brings the markers back with the nodes."""
    sim = _system("single")
    sim.fluid.run(0, 3)
    sim.fluid.sync()
    blob = sim.fluid.save_checkpoint()
    lag0 = _lag(sim).copy()
    _host_write(sim)
    sim.fluid.run(3, 1)
    sim.fluid.sync()
    assert not np.array_equal(_lag(sim), lag0)
    sim.fluid.load_checkpoint(blob)
    sim.fluid.run(3, 1)  # iteration 3 again: no mechanics, the gather comes from the load
    sim.fluid.sync()
    ref = _system("single")
    ref.fluid.run(0, 4)
    ref.fluid.sync()
    assert np.array_equal(_lag(sim), _lag(ref))
    sim.close()
    ref.close()


def test_batch_member_sees_node_changes_between_runs(gpu):
    """The batched gel kernel packs markers by the same rule: a field write to a
    member between batch runs reaches its markers at the next iteration."""
    from glsm_fluid_3d_b200 import Batch

    sim = _system("single")
    b = Batch()
    b.add(sim.fluid, 0, 0)
    b.run(3)
    b.sync()
    before = _lag(sim).copy()
    _host_write(sim)
    b.run(1)  # iteration 3: no mechanics
    b.sync()
    d = _lag(sim) - before
    b.remove(sim.fluid)
    b.close()
    sim.close()
    assert np.allclose(d[:, 0], SHIFT, atol=4e-6), (d[:, 0].min(), d[:, 0].max())
    assert np.abs(d[:, 1:]).max() == 0.0

