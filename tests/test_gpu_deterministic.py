"""Deterministic spreads (glsm_fluid_set_deterministic): every cell inside a
marker box gathers its IBM force and concentration source from the markers in
a fixed order instead of the markers adding them with float atomics.

* the results agree with the FP64 oracle as closely as the atomic form does;
* a run repeats bit for bit (fused graph and per-method paths);
* a system gives bit-identical results alone and inside a batch.
"""
import numpy as np
import pytest

from cases import CASES, build, collect
from oracle.pyoracle import Oracle
from parity import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"u": 2e-4, "Ul": 2e-4, "Fdrag": 2e-5, "pop": 1e-6, "rho": 1e-6, "c1": 1e-5, "Dl": 1e-5, "Sl": 1e-5,
       "Cl": 1e-5, "Frep": 1e-5, "lag": 1e-7, "Vl": 1e-6, "un_robin": 1e-5, "un_norm": 1e-6}
GEL_TOL = 1e-8


def _run(case, methods=False, deterministic=True):
    from glsm_fluid_3d_b200 import System

    sim = build(System, case, methods=methods, deterministic=deterministic)
    sim.run(0, CASES[case]["iters"])
    out = collect(sim, case)
    sim.close()
    return out


@pytest.mark.parametrize("case", list(CASES))
def test_deterministic_matches_oracle(gpu, case):
    got = _run(case)
    ref = build(Oracle, case)
    ref.run(0, CASES[case]["iters"])
    want = collect(ref, case)
    ref.close()
    bad = []
    for k in want:
        if k.endswith("_T1"):
            continue
        name = k.split("_", 1)[1] if k.startswith("g") and "_" in k else k
        tol = TOL.get(name, GEL_TOL if k.startswith("g") else 1e-4)
        e = rel_l2(got[k], want[k])
        if not e <= tol:
            bad.append((k, e, tol))
    assert not bad, bad


@pytest.mark.parametrize("methods", [False, True], ids=["fused", "methods"])
def test_deterministic_runs_repeat_bit_for_bit(gpu, methods):
    a = _run("pair", methods=methods)
    b = _run("pair", methods=methods)
    diff = [k for k in a if not np.array_equal(a[k], b[k])]
    assert not diff, diff


def test_deterministic_close_to_atomic(gpu):
    a = _run("single", deterministic=True)
    b = _run("single", deterministic=False)
    for k in ("u", "pop", "Fdrag", "c1"):
        assert rel_l2(a[k], b[k]) < 1e-5, k


def test_deterministic_same_alone_and_in_batch(gpu):
    from glsm_fluid_3d_b200 import Batch, System

    def make(dims, pos, seed):
        s = System(*dims, nsub=3, deterministic=True)
        s.add_gel((3, 3, 3), pos, 1, 1)
        s.gel_noise(0, seed, 1e-3)
        s.set_params(beta=1.0, ramp_steps=0.0)
        s.finalize()
        return s

    specs = [((20, 18, 22), (4.75, 4.25, 5.25), 11), ((24, 20, 16), (5.75, 4.75, 3.75), 12)]
    alone = []
    for dims, pos, seed in specs:
        s = make(dims, pos, seed)
        s.run(0, 6)
        alone.append((s.fluid.read("u"), s.fluid.read("pop"), s.gels[0].read("rn")))
        s.close()
    systems = [make(*sp) for sp in specs]
    b = Batch()
    for s in systems:
        b.add(s.fluid, 0, 6)
    b.run(6)
    b.sync()
    for s, want in zip(systems, alone):
        got = (s.fluid.read("u"), s.fluid.read("pop"), s.gels[0].read("rn"))
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
    for s in systems:
        b.remove(s.fluid)
        s.close()
    b.close()


def test_deterministic_same_alone_and_in_a_mixed_batch(gpu):
    """The batch launches its systems in groups (storage and FP16 rounding, x
    periodicity, substep parity); one batch holding every kind, with systems that join with
    an odd substep count after running alone first, still reproduces each
    system alone bit for bit."""
    from glsm_fluid_3d_b200 import Batch, System

    # (dims, gel position, storage, periodic, iterations alone before joining)
    specs = [((20, 18, 22), (4.75, 4.25, 5.25), "f32", (0, 0, 0), 0),
             ((24, 20, 16), (5.75, 4.75, 3.75), "f16", (0, 0, 0), 1),
             ((18, 22, 20), (4.25, 5.75, 4.75), "bf16", (1, 0, 0), 0),
             ((22, 16, 18), (5.25, 3.75, 4.25), "f32", (1, 0, 1), 1),
             ((16, 24, 20), (3.75, 5.25, 4.75), "f16", (1, 0, 0), 2),
             ((20, 20, 18), (4.75, 4.75, 4.25), "f16c", (0, 0, 0), 1),
             ((18, 20, 22), (4.25, 4.75, 5.25), "f16c2", (1, 0, 0), 0)]

    def make(dims, pos, storage, periodic, seed):
        s = System(*dims, nsub=3, storage=storage, deterministic=True)
        s.add_gel((3, 3, 3), pos, 1, 1)
        s.gel_noise(0, seed, 1e-3)
        s.set_params(beta=1.0, ramp_steps=0.0, periodic=periodic)
        s.finalize()
        return s

    total = 7
    alone = []
    for k, (dims, pos, storage, per, pre) in enumerate(specs):
        s = make(dims, pos, storage, per, 20 + k)
        s.run(0, total)
        alone.append((s.fluid.read("u"), s.fluid.read("pop"), s.gels[0].read("rn")))
        s.close()
    systems = []
    b = Batch()
    for k, (dims, pos, storage, per, pre) in enumerate(specs):
        s = make(dims, pos, storage, per, 20 + k)
        if pre:
            s.run(0, pre)
        s.fluid.sync()
        b.add(s.fluid, pre, total - pre)
        systems.append(s)
    b.run(total)
    b.sync()
    for k, (s, want) in enumerate(zip(systems, alone)):
        got = (s.fluid.read("u"), s.fluid.read("pop"), s.gels[0].read("rn"))
        for name, g, w in zip(("u", "pop", "rn"), got, want):
            assert np.array_equal(g, w), (k, specs[k][2], name)
    for s in systems:
        b.remove(s.fluid)
        s.close()
    b.close()


def test_l2_persisting_window_changes_no_result(gpu):
    """The L2 access-policy window of the substep launches (opt-in) only
    steers caching: with deterministic spreads the results are bit-identical
    with it switched off, and releasing the persisting lines between runs
    changes nothing either."""
    from glsm_fluid_3d_b200 import System, l2_reset_persisting

    outs = []
    for on in (False, True):
        sim = build(System, "pair", deterministic=True)
        sim.fluid.set_l2_persisting(on)
        sim.run(0, CASES["pair"]["iters"] // 2)
        l2_reset_persisting()
        sim.run(CASES["pair"]["iters"] // 2, CASES["pair"]["iters"] - CASES["pair"]["iters"] // 2)
        outs.append(collect(sim, "pair"))
        sim.close()
    diff = [k for k in outs[0] if not np.array_equal(outs[0][k], outs[1][k])]
    assert not diff, diff


def test_l2_setaside_follows_the_fluids_that_use_it(gpu):
    """The persisting L2 set-aside exists only while a fluid keeps its
    populations L2-persisting: sized to the largest such array, released when
    the last one turns the window off, is destroyed or joins a batch."""
    from glsm_fluid_3d_b200 import Batch, System, l2_persisting_setaside

    def make(dims, storage):
        s = System(*dims, nsub=3, storage=storage)
        s.add_gel((3, 3, 3), (4.75, 4.75, 4.75), 1, 1)
        s.set_params(beta=1.0, ramp_steps=0.0)
        s.finalize()
        return s

    assert l2_persisting_setaside() == 0
    a = make((64, 64, 64), "f32")
    b = make((24, 24, 24), "f16")
    assert l2_persisting_setaside() == 0  # off by default
    a.fluid.set_l2_persisting(True)
    big = l2_persisting_setaside()
    assert big > 0
    b.fluid.set_l2_persisting(True)
    assert l2_persisting_setaside() == big  # the largest window in use
    a.fluid.set_l2_persisting(False)
    small = l2_persisting_setaside()
    assert 0 < small < big
    a.fluid.set_l2_persisting(True)
    a.close()  # destroying a user releases its share
    assert l2_persisting_setaside() == small
    batch = Batch()
    batch.add(b.fluid, 0, 2)  # joining a batch turns the window off
    assert l2_persisting_setaside() == 0
    batch.run(2)
    batch.sync()
    batch.remove(b.fluid)
    batch.close()
    b.close()
