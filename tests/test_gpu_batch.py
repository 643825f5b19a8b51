"""Batched execution and the continuous-batching server.

A system's result must be the same alone and in the mix: systems of different
lattice sizes, gel counts and storages advanced together by one batch (one
persistent launch per substep for each group of systems that share storage
and substep parity), including a system that joins
while the others are running, agree with the same systems advanced alone.  The
spreads use float atomics, so agreement is to round-off (relative L2 <= 1e-5)
for FP32 storage and to FP16 precision for FP16 storage.
"""
import numpy as np
import pytest

from parity import rel_l2

pytestmark = pytest.mark.gpu

SPECS = [
    dict(dims=(24, 24, 24), gels=[((6, 6, 6), (5.75, 5.75, 5.75))], storage="f32", seed=1),
    dict(dims=(32, 28, 30), gels=[((4, 4, 4), (4.0, 6.5, 7.0)), ((4, 4, 4), (10.5, 6.5, 7.0))], storage="f32",
         seed=2),
    dict(dims=(20, 20, 36), gels=[((3, 3, 8), (4.75, 4.75, 8.75))], storage="f16", seed=3),
]


def make(spec):
    from glsm_fluid_3d_b200 import System

    s = System(*spec["dims"], nsub=25, storage=spec["storage"])
    for k, (size, pos) in enumerate(spec["gels"]):
        s.add_gel(size, pos, 1, k + 1)
        s.gel_noise(k, spec["seed"], 1e-3)
    s.set_params(beta=1.0, ramp_steps=0.0)
    s.finalize()
    return s


def state(s):
    out = {"u": s.fluid.read("u"), "c1": s.fluid.read("c1"), "pop": s.fluid.read("pop")}
    for k, g in enumerate(s.gels):
        out[f"g{k}_rn"] = g.read("rn")
        out[f"g{k}_um"] = g.read("um")
    return out


def compare(a, b, tol):
    return {k: rel_l2(a[k], b[k]) for k in b if rel_l2(a[k], b[k]) > tol.get(k.split("_")[-1], 1e-5)}


TOL = {"u": 1e-5, "c1": 1e-5, "pop": 1e-6, "rn": 1e-9, "um": 1e-9}
# FP16 storage: a round-off-sized difference in the order of the float atomics
# flips FP16 roundings, so agreement is to FP16 precision (the tolerance of the
# FP16-storage tests against the FP64 oracle)
TOL16 = {"u": 2e-3, "c1": 1e-4, "pop": 1e-5, "rn": 1e-7, "um": 1e-7}


def test_alone_and_in_the_mix(gpu):
    from glsm_fluid_3d_b200 import Batch

    # systems 0 and 1 run 3 + 5 + 3 = 11 iterations in the batch; system 2 runs
    # 5 in the mix and 3 more alone
    alone = []
    for spec, n in zip(SPECS, (11, 11, 8)):
        s = make(spec)
        s.fluid.run(0, n)
        s.fluid.sync()
        alone.append(state(s))
        s.close()
    # the same systems in one batch; the third joins after 3 iterations
    systems = [make(spec) for spec in SPECS]
    b = Batch()
    b.add(systems[0].fluid, 0)
    b.add(systems[1].fluid, 0)
    b.run(3)
    b.sync()
    b.add(systems[2].fluid, 0)
    b.run(5)
    b.sync()
    b.remove(systems[2].fluid)
    b.run(3)  # third system: 5 iterations in the mix, then 3 more alone
    b.sync()
    systems[2].fluid.run(5, 3)
    systems[2].fluid.sync()
    for k in range(3):
        got = state(systems[k])
        bad = compare(got, alone[k], TOL16 if SPECS[k]["storage"] == "f16" else TOL)
        assert not bad, (k, bad)
    b.close()
    for s in systems:
        s.close()


def test_server_completes_requests_with_equal_results(gpu):
    from glsm_fluid_3d_b200 import serving

    reqs = serving.make_requests(n=10, rate=200.0, seed=7, step_scale=0.004, sides=(24, 32))
    for r in reqs:
        r.storage = "f32"
    srv = serving.Server(budget_bytes=8e9, max_chunk=4, keep_results=True)
    st = srv.serve(reqs)
    summ = st.summary()
    assert summ["requests"] == len(reqs)
    assert summ["p99_latency_s"] >= summ["p50_latency_s"] > 0
    assert summ["max_resident_systems"] >= 2  # requests overlapped on the device
    _, seq = serving.sequential(reqs, keep_results=True, storage=None)
    for r in reqs:
        bad = compare(srv.results[r.rid], seq[r.rid], TOL)
        assert not bad, (r.rid, bad)


def test_server_respects_hbm_budget(gpu):
    from glsm_fluid_3d_b200 import serving

    reqs = serving.make_requests(n=4, rate=1000.0, seed=3, step_scale=0.002, sides=(32,))
    one = max(serving.device_bytes(r) for r in reqs)
    st = serving.Server(budget_bytes=one * 1.5, max_chunk=2).serve(reqs)
    assert st.max_resident == 1 and len(st.latencies) == 4
