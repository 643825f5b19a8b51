"""The serving comparison's one-at-a-time server (serving.fifo): host logic,
no GPU.  A request starts when it has arrived and the previous one is done;
latency is completion minus arrival."""
import math

import pytest

from glsm_fluid_3d_b200 import serving


def _req(rid, arrival, side=32, steps=10):
    return serving.Request(rid, arrival, side, [], 0.9, steps, "f32", 0)


def test_fifo_waits_for_arrivals_and_for_the_previous_request():
    reqs = [_req(0, 0.0), _req(1, 0.1), _req(2, 5.0)]
    out = serving.fifo(reqs, [1.0, 1.0, 0.5])
    # 0: [0, 1]; 1 arrives at 0.1, runs [1, 2]; 2 arrives at 5, runs [5, 5.5]
    assert out["makespan_s"] == pytest.approx(5.5)
    lat = sorted([1.0, 1.9, 0.5])
    assert out["p50_latency_s"] == pytest.approx(lat[1])
    assert out["p99_latency_s"] == pytest.approx(lat[2])
    work = sum(r.cells * 25.0 * r.steps for r in reqs)
    assert out["aggregate_mlups"] == pytest.approx(round(work / 5.5 / 1e6, 1))


def test_fifo_orders_by_arrival_not_by_list_position():
    a, b = _req(0, 2.0), _req(1, 0.0)
    out = serving.fifo([a, b], [1.0, 3.0])  # b (3 s) first, then a at 3
    assert out["makespan_s"] == pytest.approx(4.0)
    assert out["p99_latency_s"] == pytest.approx(3.0)  # b: 3 - 0; a: 4 - 2 = 2


def test_fifo_of_simultaneous_arrivals_is_the_sum_of_the_solves():
    reqs = serving.make_requests(20, 8.0, 7, 0.1)
    at_once = [serving.Request(r.rid, 0.0, r.side, r.gels, r.f, r.steps, r.storage, r.seed) for r in reqs]
    d = [0.01 * (k + 1) for k in range(20)]
    out = serving.fifo(at_once, d)
    assert out["makespan_s"] == pytest.approx(round(sum(d), 3))
    assert math.isfinite(out["p50_latency_s"])
