"""Continuous-batching serving loop for independent gel-fluid simulations.

Requests arrive over (wall-clock) time.  Each request is one coupled system:
a cubic lattice, 1-4 gels, a BZ parameter f, a number of iterations and a
population storage.  The server admits arriving requests as long as the HBM
budget allows, keeps every admitted system resident on the device and advances
all of them together: one `Batch` (C ABI glsm_batch_*) whose iteration is a CUDA
graph of batched launches -- one persistent launch per LBM substep for all
members.  Between chunks of iterations it retires finished systems (reading
their results back) and admits new arrivals, so requests that arrive while
others run join the running batch.

`sequential()` runs the same requests one after another, each alone with the
plain FP32 form, as the baseline; `fifo()` replays its measured solve times as
a one-at-a-time server on the same arrivals, for like-for-like makespan and
latency figures.
"""
from __future__ import annotations

import dataclasses
import math
import random
import statistics
import time
from typing import Dict, List, Optional

import numpy as np

from . import Batch, System

SIDES = (32, 48, 64, 96, 128)
F_REF = 0.9


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of serving
    side: int               # lattice cells per axis
    gels: list              # [(size (ex, ey, ez), position (x, y, z))]
    f: float                # BZ stoichiometric factor
    steps: int              # coupled iterations
    storage: str            # "f32" or "f16"
    seed: int

    @property
    def cells(self) -> int:
        return self.side ** 3


def _place_gels(rng: random.Random, side: int, n: int):
    """n non-overlapping cubic gels of 4-8 elements, 1.5 units from the walls."""
    extent = (side - 1) * 0.5  # physical size of the lattice (h = 0.5)
    placed = []
    for _ in range(n):
        for _attempt in range(200):
            e = rng.randint(4, 8)
            half = e / 2.0
            lo, hi = half + 1.5, extent - half - 1.5
            if hi <= lo:
                continue
            pos = tuple(rng.uniform(lo, hi) for _ in range(3))
            if all(max(abs(pos[k] - q[1][k]) for k in range(3)) > half + q[0][0] / 2.0 + 1.0 for q in placed):
                placed.append(((e, e, e), pos))
                break
    return placed or [((4, 4, 4), (extent / 2,) * 3)]


def make_requests(n: int = 256, rate: float = 8.0, seed: int = 2024, step_scale: float = 1.0,
                  sides=SIDES) -> List[Request]:
    """The serving ensemble: seeded Poisson arrivals at `rate` per second, side
    from `sides`, 1-4 gels of 4-8 elements, f within +-10% of 0.9, 500-5000
    iterations (times step_scale), FP32 or FP16 storage half and half."""
    rng = random.Random(seed)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.expovariate(rate)
        side = rng.choice(sides)
        gels = _place_gels(rng, side, rng.randint(1, 4))
        f = F_REF * rng.uniform(0.9, 1.1)
        steps = max(1, int(round(rng.randint(500, 5000) * step_scale)))
        storage = "f32" if rng.random() < 0.5 else "f16"
        reqs.append(Request(i, t, side, gels, f, steps, storage, rng.randrange(1 << 30)))
    return reqs


def device_bytes(req: Request) -> int:
    """Device memory of one system: populations, u, IBM force, two
    concentration fields and the source, plus the gels (FP64, ~2.3 kB per node)."""
    n = req.cells
    s = (n + 63) // 64 * 64
    pop = 19 * s * (4 if req.storage == "f32" else 2)
    gel = sum(int((e[0] + 3) * (e[1] + 3) * (e[2] + 3) * 2400) for e, _ in req.gels)
    return pop + 32 * n + 12 * n + gel + (1 << 20)


def build_system(req: Request, storage: Optional[str] = None) -> System:
    s = System(req.side, req.side, req.side, nsub=25, storage=storage or req.storage)
    for k, (size, pos) in enumerate(req.gels):
        s.add_gel(size, pos, 1, k + 1)
        s.gels[k].set_bz_f(req.f)
        s.gel_noise(k, req.seed, 1e-3)
    s.finalize()
    return s


def result_of(s: System) -> Dict[str, np.ndarray]:
    """What a request returns: the gels' node positions and chemistry, and the
    fluid velocity and concentration fields."""
    out = {"u": s.fluid.read("u"), "c1": s.fluid.read("c1")}
    for k, g in enumerate(s.gels):
        out[f"g{k}_rn"] = g.read("rn")
        out[f"g{k}_um"] = g.read("um")
    return out


@dataclasses.dataclass
class Stats:
    latencies: List[float]
    makespan: float
    cell_updates: float
    max_resident: int
    batches: int
    build_s: float = 0.0  # host time spent building systems (overlapped with running chunks)
    wait_s: float = 0.0   # host time blocked on running chunks

    def summary(self) -> dict:
        lat = sorted(self.latencies)
        pct = lambda p: lat[min(len(lat) - 1, int(math.ceil(p / 100 * len(lat))) - 1)] if lat else float("nan")  # noqa: E731
        return {"requests": len(lat), "makespan_s": round(self.makespan, 3),
                "aggregate_mlups": round(self.cell_updates / self.makespan / 1e6, 1),
                "p50_latency_s": round(pct(50), 3), "p99_latency_s": round(pct(99), 3),
                "mean_latency_s": round(statistics.mean(lat), 3) if lat else None,
                "max_resident_systems": self.max_resident, "batch_runs": self.batches,
                "build_s": round(self.build_s, 3), "wait_s": round(self.wait_s, 3)}


class Server:
    """Admits requests by HBM budget and advances all resident systems together.

    Each round launches a chunk of batched iterations -- up to the iteration at
    which the first member completes, at most max_chunk -- and, while it runs
    on the device, builds the systems of the requests that have arrived (as far
    as the budget allows); after the chunk it retires the finished systems
    (reading their results) and adds the newly built ones to the batch."""

    def __init__(self, budget_bytes: float = 150e9, max_chunk: int = 20, keep_results: bool = False):
        self.budget = budget_bytes
        self.max_chunk = max_chunk
        self.keep_results = keep_results
        self.results: Dict[int, Dict[str, np.ndarray]] = {}

    def serve(self, requests: List[Request], clock=time.perf_counter) -> Stats:
        pending = sorted(requests, key=lambda r: r.arrival)
        active = {}  # rid -> [request, system, remaining]
        built = []   # [request, system] built while the batch ran, not yet added
        used = 0
        batch = Batch()
        lat, max_res, runs = [], 0, 0
        work = build_s = wait_s = 0.0
        t0 = clock()

        def admit():
            nonlocal used, build_s
            tb = clock()
            while pending and pending[0].arrival <= clock() - t0 and used + device_bytes(pending[0]) <= self.budget:
                req = pending.pop(0)
                built.append([req, build_system(req)])
                used += device_bytes(req)
            build_s += clock() - tb

        try:
            while pending or active or built:
                for req, s in built:
                    batch.add(s.fluid, 0, req.steps)  # the device stops it after req.steps iterations
                    active[req.rid] = [req, s, req.steps]
                built.clear()
                max_res = max(max_res, len(active))
                if not active:
                    admit()
                    if not built and pending:  # idle until the next arrival
                        time.sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                    continue
                # the chunk ends when the first member finishes (or after
                # max_chunk iterations, so that arrivals join soon): no member
                # idles inside a chunk, and each is retired the moment it is done
                chunk = min(self.max_chunk, min(v[2] for v in active.values()))
                batch.run(chunk)
                admit()  # overlaps the chunk running on the device
                tw = clock()
                batch.sync()
                wait_s += clock() - tw
                runs += 1
                done = []
                for rid, v in active.items():
                    ran = min(chunk, v[2])
                    v[2] -= ran
                    work += v[0].cells * 25.0 * ran
                    if v[2] <= 0:
                        done.append(rid)
                for rid in done:
                    req, s, _ = active.pop(rid)
                    batch.remove(s.fluid)
                    if self.keep_results:
                        self.results[rid] = result_of(s)
                    s.close()
                    used -= device_bytes(req)
                    lat.append(clock() - t0 - req.arrival)
        finally:
            for v in active.values():
                batch.remove(v[1].fluid)
                v[1].close()
            for _, s in built:
                s.close()
            batch.close()
        return Stats(lat, clock() - t0, work, max_res, runs, build_s, wait_s)


def sequential(requests: List[Request], clock=time.perf_counter, keep_results: bool = False,
               storage: Optional[str] = "f32"):
    """The baseline: each request alone, one after another, with the plain FP32
    form (storage=None keeps each request's own storage), fused graph-captured
    iterations."""
    t0 = clock()
    work = 0.0
    results = {}
    durations = []
    for req in requests:
        ts = clock()
        s = build_system(req, storage=storage)
        s.fluid.run(0, req.steps)
        s.fluid.sync()
        if keep_results:
            results[req.rid] = result_of(s)
        s.close()
        durations.append(clock() - ts)
        work += req.cells * 25.0 * req.steps
    dt = clock() - t0
    return {"requests": len(requests), "seconds": round(dt, 3), "mlups": round(work / dt / 1e6, 1),
            "durations_s": durations}, results


def fifo(requests: List[Request], durations: List[float]) -> dict:
    """A one-at-a-time server on the same arrivals: request i starts when it has
    arrived and request i-1 is done, and takes durations[i] (its measured solve
    time, build included).  Makespan, p50/p99 latency, aggregate MLUPS."""
    t = 0.0
    lat = []
    work = 0.0
    for req, d in sorted(zip(requests, durations), key=lambda x: x[0].arrival):
        t = max(t, req.arrival) + d
        lat.append(t - req.arrival)
        work += req.cells * 25.0 * req.steps
    lat.sort()
    pct = lambda p: lat[min(len(lat) - 1, int(math.ceil(p / 100 * len(lat))) - 1)]  # noqa: E731
    return {"makespan_s": round(t, 3), "p50_latency_s": round(pct(50), 3), "p99_latency_s": round(pct(99), 3),
            "aggregate_mlups": round(work / t / 1e6, 1)}


def main():
    import argparse
    import json

    p = argparse.ArgumentParser(description="serving ensemble: continuous batching vs sequential plain solves")
    p.add_argument("--requests", type=int, default=256)
    p.add_argument("--rate", type=float, default=8.0, help="Poisson arrivals per second")
    p.add_argument("--step-scale", type=float, default=0.1, help="scales the 500-5000 requested iterations")
    p.add_argument("--budget-gb", type=float, default=150.0)
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--no-sequential", action="store_true")
    a = p.parse_args()
    reqs = make_requests(a.requests, a.rate, a.seed, a.step_scale)
    stats = Server(a.budget_gb * 1e9).serve(reqs).summary()
    line = {"metric": "serving aggregate MLUPS", "serving": stats,
            "config": {"requests": a.requests, "rate_per_s": a.rate, "step_scale": a.step_scale,
                       "sides": list(SIDES), "budget_gb": a.budget_gb, "seed": a.seed}}
    if not a.no_sequential:
        base, _ = sequential(reqs)
        seq = fifo(reqs, base.pop("durations_s"))
        line["sequential_plain_f32"] = base
        line["sequential_fifo"] = seq
        line["speedup_vs_sequential"] = round(seq["makespan_s"] / stats["makespan_s"], 2)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
