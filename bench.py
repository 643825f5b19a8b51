#!/usr/bin/env python
"""Coupled MLUPS of the gel-fluid step on B200.

Workload (the reference's default configuration): a 101x101x101 D3Q19 lattice,
two 6x6x6-element gels at (16.67, 25, 25) and (33.33, 25, 25) in physical units
(the relative layout of src/sim.cpp:26-30), Nsub = 25 LBM substeps per gel
step, seeded chemistry noise.  One "step" is one coupled iteration (gels, marker
pack, 25 IBM+LBM substeps, concentration, repulsion, scatter).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f32|f16|bf16]
    python bench.py --impl reference      # the reference's own CUDA kernels

Prints one JSON line.  Multi-GPU runs are independent replicas (one per rank,
launched by torch.distributed.run); the job time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED, AMP = 12345, 1e-3


def _rods():
    """6 x 6 rods of 4x4x12 elements on a 32-unit pitch (the x/y period of the
    384x384 lattice), standing on the z = 0 wall, anchored below z = 1.5 and
    quiescent until a seeded delay uniform in [0, 49150) (as in
    src/sim_array.cpp:42-51, which fires each gel's pulse at its delay)."""
    import random

    rng = random.Random(SEED)
    gels = []
    for iy in range(6):
        for ix in range(6):
            gels.append(dict(size=(4, 4, 12), pos=(16.0 + 32.0 * ix, 16.0 + 32.0 * iy, 7.5), anchor=1.5,
                             delay=int(rng.random() * 49150)))
    return gels


# the measured workloads; "D" (the reference's default configuration) is the headline
WORKLOADS = {
    "D": dict(dims=(101, 101, 101), nsub=25, periodic=(0, 0, 0),
              gels=[dict(size=(6, 6, 6), pos=(16.67, 25.0, 25.0)), dict(size=(6, 6, 6), pos=(33.33, 25.0, 25.0))],
              desc="101^3 D3Q19 lattice, two 6x6x6-element gels as in sim.cpp, Nsub=25, coupled step "
                   "(gel mechanics+BZ chemistry, IBM, LBM, concentration)"),
    "S": dict(dims=(48, 48, 48), nsub=2, periodic=(0, 0, 0),
              gels=[dict(size=(6, 6, 6), pos=(11.75, 11.75, 11.75))],
              desc="48^3 D3Q19 lattice, one centred 6x6x6-element gel, Nsub=2, coupled step"),
    "P": dict(dims=(256, 256, 256), nsub=25, periodic=(0, 0, 0),
              gels=[dict(size=(6, 6, 6), pos=(63.75 + dx, 63.75 + dy, 63.75 + dz))
                    for dz in (-10.0, 10.0) for dy in (-10.0, 10.0) for dx in (-10.0, 10.0)],
              desc="256^3 D3Q19 lattice, eight 6x6x6-element gels in a 2x2x2 block 40 cells apart, Nsub=25, "
                   "coupled step"),
    "L": dict(dims=(384, 384, 192), nsub=3, periodic=(1, 1, 0), gels=_rods(),
              desc="384x384x192 D3Q19 lattice periodic in x and y, 36 anchored 4x4x12-element rods on the "
                   "z = 0 wall with seeded activation delays, Nsub=3, coupled step"),
}
W = WORKLOADS["D"]
DIMS, NSUB = W["dims"], W["nsub"]
BYTES_PER_CELL = {"f32": 152, "f16": 76, "bf16": 76, "f16c": 76, "f16c2": 76}  # one read + one write of 19 populations
FLUSH_BYTES = 256 << 20  # > the 126 MB L2
L2_PROBE_BYTES = 24 << 20  # two buffers: a 48 MiB footprint, inside the 126 MB L2
L2_PROBE_REPS = 400


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f16c", "f16c2"],
                   help="f16c / f16c2: FP16 storage with the mass- and momentum-conserving rounding on every / "
                        "every second substep")
    p.add_argument("--workload", default="D", choices=sorted(WORKLOADS),
                   help="D: 101^3 two gels (default); S: 48^3 one gel; P: 256^3 eight gels; L: 384x384x192 rods")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-l2-persisting", action="store_true",
                   help="leave the population array's L2 access-policy window off")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    p.add_argument("--no-f16", action="store_true", help="skip the FP16 forms' sub-object")
    p.add_argument("--f16-steps", type=int, default=300, help="timed steps of each FP16 form")
    p.add_argument("--no-serving", action="store_true", help="skip the serving sub-object")
    p.add_argument("--serving-requests", type=int, default=64)
    p.add_argument("--serving-step-scale", type=float, default=0.1)
    return p.parse_args()


def select(name):
    """Make `name` the workload of this run."""
    global W, DIMS, NSUB
    W = WORKLOADS[name]
    DIMS, NSUB = W["dims"], W["nsub"]


def workload_desc(storage):
    return {
        "workload": W["desc"], "lattice": list(DIMS), "gels": len(W["gels"]),
        "gel_elements": sorted({tuple(g["size"]) for g in W["gels"]}), "nsub": NSUB,
        "periodic": list(W["periodic"]), "storage": storage,
        "parallelism": "replicas (one independent system per GPU)",
        "l2": "persisting L2 lines released and a 256 MiB buffer written between timed steps",
    }


def configure(sim):
    """Gels, seeded chemistry noise, anchors and activation delays of the workload."""
    for k, g in enumerate(W["gels"]):
        sim.add_gel(g["size"], g["pos"], 1, k + 1)
    for k, g in enumerate(W["gels"]):
        sim.gel_noise(k, SEED, AMP)
        if "anchor" in g:
            sim.set_anchor(k, g["anchor"])
        if g.get("delay", 0) > 0:
            sim.reset_quiescent(k)
            sim.set_active_from(k, g["delay"])
    sim.set_params(beta=1.0, ramp_steps=20000.0, periodic=W["periodic"])
    sim.finalize()
    return sim


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def ncu_traffic(storage):
    """DRAM bytes per substep launch from the committed ncu summary of this
    workload and storage, if present."""
    path = os.path.join(ROOT, "profiles", f"lbm_substep_{storage}_{DIMS[0]}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi samples; stats are taken over the samples inside [t0, t1]."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.index), "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self, t0, t1):
        import datetime

        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[2]), float(parts[3]), float(parts[4]),
                             {n for n, v in zip(names, parts[6:10]) if v.lower().startswith("active")}))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        inside = [r for r in rows if t0 - 0.05 <= r[0] <= t1 + 0.05]
        if not inside:  # region shorter than the sampling interval: the samples around it
            inside = sorted(rows, key=lambda r: min(abs(r[0] - t0), abs(r[0] - t1)))[:2]
        sm = [r[1] for r in inside]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[2] for r in inside),
                "power_w_max": max(r[3] for r in inside),
                "reasons": sorted(set().union(*[r[4] for r in inside])), "samples": len(inside)}


def max_over_ranks(value, world, device):
    """The job time of a replicated run: the largest of the ranks' times (every
    rank calls this with its own; NCCL on GPUs, any backend that has MAX)."""
    if world <= 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_value(cells, nsub, steps, world, t_seconds):
    """Whole-job MLUPS of `world` replicas, each advancing `cells` x `nsub` cell
    updates per step for `steps` steps, over the job time."""
    return world * cells * nsub * steps / t_seconds / 1e6


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_system(storage):
    from glsm_fluid_3d_b200 import System

    return configure(System(*DIMS, nsub=NSUB, storage=storage))


def cpu_baseline(budget_s):
    """The FP64 oracle (OpenMP over all host cores) on a bounded sample of the workload."""
    from oracle import pyoracle

    cores = pyoracle.threads(os.cpu_count() or 1)
    o = configure(pyoracle.Oracle(*DIMS, nsub=NSUB))
    o.run(0, 1)  # warm-up
    n, t0 = 0, time.perf_counter()
    while n < 20:
        o.run(1 + n, 1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    cells = DIMS[0] * DIMS[1] * DIMS[2]
    return {"value": round(cells * NSUB * n / dt / 1e6, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
            "sample": f"{n} coupled iterations of the same workload after 1 warm-up, FP64 oracle "
                      f"(oracle/glsm_oracle.cpp, OpenMP), {dt:.1f} s"}


def barrier(world):
    """All ranks here and the device idle."""
    import torch

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()


def timed_steps(s, K, warmup, world, it0=0):
    """K coupled iterations of system s, each between CUDA events on the system
    stream, with the persisting L2 lines released and L2 flushed before each;
    returns (total device ms over the K steps, next iteration, clock stats)."""
    import torch

    from glsm_fluid_3d_b200 import l2_reset_persisting

    fluid = s.fluid
    stream = torch.cuda.ExternalStream(s.coupler.stream())
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    it = it0
    for _ in range(warmup):
        fluid.run(it, 1)
        it += 1
    fluid.sync()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)  # let the sampler settle
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    barrier(world)
    t_wall0 = time.time()
    for k in range(K):
        # between timed steps: the previous step done, its persisting L2 lines
        # (the population array's access-policy window) released, L2 flushed
        stream.synchronize()
        l2_reset_persisting()
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[k][0].record(stream)
            fluid.run(it, 1)
            ev[k][1].record(stream)
        it += 1
    stream.synchronize()
    barrier(world)
    clk = clocks.stop(t_wall0, time.time())
    fluid.sync()
    return sum(a.elapsed_time(b) for a, b in ev), it, clk


def pattern_peak(storage):
    """The substep kernel's access pattern without the collision on this
    workload's lattice and element size (glsm_pattern_bandwidth): the even and
    odd forms' GB/s and their harmonic mean (the substeps alternate)."""
    from glsm_fluid_3d_b200 import pattern_bandwidth

    ge, go = pattern_bandwidth(DIMS, "f32" if storage == "f32" else "f16", 20)
    return {"even": round(ge, 1), "odd": round(go, 1), "mean": round(2.0 / (1.0 / ge + 1.0 / go), 1)}


def substep_roofline(s, storage, it, l2, pattern=None):
    """Achieved bandwidth of the substep kernel: graphs of one and of two velocity
    steps (nsub and 2 nsub substep launches) timed with one event pair each on
    the system stream; their difference over nsub is the launch time without
    the graph's launch overhead.  Returns (roofline dict, next iteration)."""
    import statistics as st

    fluid = s.fluid
    one, two, prof = [], [], []
    for rep in range(9):
        if rep < 6:
            n = 1 + rep % 2
            t = fluid.profile_substeps(it, n_steps=n)
            (one if n == 1 else two).append(t)
        else:
            n = 1
            prof.extend(fluid.profile_velocity(it).tolist())
        for j in range(n):  # keep the state consistent for what follows
            s.coupler.packFromGels()
            fluid.stepConcentration(it + j)
        it += n
    fluid.sync()
    avg_ms = (st.median(two) - st.median(one)) / NSUB
    N = DIMS[0] * DIMS[1] * DIMS[2]
    bpc = BYTES_PER_CELL[storage]
    achieved = bpc * N / (avg_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": ncu_traffic(storage), "peak_kind": peak_kind,
            "l2_peak": round(l2, 1), "frac_l2": round(achieved / l2, 4),
            "l2_peak_how": f"glsm_copy_bandwidth: 2 x {L2_PROBE_BYTES >> 20} MiB copied back and forth "
                           f"{L2_PROBE_REPS} times in one launch, L1 bypassed (measured in this run)",
            "pattern_peak": pattern["mean"] if pattern else None,
            "frac_pattern": round(achieved / pattern["mean"], 4) if pattern else None,
            "pattern_peak_how": ("glsm_pattern_bandwidth: the substep's 19-plane in-place read and write without the "
                                 f"collision on this lattice, even {pattern['even']} / odd {pattern['odd']} GB/s, "
                                 "harmonic mean (measured in this run, no L2 window)") if pattern else None,
            "kernel": "lbm_substep_kernel", "bytes_per_launch": bpc * N, "avg_launch_ms": round(avg_ms, 5),
            "avg_launch_ms_one_graph": round(st.median(one) / NSUB, 5),
            "avg_launch_ms_event_pairs": round(st.mean(prof), 5),
            "timing": f"graphs of {NSUB} and {2 * NSUB} substep launches (one and two velocity steps), 3 each, "
                      f"one event pair around each graph: (median 2-step - median 1-step) / {NSUB}",
            "note": "algorithmic bytes = one read + one write of 19 populations per cell; the 78 MB population "
                    "array of 101^3 fits in L2, so achieved can exceed the HBM copy peak"}
    return roof, it


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    # one population copy of 101^3 (78 MB FP32, 39 MB FP16) fits in L2: the
    # achieved bandwidth is also set against a measured L2 copy bandwidth,
    # taken before the system reserves its persisting part of L2
    from glsm_fluid_3d_b200 import copy_bandwidth

    l2 = copy_bandwidth(L2_PROBE_BYTES, L2_PROBE_REPS)
    pattern = pattern_peak(args.storage)
    s = make_system(args.storage)
    fluid = s.fluid
    fluid.set_l2_persisting(not args.no_l2_persisting)  # one system alone on the GPU
    K = args.steps
    t_ms, it, clk = timed_steps(s, K, args.warmup, world)
    t_ms = max_over_ranks(t_ms, world, "cuda")
    N = DIMS[0] * DIMS[1] * DIMS[2]
    value = job_value(N, NSUB, K, world, t_ms / 1e3)

    # dominant kernel: the substep kernel, timed as it runs inside the fused
    # iteration (graphs of its launches on the system stream)
    roof, it = substep_roofline(s, args.storage, it, l2, pattern)

    # end to end through the C ABI with host buffers: restart the state from
    # pinned host memory, run K iterations transferring the gels' node velocities
    # to the host every step (the reference driver's observable; an output
    # snapshot per step, so the next step is queued without waiting for the
    # transfer), read u and c back at the end
    e2e = None
    if not args.no_e2e:
        pin = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()  # noqa: E731
        gels = s.gels
        host_rn = [pin(g.nN * 3, torch.float64) for g in gels]
        host_um = [pin(g.nE, torch.float64) for g in gels]
        host_vm = [pin(g.nE, torch.float64) for g in gels]
        host_vel = [[pin(g.nN * 3, torch.float64) for _ in range(2)] for g in gels]  # alternate steps
        host_u = pin(3 * N, torch.float32)
        host_c = pin(N, torch.float32)
        for g, a, b, c in zip(gels, host_rn, host_um, host_vm):
            a[:] = g.read("rn")
            b[:] = g.read("um")
            c[:] = g.read("vm")
        fluid.read_into("u", host_u)
        fluid.read_into("c1", host_c)
        h2d = sum(a.nbytes + b.nbytes + c.nbytes for a, b, c in zip(host_rn, host_um, host_vm)) + host_u.nbytes + \
            host_c.nbytes
        d2h = K * sum(v[0].nbytes for v in host_vel) + host_u.nbytes + host_c.nbytes
        barrier(world)
        t0 = time.perf_counter()
        for g, a, b, c in zip(gels, host_rn, host_um, host_vm):
            g.write("rn", a)
            g.write("um", b)
            g.write("vm", c)
        fluid.write("u", host_u)
        fluid.write("c1", host_c)
        for k in range(K):
            fluid.run(it, 1)
            it += 1
            for g, v in zip(gels, host_vel):
                g.snapshot(["Veln"], [v[k % 2]])
        for g in gels:
            g.snapshot_wait()
        fluid.read_into("u", host_u)
        fluid.read_into("c1", host_c)
        barrier(world)
        t_e2e = max_over_ranks(time.perf_counter() - t0, world, "cuda")
        e2e = {"value": round(job_value(N, NSUB, K, world, t_e2e), 1), "unit": "MLUPS",
               "h2d_bytes_per_step": int(h2d / K), "d2h_bytes_per_step": int(d2h / K),
               "timing": "host wall clock around the whole job, device synchronised at both ends",
               "job": "restart of gel chemistry/positions and u, c from pinned host memory (H2D), K fused "
                      "iterations via glsm_fluid_run with every gel's Veln transferred to pinned host memory "
                      "each step (glsm_gel_snapshot, D2H on a copy stream), final u and c read back (D2H); "
                      "bytes are totals divided by K"}
        assert np.isfinite(host_u).all()
        assert all(np.isfinite(v[(K - 1) % 2]).all() for v in host_vel)  # (zero for gels not yet active)

    s.close()
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(args.cpu_seconds)
    f16 = None
    if world == 1 and args.storage == "f32" and not args.no_f16:
        f16 = f16_forms(args, value, l2)
    serve = None
    if world == 1 and args.workload == "D" and not args.no_serving:
        serve = serving_summary(args)

    # gel, concentration markers, repulsion, the substeps, conv-diff (the iteration
    # counter is set only at the first run call: the timed steps continue the warm-up)
    launches_per_step = 1 + 1 + 1 + NSUB + 1
    line = {
        "metric": "coupled MLUPS", "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(t_ms / K, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.storage, "data": "synthetic (seeded gel chemistry noise, fluid at rest)",
        "config": workload_desc(args.storage), "l2_persisting": not args.no_l2_persisting,
        "roofline": roof, "cpu_baseline": base, "e2e": e2e,
        "clocks": clk, "gpu_launches": launches_per_step * K,
    }
    if f16 is not None:
        line["f16"] = f16
    if serve is not None:
        line["serving"] = serve
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def f16_forms(args, f32_value, l2):
    """The FP16-storage forms on the same workload and timing method, with fewer
    timed steps: nearest rounding and the conserving rounding (the form that
    keeps the 10,000-iteration velocity error within 1e-3)."""
    out = {}
    N = DIMS[0] * DIMS[1] * DIMS[2]
    K = max(1, min(args.steps, args.f16_steps))
    pattern = pattern_peak("f16")
    for storage in ("f16", "f16c"):
        s = make_system(storage)
        s.fluid.set_l2_persisting(not args.no_l2_persisting)
        t_ms, it, clk = timed_steps(s, K, args.warmup, 1)
        roof, it = substep_roofline(s, storage, it, l2, pattern)
        s.close()
        v = job_value(N, NSUB, K, 1, t_ms / 1e3)
        out[storage] = {"value": round(v, 1), "unit": "MLUPS", "steps": K, "ms_per_step": round(t_ms / K, 4),
                        "vs_f32": round(v / f32_value, 3),
                        "roofline": {k: roof[k] for k in ("achieved", "peak", "unit", "frac", "l2_peak", "frac_l2",
                                                          "pattern_peak", "frac_pattern", "bytes_per_launch",
                                                          "avg_launch_ms", "traffic")},
                        "clocks": clk}
    out["note"] = ("FP16 deviations f_q - w_q scaled by 2^20, FP32 collision; f16 rounds to nearest, f16c with the "
                   "mass- and momentum-conserving rounding; same workload, L2 flush and timing as the headline")
    return out


def serving_summary(args):
    """A short run of the serving ensemble (continuous batching with HBM-budget
    admission) beside the same requests run one after another with the plain
    FP32 form: aggregate MLUPS, p50/p99 completion latency, speed-up."""
    from glsm_fluid_3d_b200 import serving

    import dataclasses

    reqs = serving.make_requests(args.serving_requests, 8.0, 2024, args.serving_step_scale)
    stats = serving.Server(150e9).serve(reqs).summary()
    at_once = [dataclasses.replace(r, arrival=0.0) for r in reqs]
    sat = serving.Server(150e9).serve(at_once).summary()
    base, _ = serving.sequential(reqs)
    seq = serving.fifo(reqs, base["durations_s"])
    return {"aggregate_mlups": stats["aggregate_mlups"], "p50_latency_s": stats["p50_latency_s"],
            "p99_latency_s": stats["p99_latency_s"], "makespan_s": stats["makespan_s"],
            "max_resident_systems": stats["max_resident_systems"],
            "sequential_fifo": seq,
            "speedup_vs_sequential": round(seq["makespan_s"] / stats["makespan_s"], 3),
            "saturated": {"makespan_s": sat["makespan_s"], "aggregate_mlups": sat["aggregate_mlups"],
                          "max_resident_systems": sat["max_resident_systems"],
                          "sequential_plain_f32_s": base["seconds"], "sequential_plain_f32_mlups": base["mlups"],
                          "speedup_vs_sequential": round(base["seconds"] / sat["makespan_s"], 3)},
            "requests": len(reqs),
            "config": {"arrivals": "seeded Poisson, 8 per second; saturated: all at t = 0",
                       "sequential": "the same requests one at a time with the plain FP32 form, each solve's "
                                     "measured time (build included) replayed as a FIFO server on the same "
                                     "arrivals", "sides": list(serving.SIDES),
                       "gels": "1-4 of 4-8 elements", "steps": f"500-5000 x {args.serving_step_scale}",
                       "storage": "FP32 / FP16 half and half", "budget_gb": 150}}


def run_reference(args, world, rank, local):
    """The reference's own CUDA kernels (src/*.cu built unmodified for sm_100a)."""
    if rank != 0:
        return
    import torch

    from oracle import pyref

    if not pyref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libglsm_ref.so was not built "
                                                                "(the reference sources were absent at build time)"}))
        return
    torch.cuda.set_device(local)
    if any(W["periodic"]):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no periodic boundaries "
                                                                "(this workload's x/y periodicity is an extension)"}))
        return
    r = pyref.Reference(*DIMS, nsub=NSUB)
    for k, g in enumerate(W["gels"]):
        r.add_gel(g["size"], g["pos"], 1, k + 1)
    for k, g in enumerate(W["gels"]):
        r.gel_noise(k, SEED, AMP)
    r.set_params(beta=1.0, ramp_steps=20000.0)
    r.finalize()
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    it = 0
    r.time(it, args.warmup)
    it += args.warmup
    K = min(args.steps, 300)  # the reference is ~8 ms per step
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    t_wall0 = time.time()
    t_ms = 0.0
    for _ in range(K):
        flush.zero_()  # legacy default stream: ordered with the reference's streams
        t_ms += r.time(it, 1)
        it += 1
    torch.cuda.synchronize()
    clk = clocks.stop(t_wall0, time.time())
    r.close()
    N = DIMS[0] * DIMS[1] * DIMS[2]
    value = N * NSUB * K / (t_ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": "coupled MLUPS", "value": round(value, 1), "unit": "MLUPS",
        "n_gpus": world, "n_gpus_used": 1, "steps": K, "warmup": args.warmup, "ms_per_step": round(t_ms / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded gel chemistry noise, fluid at rest)", "config": workload_desc("f32"),
        "cpu_baseline": {"value": round(value, 1), "unit": "MLUPS", "cores": None, "kind": "reference",
                         "device": "cuda:0",
                         "sample": f"{K} coupled iterations of the reference's CUDA kernels (its only "
                                   f"implementation; oracle/_ref) in the stock call order of src/sim.cpp"},
        "e2e": {"value": round(value, 1), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    select(args.workload)
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
