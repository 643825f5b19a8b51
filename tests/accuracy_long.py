"""Long-horizon accuracy of the CUDA path against the FP64 oracle.

Runs the bench workload (101^3, two 6^3 gels as in sim.cpp, Nsub = 25, seed
12345, noise 1e-3; --workload P: 256^3 with eight 6^3 gels) and saves checkpoints of u, c1 and every gel's node
positions and chemistry, plus the centre-element vm trace every 10 steps.

    python tests/accuracy_long.py oracle --out DIR [--steps 1000,5000,10000]
    python tests/accuracy_long.py gpu --storage f32|f16|bf16 --out DIR [--steps ...]
    python tests/accuracy_long.py compare --ref DIR --got DIR

Errors reported: relative L2 of u, c1, gel displacement rn - rn(0) and the
centre-element vm trace (the BZ phase signal of tools/analyze_phase.py), plus
absolute max errors.  The oracle is test infrastructure; this script only
compares.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

DIMS = (101, 101, 101)
NSUB = 25
GELS = [((6, 6, 6), (16.67, 25.0, 25.0)), ((6, 6, 6), (33.33, 25.0, 25.0))]
# the workloads: D (the reference's default, above) and P (256^3, eight 6^3 gels
# in a 2x2x2 block 40 cells apart, box-centred)
WORKLOADS = {
    "D": (DIMS, GELS),
    "P": ((256, 256, 256), [((6, 6, 6), (63.75 + dx, 63.75 + dy, 63.75 + dz))
                            for dz in (-10.0, 10.0) for dy in (-10.0, 10.0) for dx in (-10.0, 10.0)]),
}
SEED, AMP = 12345, 1e-3
TRACE_EVERY = 10


def center_slot(LX, LY, LZ):
    return (LX // 2) + (LX + 1) * ((LY // 2) + (LY + 1) * (LZ // 2))


def run(backend, out, steps, storage="f32", workload="D"):
    os.makedirs(out, exist_ok=True)
    dims, gels = WORKLOADS[workload]
    if backend == "oracle":
        from oracle.pyoracle import Oracle

        sim = Oracle(*dims, nsub=NSUB)
    else:
        from glsm_fluid_3d_b200 import System

        sim = System(*dims, nsub=NSUB, storage=storage)
    for k, (size, pos) in enumerate(gels):
        sim.add_gel(size, pos, 1, k + 1)
        sim.gel_noise(k, SEED, AMP)
    sim.finalize()
    L = size[0] + 1
    cslot = center_slot(L, L, L)
    rn0 = [sim.get(20, g) for g in range(len(gels))]
    trace = []
    it, t0 = 0, time.time()
    for target in steps:
        while it < target:
            n = min(TRACE_EVERY - it % TRACE_EVERY, target - it)
            sim.run(it, n)
            it += n
            if it % TRACE_EVERY == 0:
                trace.append([it] + [float(sim.get(25, g)[cslot]) for g in range(len(gels))])
        data = {"u": sim.get(2).astype(np.float32), "c1": sim.get(3).astype(np.float32)}
        for g in range(len(gels)):
            data[f"g{g}_disp"] = sim.get(20, g) - rn0[g]
            data[f"g{g}_um"] = sim.get(24, g)
            data[f"g{g}_vm"] = sim.get(25, g)
        np.savez_compressed(os.path.join(out, f"ckpt_{target}.npz"), **data)
        np.save(os.path.join(out, "trace.npy"), np.array(trace))
        print(f"{backend} {storage} step {target} saved after {time.time() - t0:.0f} s", flush=True)


def compare(ref, got):
    res = {}
    for f in sorted(os.listdir(got)):
        if not f.startswith("ckpt_"):
            continue
        step = int(f[5:-4])
        a, b = np.load(os.path.join(got, f)), np.load(os.path.join(ref, f))
        row = {}
        for k in b.files:
            x, y = a[k].astype(np.float64), b[k].astype(np.float64)
            den = np.linalg.norm(y)
            row[k] = {"rel_l2": float(np.linalg.norm(x - y) / den) if den else float(np.linalg.norm(x - y)),
                      "max_abs": float(np.abs(x - y).max()), "scale": float(np.abs(y).max())}
        res[step] = row
    ta, tb = np.load(os.path.join(got, "trace.npy")), np.load(os.path.join(ref, "trace.npy"))
    n = min(len(ta), len(tb))
    x, y = ta[:n, 1:], tb[:n, 1:]
    res["vm_trace"] = {"steps": int(ta[n - 1, 0]) if n else 0,
                       "rel_l2": float(np.linalg.norm(x - y) / np.linalg.norm(y)), "max_abs": float(np.abs(x - y).max())}
    return res


def main():
    p = argparse.ArgumentParser()
    p.add_argument("mode", choices=["oracle", "gpu", "compare"])
    p.add_argument("--out")
    p.add_argument("--ref")
    p.add_argument("--got")
    p.add_argument("--storage", default="f32")
    p.add_argument("--steps", default="1000,5000,10000")
    p.add_argument("--threads", type=int, default=0)
    p.add_argument("--workload", default="D", choices=sorted(WORKLOADS))
    a = p.parse_args()
    steps = [int(s) for s in a.steps.split(",")]
    if a.mode == "compare":
        print(json.dumps(compare(a.ref, a.got)))
        return
    if a.mode == "oracle" and a.threads:
        from oracle import pyoracle

        pyoracle.threads(a.threads)
    run(a.mode, a.out, steps, a.storage, a.workload)


if __name__ == "__main__":
    main()
