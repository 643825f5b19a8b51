"""Generate the golden fixtures from the reference's own CUDA kernels.

Runs on a machine with a GPU and a built oracle/_ref/libglsm_ref.so (the
reference's src/*.cu compiled for sm_100a by oracle/Makefile).  Writes
<outdir>/<case>.npz with the reference's outputs (float64 arrays) for every
case in cases.py.  Usage:

    python tests/golden/make_golden.py [outdir]     # default: tests/golden
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from cases import CASES, build, collect  # noqa: E402
from oracle.pyref import Reference  # noqa: E402


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(outdir, exist_ok=True)
    for name, c in CASES.items():
        sim = build(Reference, name)
        sim.run(0, c["iters"])
        data = collect(sim, name)
        sim.close()
        # float32 storage for the fluid-side (FP32 in the reference), float64 for the gel
        packed = {k: (v.astype(np.float32) if not k.startswith("g") else v) for k, v in data.items()}
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), **packed)
        print(name, {k: v.shape for k, v in data.items() if k in ("u", "pop", "lag")}, flush=True)


if __name__ == "__main__":
    main()
