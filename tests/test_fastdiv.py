"""The multiply-high division used for cell coordinates (csrc/fastdiv.h) is
exact: compiled for the host with g++ and checked against integer division."""
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r'''
#include <cstdio>
#include "fastdiv.h"
int main() {
    unsigned d, n; int bad = 0;
    while (scanf("%u %u", &d, &n) == 2) {
        glsm::FastDiv f = glsm::make_fastdiv(d);
        if (glsm::fdiv(n, f) != n / d) bad++;
    }
    printf("%d\n", bad);
    return 0;
}
'''


def test_fastdiv_exact():
    rng = np.random.default_rng(7)
    divs = [1, 2, 3, 7, 48, 101, 128, 192, 256, 384, 10201, 65536, 147456, 2304, 9409, 16384 + 1]
    pairs = []
    for d in divs:
        ns = np.concatenate([np.arange(0, 4096), rng.integers(0, 2**31, 4000), [2**31 - 1, 2**32 - 1,
                             d * 1000 - 1, d * 1000, d * 1000 + 1]])
        pairs += [(d, int(n)) for n in ns]
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "t.cpp")
        exe = os.path.join(td, "t")
        open(src, "w").write(DRIVER)
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "glsm_fluid_3d_b200", "csrc"),
                               src, "-o", exe])
        out = subprocess.run([exe], input="\n".join(f"{d} {n}" for d, n in pairs), capture_output=True,
                             text=True, check=True).stdout
    assert int(out.strip()) == 0
