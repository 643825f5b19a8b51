"""The C++ drop-in classes (include/glsm/{gel,coupling,fluid}.h): drivers written
against the reference's Gel / Coupler / Fluid compile unchanged and run.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _reference_sim():
    """The reference's src/sim.cpp where the reference is mounted: GLSM_REF_SRC,
    else the directory the oracle build recorded in oracle/_ref/ref_src."""
    d = os.environ.get("GLSM_REF_SRC")
    rec = os.path.join(ROOT, "oracle", "_ref", "ref_src")
    if not d and os.path.exists(rec):
        d = open(rec).read().strip()
    return os.path.join(d, "sim.cpp") if d else ""


REF_SIM = _reference_sim()


def compile_driver(src, exe):
    from glsm_fluid_3d_b200 import build

    build.build()
    libdir = os.path.join(ROOT, "glsm_fluid_3d_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include", "glsm"), "-I", os.path.join(CUDA, "include"),
           src, "-o", exe, "-L", libdir, "-lglsm_b200", f"-Wl,-rpath,{libdir}", "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    subprocess.check_call(cmd)


def test_example_driver_compiles(tmp_path):
    compile_driver(os.path.join(ROOT, "tests", "drivers", "sim_twogels.cpp"), str(tmp_path / "sim"))


@pytest.mark.skipif(not os.path.exists(REF_SIM), reason="reference sources not mounted here")
def test_reference_sim_cpp_compiles_unchanged(tmp_path):
    """The reference's own src/sim.cpp compiles and links against the drop-in headers."""
    compile_driver(REF_SIM, str(tmp_path / "sim_ref"))


@pytest.mark.gpu
def test_write_files_does_not_wait_for_the_device(gpu, tmp_path):
    """Gel::writeFiles / Fluid::writeFiles return while the device still works
    through 300 queued iterations of the 101^3 workload (an output snapshot
    instead of a synchronous copy), and the files they write equal those of the
    synchronous copyDataToHost + recordData of the same state."""
    exe = str(tmp_path / "dat_async")
    compile_driver(os.path.join(ROOT, "tests", "drivers", "dat_async.cpp"), exe)
    env = dict(os.environ)
    env.pop("IBM_BETA", None)
    env.pop("IBM_RAMP_STEPS", None)
    d = tmp_path / "out"
    out = subprocess.run([exe, str(d)], capture_output=True, text=True, env=env, check=True).stdout
    t = {k: float(v) for k, v in re.findall(r"(\w+_ms)=([\d.]+)", out)}
    print(out.strip())
    assert "N=1030301" in out
    # the device had most of the 300 iterations (~0.6 ms each) still to run
    # when the calls returned
    assert t["drain_ms"] > 60.0, t
    assert t["writefiles_ms"] < 0.25 * t["drain_ms"], t
    for name in ["gel1rn", "gel1Fn", "gel1Veln", "gel1rm", "gel1um", "gel1vm", "gel1wm", "gel2rn", "gel2um",
                 "Velb", "Conc"]:
        assert open(d / f"{name}2.dat").read() == open(d / f"{name}3.dat").read(), name


@pytest.mark.gpu
def test_driver_matches_python_path(gpu, tmp_path):
    """The C++ driver and the Python per-method loop give the same gel state and
    the same .dat contents after 20 iterations."""
    from glsm_fluid_3d_b200 import System

    exe = str(tmp_path / "sim")
    compile_driver(os.path.join(ROOT, "tests", "drivers", "sim_twogels.cpp"), exe)
    env = dict(os.environ)
    env.pop("IBM_BETA", None)
    env.pop("IBM_RAMP_STEPS", None)
    out = subprocess.run([exe, "20", str(tmp_path / "data")], capture_output=True, text=True, env=env, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("iter=")]
    assert lines and "Nsub=25" in lines[0] and "h=0.5" in lines[0]
    vmax_cpp = float(re.search(r"Vg_max=(\S+)", lines[-1]).group(1))
    assert os.path.exists(tmp_path / "data" / "gel1um0.dat") and os.path.exists(tmp_path / "data" / "Velb0.dat")

    s = System(41, 21, 21, nsub=25, methods=True)
    s.add_gel((6, 6, 6), (6.0, 5.0, 5.0), 1, 1)
    s.add_gel((6, 6, 6), (14.0, 5.0, 5.0), 1, 2)
    s.finalize()
    s.run(0, 21)
    vmax_py = max(np.sqrt((s.gels[k].read("Veln").reshape(-1, 3) ** 2).sum(1)).max() for k in range(2))
    s.close()
    assert abs(vmax_cpp - vmax_py) <= 1e-9 * max(vmax_py, 1e-30)
    # the .dat format of the reference: right-aligned "%f" fields, six spaces apart
    first = open(tmp_path / "data" / "gel1rn0.dat").readline()
    assert re.fullmatch(r"\s*-?\d+\.\d{6} {6}\s*-?\d+\.\d{6} {6}\s*-?\d+\.\d{6}\n", first)
