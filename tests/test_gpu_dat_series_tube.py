"""The reference-facing outputs and scenario features, against the reference's
own CUDA build and the FP64 oracle:

* .dat files: the drop-in classes' Gel::writeFiles / Fluid::writeFiles
  (csrc/dropin.cpp) and the reference's (src/gel.cu:452-553,
  src/fluid.cu:115-150) on the same seeded case hold the same numbers, line
  for line, in the same text layout;
* text restart: the drop-in constructors with a start time read those files
  back (setGoonValue, src/gel.cu:221-282, src/fluid.cu:57-83) and write them
  out again unchanged, and the reference's own constructors restart from the
  files the drop-in wrote;
* centre-element series (Gel::recordCenter, src/gel.cu:706-712,
  src/gel_kernels.cu:823-835): the records at iterations 0, 1000 and 2000;
* tube mask (Gel::buildTubeMask, src/gel.cu:811-867; isVoidElement,
  src/gel_kernels.cu:104-117): square and cylindrical tubes over 30
  iterations.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from cases import build, collect
from oracle import pyoracle, pyref
from parity import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NUM = re.compile(r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?|-?nan|-?inf")

# the drivers' case (tests/drivers/dat_case.cpp): one gel in a 21^3 lattice,
# fluidSize 10 (h = 0.5), the stock Nsub of that lattice
DAT_CASE = dict(dims=(21, 21, 21), nsub=25, beta=1.0, ramp=0.0, seed=12345, amp=1e-3,
                gels=[dict(size=(6, 6, 6), pos=(4.75, 5.0, 5.25), type=1)])
DAT_ITERS = 40
GEL_FILES = ["rn", "Fn", "Veln", "rm", "um", "vm", "wm"]


def _need_reference():
    if not pyref.available():
        pytest.fail("oracle/_ref/libglsm_ref.so missing: the reference build travels with the repository")


def _driver(tmp_path):
    from test_dropin_cpp import compile_driver

    exe = str(tmp_path / "dat_case")
    compile_driver(os.path.join(ROOT, "tests", "drivers", "dat_case.cpp"), exe)
    return exe


def _env():
    env = dict(os.environ)
    env.pop("IBM_BETA", None)
    env["IBM_RAMP_STEPS"] = "0"
    return env


def _numbers(path):
    """(fields per line, numbers) of a .dat file.  Field widths are not compared
    here: a value's sign changes its padding, and round-off-sized values (u of
    order 1e-8) may change sign between two correct runs; the padding itself is
    checked in test_dropin_cpp.py."""
    skel, nums = [], []
    with open(path) as f:
        for line in f:
            found = NUM.findall(line)
            skel.append(len(found))
            nums.extend(float(x) for x in found)
    return skel, np.array(nums)


def _dat_names(t):
    return [f"gel1{k}{t}.dat" for k in GEL_FILES] + [f"Velb{t}.dat", f"Conc{t}.dat"]


def _reference_writes(dirpath):
    """The reference build runs the drivers' case and writes its .dat files at
    time 2 (iteration 2000) into dirpath."""
    cwd = os.getcwd()
    os.makedirs(dirpath, exist_ok=True)
    os.chdir(dirpath)
    try:
        r = build(pyref.Reference, DAT_CASE)
        r.run(0, DAT_ITERS)
        r.write_files(2000)
        r.close()
    finally:
        os.chdir(cwd)


def test_dat_files_match_the_reference_writer(gpu, tmp_path):
    _need_reference()
    exe = _driver(tmp_path)
    ours, theirs = tmp_path / "ours", tmp_path / "ref"
    out = subprocess.run([exe, "write", str(ours), str(DAT_ITERS), str(DAT_CASE["seed"])], env=_env(),
                         capture_output=True, text=True, check=True)
    assert "Nsub=25" in out.stdout, out.stdout
    _reference_writes(str(theirs))
    for name in _dat_names(2):
        sa, a = _numbers(ours / name)
        sb, b = _numbers(theirs / name)
        assert len(sa) == len(sb) and len(sa) > 0, name
        assert sa == sb, f"{name}: text layout differs"
        # six printed decimals (%f) or six significant digits (vm, wm): the two
        # agree to the last printed digit up to a rounding-boundary flip
        tol = 1e-5 * np.abs(b) + 1.5e-6 if ("vm" in name or "wm" in name) else 1.5e-6
        bad = np.abs(a - b) > tol
        print(f"{name}: {len(sa)} lines, max |diff| {np.abs(a - b).max():.2e}, {int(bad.sum())} beyond tolerance")
        assert not bad.any(), name


def test_text_restart_round_trip(gpu, tmp_path):
    """The drop-in restart reads its own files and writes them back unchanged;
    the reference's constructors restart from the same files to the same values."""
    _need_reference()
    exe = _driver(tmp_path)
    d = tmp_path / "run"
    subprocess.run([exe, "write", str(d), str(DAT_ITERS), str(DAT_CASE["seed"])], env=_env(), check=True,
                   capture_output=True)
    subprocess.run([exe, "restart", str(d)], env=_env(), check=True, capture_output=True)
    for k in ("rn", "um", "vm", "wm"):
        assert open(d / f"gel1{k}2.dat").read() == open(d / f"gel1{k}4.dat").read(), k
    for k in ("Velb", "Conc"):
        assert open(d / f"{k}2.dat").read() == open(d / f"{k}4.dat").read(), k

    # the reference restarts from the drop-in's files (time 2)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        r = pyref.Reference(21, 21, 21, nsub=25)
        r.set_start_time(2)
        r.add_gel((6, 6, 6), (4.75, 5.0, 5.25), 1, 1)
        r.set_params(beta=1.0, ramp_steps=0.0)
        r.finalize()
        um, vm, wm, rn = r.get(24), r.get(25), r.get(26), r.get(20).reshape(-1, 3)
        u, c1 = r.get(2).reshape(-1, 3), r.get(3)
        r.close()
    finally:
        os.chdir(cwd)
    L = 7  # nodes per axis of a 6x6x6-element gel
    E = lambda x, y, z: x + y * (L + 1) + z * (L + 1) ** 2  # noqa: E731
    Nd = lambda x, y, z: x + y * (L + 2) + z * (L + 2) ** 2  # noqa: E731
    elems = [E(x, y, z) for z in range(1, L) for y in range(1, L) for x in range(1, L)]
    nodes = [Nd(x, y, z) for z in range(1, L + 1) for y in range(1, L + 1) for x in range(1, L + 1)]
    assert np.array_equal(um[elems], _numbers(d / "gel1um2.dat")[1])
    assert np.array_equal(vm[elems], _numbers(d / "gel1vm2.dat")[1])
    assert np.array_equal(wm[elems], _numbers(d / "gel1wm2.dat")[1])
    assert np.array_equal(rn[nodes].ravel(), _numbers(d / "gel1rn2.dat")[1])
    # FP32 fields: the reference parses straight to float; allow the one-ulp
    # difference that parsing through double could make
    for got, name in ((u.ravel(), "Velb2.dat"), (c1, "Conc2.dat")):
        want = _numbers(d / name)[1].astype(np.float32)
        assert np.all(np.abs(got - want) <= np.spacing(np.abs(want))), name


SERIES_CASE = dict(dims=(20, 20, 20), nsub=2, beta=1.0, ramp=0.0, seed=4242, amp=1e-3,
                   gels=[dict(size=(6, 6, 6), pos=(4.75, 4.75, 4.75), type=1)])


def test_center_series_vs_reference_and_oracle(gpu):
    """Records at iterations 0, 1000 and 2000: rn, Fn, Veln of the centre node,
    vm and wm of the centre element."""
    from glsm_fluid_3d_b200 import System

    _need_reference()
    sys_ = build(System, SERIES_CASE)
    sys_.gels[0].series_config(1000, 8)
    sys_.run(0, 2001)
    ours = sys_.gels[0].series()[:3]
    sys_.close()

    r = build(pyref.Reference, SERIES_CASE)
    o = build(pyoracle.Oracle, SERIES_CASE)
    L = 7
    gi = L // 2 + (L // 2) * (L + 1) + (L // 2) * (L + 1) ** 2
    h = (L + 1) // 2
    hi = h + h * (L + 2) + h * (L + 2) ** 2
    want_oracle = []
    done = 0
    for it in (0, 1000, 2000):
        r.run(done, it + 1 - done)
        r.record_center(it)
        o.run(done, it + 1 - done)
        done = it + 1
        want_oracle.append(np.concatenate([[it], o.get(20).reshape(-1, 3)[hi], o.get(23).reshape(-1, 3)[hi],
                                           o.get(21).reshape(-1, 3)[hi], [o.get(25)[gi], o.get(26)[gi]]]))
    want_oracle = np.array(want_oracle)
    vm_c, wm_c = r.get(41), r.get(42)
    rm_c, fn_c, ve_c = r.get(43).reshape(-1, 3), r.get(44).reshape(-1, 3), r.get(45).reshape(-1, 3)
    r.close()
    o.close()
    want_ref = np.array([np.concatenate([[it], rm_c[s], fn_c[s], ve_c[s], [vm_c[s], wm_c[s]]])
                         for s, it in enumerate((0, 1000, 2000))])
    assert np.array_equal(ours[:, 0], [0, 1000, 2000])
    cols = {"rn": slice(1, 4), "Fn": slice(4, 7), "Veln": slice(7, 10), "vm": slice(10, 11), "wm": slice(11, 12)}
    for name, c in cols.items():
        e_orc, e_ref = rel_l2(ours[:, c], want_oracle[:, c]), rel_l2(ours[:, c], want_ref[:, c])
        print(f"series {name:5s} vs oracle {e_orc:.2e}  vs reference {e_ref:.2e}")
        assert e_orc < 1e-9 and e_ref < 1e-6, name


TUBE_CASE = dict(dims=(40, 20, 20), nsub=2, beta=1.0, ramp=0.0, seed=99, amp=1e-3,
                 gels=[dict(size=(10, 6, 6), pos=(9.75, 4.75, 4.75), type=1)])


@pytest.mark.parametrize("circular", [False, True], ids=["square", "cylinder"])
def test_tube_mask_vs_reference_and_oracle(gpu, circular):
    from glsm_fluid_3d_b200 import System

    _need_reference()

    def make(cls):
        s = cls(*TUBE_CASE["dims"], nsub=TUBE_CASE["nsub"])
        g = TUBE_CASE["gels"][0]
        s.add_gel(g["size"], g["pos"], g["type"], 1)
        s.gel_noise(0, TUBE_CASE["seed"], TUBE_CASE["amp"])
        if cls is System:
            s.gels[0].buildTubeMask(1, circular)
        else:
            s.build_tube_mask(0, 1, circular)
        s.set_params(beta=1.0, ramp_steps=0.0)
        s.finalize()
        s.run(0, 30)
        out = collect(s, TUBE_CASE)
        s.close()
        return out

    got, ref, orc = make(System), make(pyref.Reference), make(pyoracle.Oracle)
    um0 = orc["g0_um"]
    assert np.isfinite(um0).all()
    bad = []
    for k in ("u", "c1", "g0_um", "g0_vm", "g0_wm", "g0_rn", "g0_Veln", "g0_un_norm"):
        e_orc, e_ref, floor = rel_l2(got[k], orc[k]), rel_l2(got[k], ref[k]), rel_l2(orc[k], ref[k])
        # u, c1 and un_norm (which carries the FP32 Robin flux) as in
        # test_gpu_parity.py; the FP64 gel fields to 1e-8 of the oracle
        t_orc = {"u": 2e-4, "c1": 1e-5, "g0_un_norm": 1e-6}.get(k, 1e-8)
        t_ref = {"u": 2e-3, "c1": 1e-5, "g0_un_norm": 1e-5}.get(k, 1e-6)
        print(f"tube {'cyl' if circular else 'sq'} {k:12s} vs oracle {e_orc:.2e}  vs reference {e_ref:.2e} "
              f"(oracle vs reference {floor:.2e})")
        if not (e_orc <= t_orc and (e_ref <= t_ref or e_ref <= 1.05 * floor + 1e-12)):
            bad.append((k, e_orc, e_ref))
    assert not bad, bad
