"""Parity with the FP64 oracle for a gel larger than one pass of the gel
kernel's element stage: an 8x8x8-element gel has 9^3 = 729 element slots,
more than the 512 threads of its CTA, so the element geometry runs in two
passes and the node forces and terms read rm_loc and nmSm from global memory
instead of the stage (csrc/gel.cu element_geometry, GeomStage).  Twelve
iterations cover three mechanics iterations (0, 5, 10); tolerances as the
golden-case parity tests."""
import pytest

from cases import build, collect
from oracle.pyoracle import Oracle
from test_gpu_parity import GEL_TOL, TOL_ORACLE, _check

pytestmark = pytest.mark.gpu

LARGE = dict(dims=(28, 28, 28), nsub=2, iters=12, beta=1.0, ramp=0.0, seed=4242, amp=1e-3, save_pop=False,
             gels=[dict(size=(8, 8, 8), pos=(6.75, 6.75, 6.75), type=1)])


def _run(cls, **kw):
    sim = build(cls, LARGE, **kw)
    sim.run(0, LARGE["iters"])
    out = collect(sim, LARGE)
    sim.close()
    return out


@pytest.mark.parametrize("methods", [False, True], ids=["fused", "methods"])
def test_large_gel_matches_oracle(gpu, methods):
    from glsm_fluid_3d_b200 import System

    got = _run(System, methods=methods)
    want = _run(Oracle)
    bad = _check(got, want, TOL_ORACLE, GEL_TOL, f"large-gel/{'methods' if methods else 'fused'}")
    assert not bad, bad
