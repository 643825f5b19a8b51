"""Lattice shapes, boundaries and storages of the substep kernel against the
FP64 oracle, plus the FP64 conservation sums.

The cases reach the kernel's gather/scatter forms: odd and even dimensions
(tiles that straddle rows and planes), nz so small that every warp touches a
z wall, periodic x, y and z (alone and together), a uniform body force, no gel
at all, and the three population storages.  The conservation tests check the
device's FP64 mass and momentum sums against the populations read back, and
against the exact growth of momentum under a uniform body force.
"""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from parity import rel_l2

pytestmark = pytest.mark.gpu

# lattice, periodic axes, F_const, gels [(size, physical position)], substeps, iterations
CASES = {
    "odd_dims": dict(dims=(21, 19, 17), periodic=(0, 0, 0), force=(0.0, 0.0, 0.0),
                     gels=[((3, 3, 3), (5.0, 4.5, 4.0))], nsub=3, iters=6),
    "even_dims": dict(dims=(20, 22, 18), periodic=(0, 0, 0), force=(0.0, 0.0, 0.0),
                      gels=[((3, 3, 3), (4.75, 5.25, 4.25))], nsub=2, iters=6),
    "thin_z5": dict(dims=(18, 14, 5), periodic=(0, 0, 0), force=(1e-5, 0.0, 0.0), gels=[], nsub=3, iters=5),
    "thin_z6": dict(dims=(18, 14, 6), periodic=(0, 0, 0), force=(0.0, 2e-5, 0.0), gels=[], nsub=3, iters=5),
    "periodic_xy": dict(dims=(20, 18, 15), periodic=(1, 1, 0), force=(2e-6, 0.0, 0.0),
                        gels=[((3, 3, 3), (4.75, 4.25, 3.5))], nsub=3, iters=6),
    "periodic_z": dict(dims=(16, 17, 13), periodic=(0, 0, 1), force=(0.0, 0.0, 3e-6),
                       gels=[((3, 3, 3), (3.75, 4.0, 3.0))], nsub=2, iters=6),
    "periodic_all": dict(dims=(15, 16, 11), periodic=(1, 1, 1), force=(1e-6, -2e-6, 3e-6),
                         gels=[((2, 2, 2), (3.5, 3.75, 2.5))], nsub=3, iters=5),
}
TOL = {"f32": {"u": 2e-4, "pop": 1e-6, "rho": 1e-6},
       "f16": {"u": 2e-3, "pop": 1e-5, "rho": 1e-5},
       "bf16": {"u": 3e-2, "pop": 1e-4, "rho": 1e-4}}


def _build(cls, c, **kw):
    sim = cls(*c["dims"], nsub=c["nsub"], **kw)
    for k, (size, pos) in enumerate(c["gels"]):
        sim.add_gel(size, pos, 1, k + 1)
        sim.gel_noise(k, 4321 + k, 1e-3)
    sim.set_params(beta=1.0, ramp_steps=0.0, force=c["force"], periodic=c["periodic"])
    sim.finalize()
    return sim


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("case", list(CASES))
def test_layout_vs_oracle(gpu, case, storage):
    from glsm_fluid_3d_b200 import System

    c = CASES[case]
    sim = _build(System, c, storage=storage)
    sim.run(0, c["iters"])
    got = {"u": sim.get(2), "pop": sim.get(0), "rho": sim.get(1)}
    sim.close()
    ref = _build(Oracle, c)
    ref.run(0, c["iters"])
    want = {"u": ref.get(2), "pop": ref.get(0), "rho": ref.get(1)}
    ref.close()
    bad = []
    for k, tol in TOL[storage].items():
        e = rel_l2(got[k], want[k])
        print(f"{case} {storage} {k} rel_l2={e:.2e}")
        if not e <= tol:
            bad.append((k, e, tol))
    assert not bad, bad


# D3Q19 velocities in the reference's direction order (src/fluid.cu:202-215)
C = np.array([(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
              (1, 1, 0), (-1, 1, 0), (-1, -1, 0), (1, -1, 0), (1, 0, 1), (-1, 0, 1), (-1, 0, -1), (1, 0, -1),
              (0, 1, 1), (0, 1, -1), (0, -1, -1), (0, -1, 1)], dtype=np.float64)


W32 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float32).astype(np.float64)


def _host_sums(fluid):
    """Mass and momentum of the populations read back in the reference layout.
    The read-back values are FP32 f = d + w; summing them directly would add the
    FP32 rounding of w once per cell, so the sums run over f - w(FP32)."""
    f = fluid.read("pop").astype(np.float64).reshape(19, -1)
    d = f - W32[:, None]
    return f.shape[1] + float(d.sum()), C.T @ d.sum(axis=1)


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("nsub", [2, 3])
def test_conservation_with_walls(gpu, storage, nsub):
    """Bounce-back walls and IBM (Guo) forcing conserve the mass; the FP64 sums
    agree with the populations read back, after odd and even substep counts."""
    from glsm_fluid_3d_b200 import System

    c = dict(CASES["odd_dims"], nsub=nsub)
    sim = _build(System, c, storage=storage)
    N = int(np.prod(c["dims"]))
    # per substep every stored population rounds once: 2^-24 relative in FP32,
    # 2^-12 in FP16, whose values near the gel are large enough to dominate
    tol = 1e-9 if storage == "f32" else 2e-7
    for it in range(4):
        sim.run(it, 1)
        m, px, py, pz = sim.fluid.conservation()
        assert abs(m - N) / N < tol, (it, m - N)
        hm, hp = _host_sums(sim.fluid)
        assert abs(hm - m) / N < 1e-8, (it, hm, m)
        np.testing.assert_allclose([px, py, pz], hp, rtol=0, atol=2e-6 * N ** 0.5)
    sim.close()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_momentum_grows_by_the_body_force(gpu, storage):
    """All axes periodic, no gel: every substep adds N F_const to the population
    momentum (Guo forcing), and the mass stays N."""
    from glsm_fluid_3d_b200 import System

    F = (2e-6, -1e-6, 3e-6)
    c = dict(dims=(17, 14, 13), periodic=(1, 1, 1), force=F, gels=[], nsub=3)
    sim = _build(System, c, storage=storage)
    N = int(np.prod(c["dims"]))
    rtol = 1e-5 if storage == "f32" else 2e-3
    for it in range(3):
        sim.run(it, 1)
        m, px, py, pz = sim.fluid.conservation()
        s = 3 * (it + 1)
        assert abs(m - N) / N < 1e-9
        np.testing.assert_allclose([px, py, pz], [N * F[0] * s, N * F[1] * s, N * F[2] * s], rtol=rtol)
    sim.close()
