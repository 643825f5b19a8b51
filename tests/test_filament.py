"""The filament (iso-line) diagnostic calFilamentD (src/gel_kernels.cu:837-866):
the oracle's restatement against known crossings on the CPU, and the CUDA
kernel (glsm_gel_filament) against the oracle on random nodal fields."""
import numpy as np
import pytest

from oracle.pyoracle import filament, iso_crossing


def test_iso_crossing_known_answers():
    # u = 0.15 + (y - 0.7), v = 0.15 + (x - 0.3): crossing at (0.3, 0.7)
    r = iso_crossing(0.15 - 0.7, 0.15 - 0.7, 1.15 - 0.7, 1.15 - 0.7, 0.15 - 0.3, 1.15 - 0.3, 0.15 - 0.3, 1.15 - 0.3)
    assert r is not None and abs(r[0] - 0.3) < 1e-12 and abs(r[1] - 0.7) < 1e-12
    # the same crossing with u and v swapped is not found: y is solved from the
    # u contour, which then does not depend on y (as in the reference)
    assert iso_crossing(0.15 - 0.3, 1.15 - 0.3, 0.15 - 0.3, 1.15 - 0.3, 0.15 - 0.7, 0.15 - 0.7, 1.15 - 0.7,
                        1.15 - 0.7) is None
    # both fields above the iso value everywhere: no crossing
    assert iso_crossing(0.5, 0.6, 0.7, 0.8, 0.5, 0.6, 0.7, 0.8) is None
    # parallel contours (u = v): no isolated crossing
    assert iso_crossing(0.1, 0.2, 0.1, 0.2, 0.1, 0.2, 0.1, 0.2) is None


def test_filament_places_points_in_node_units():
    LX = LY = LZ = 4
    n = (LX + 2) * (LY + 2) * (LZ + 2)
    u = np.full(n, 0.5)
    v = np.full(n, 0.5)
    sx, sxy = LX + 2, (LX + 2) * (LY + 2)
    for zi in range(LZ + 2):
        for yi in range(LY + 2):
            for xi in range(LX + 2):
                k = xi + yi * sx + zi * sxy
                u[k] = 0.15 + (yi - 1.5)   # u = 0.15 on y = 1.5
                v[k] = 0.15 + (xi - 2.25)  # v = 0.15 on x = 2.25
    pts = filament(u, v, LX, LY, LZ)
    assert pts.shape == (LZ - 1, 3)
    np.testing.assert_allclose(pts[:, 0], 2.25, atol=1e-12)
    np.testing.assert_allclose(pts[:, 1], 1.5, atol=1e-12)
    np.testing.assert_allclose(pts[:, 2], [1, 2, 3])


@pytest.mark.gpu
def test_gpu_filament_matches_oracle(gpu):
    from glsm_fluid_3d_b200 import Gel

    g = Gel((6, 5, 7), (10.0, 10.0, 10.0), 1, 1)
    rng = np.random.default_rng(7)
    n = g.read("un_norm").size
    u = 0.15 + 0.1 * rng.standard_normal(n)
    v = 0.15 + 0.1 * rng.standard_normal(n)
    g.write("un_norm", u)
    g.write("vn_norm", v)
    got = g.filament()
    want = filament(u, v, g.LX, g.LY, g.LZ)
    assert want.shape[0] > 10
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    assert g.filament(max_points=3).shape == (3, 3)
    g.close()
