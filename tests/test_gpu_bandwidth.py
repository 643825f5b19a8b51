"""The copy-bandwidth probe behind the L2 roofline denominator of the bench
(glsm_copy_bandwidth): with a footprint far above the 126 MB L2 it measures
the HBM copy bandwidth of a B200, with one well inside L2 a higher figure."""
import pytest

pytestmark = pytest.mark.gpu


def test_l2_copy_bandwidth_exceeds_hbm(gpu):
    from glsm_fluid_3d_b200 import copy_bandwidth

    hbm = copy_bandwidth(1 << 30, 6)
    l2 = copy_bandwidth(24 << 20, 400)
    assert 3000.0 < hbm < 9000.0, hbm  # the B200's HBM3e copy bandwidth, GB/s
    assert l2 > 1.2 * hbm, (l2, hbm)
