"""The float32 restatement of the conserving FP16 rounding (CPU): every output
is an FP16 number close to its input, and the cells' summed mass and momentum
rounding errors are smaller than with round-to-nearest."""
import numpy as np

from oracle.pyoracle import D3Q19_C, conserve_round_f16


def test_conserving_rounding_properties():
    rng = np.random.default_rng(3)
    v = (rng.standard_normal((20_000, 19)) * 10.0 ** rng.uniform(0, 3, size=(20_000, 1))).astype(np.float32)
    got = conserve_round_f16(v)
    rn = v.astype(np.float16).astype(np.float32)
    assert np.array_equal(got.astype(np.float16).astype(np.float32), got)
    spacing = np.maximum(np.abs(rn) * 2.0 ** -10, 2.0 ** -24)
    assert (np.abs(got.astype(np.float64) - v) <= 1.5 * spacing + 1e-30).all()
    assert np.array_equal(got[:, 0], rn[:, 0])  # the rest population keeps round-to-nearest

    def rms(x):
        e = v.astype(np.float64) - x
        return np.sqrt((e.sum(1) ** 2).mean()), np.sqrt(((e @ D3Q19_C) ** 2).sum(1).mean())

    (m_rn, p_rn), (m_c, p_c) = rms(rn), rms(got)
    assert m_c < 0.5 * m_rn and p_c < 0.7 * p_rn, (m_rn, m_c, p_rn, p_c)
