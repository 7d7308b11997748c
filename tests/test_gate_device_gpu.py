"""The gate model with its numerics on the GPU (FP64 covariances and
Cholesky factors, FP32 draws) against the host restatement, which is pinned
bit-for-bit to the reference's gate_for: same draws, so the same gate up to
rounding."""
import numpy as np
import pytest

from apogee_b200 import gatemodel, synthetic

pytestmark = pytest.mark.gpu


def inspiral_power(n, exponent=-7 / 3.0, knee_frac=0.0150):
    p = np.zeros(n, dtype=np.float32)
    k = np.arange(1, n // 2).astype(np.float64)
    p[1:n // 2] = (k ** exponent / ((knee_frac * n / k) ** 4 + 1.0)).astype(np.float32)
    return p / p.sum()


def bank_power(n, nt=16):
    H = synthetic.template_bank(n, nt, np.random.default_rng(1)).astype(np.complex128)
    return (np.abs(H) ** 2).mean(0).astype(np.float32)


@pytest.mark.parametrize("n,band,snr,fd,kind", [
    (4096, 512, 5.5, 1e-2, "bank"),
    (4096, 1024, 6.0, 1e-3, "inspiral"),
    (16384, 2048, 5.5, 1e-2, "white"),
    (262144, 16384, 6.0, 1e-3, "bank"),
])
def test_device_gate_matches_host(n, band, snr, fd, kind):
    p = {"bank": bank_power, "inspiral": inspiral_power,
         "white": lambda n: np.ones(n, np.float32)}[kind](n)
    nsamp = gatemodel.samples_for(fd)
    host = gatemodel.kept_coarse(p, n, band, snr, nsamp)
    dev = gatemodel.kept_coarse(p, n, band, snr, nsamp, device=0)
    assert host is not None and dev is not None
    # the fine stage keeps the same draws except at its own rounding edge
    assert abs(len(host) - len(dev)) <= max(2, len(host) // 10000)
    m = min(len(host), len(dev))
    np.testing.assert_allclose(dev[:m], host[:m], rtol=1e-5, atol=1e-6)
    g_host = gatemodel.gate_for(p, n, band, snr, fd)
    g_dev = gatemodel.gate_for(p, n, band, snr, fd, device=0)
    assert g_host is not None and g_dev is not None
    assert abs(g_dev - g_host) <= 1e-5 * g_host, (g_dev, g_host)
