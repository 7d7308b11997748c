"""Edge cases the reference's own adversarial tests pin
(tests/test_adversarial.py in the reference: peaks on bin and window edges,
ragged bins, amplitude scale, zero inputs, a single frequency bin, a
threshold equal to the peak, binsize 1), run through every kernel family
here -- the one-pair kernel (n = 64 ... 16384), the packed n = 4096 kernel
(whole window, bins a multiple of 32 lags) and the two-pass kernels
(n >= 32768) -- against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu

LENGTHS = [64, 1024, 4096, 16384, 65536]


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def shifted(h, lag, amp=1.0):
    """A data spectrum whose correlation with h peaks at `lag`."""
    n = h.shape[-1]
    k = np.arange(n)
    return (amp * h.astype(np.complex128) * np.exp(-2j * np.pi * k * lag / n)).astype(np.complex64)


def run(D, H, **kw):
    import apogee_b200 as mf
    f = mf.MatchedFilter(D.shape[1], D.shape[0], H.shape[0])
    f.set_data(D)
    f.set_templates(H)
    return f.run(**kw).copy()


@pytest.mark.parametrize("n", LENGTHS)
def test_peak_on_every_bin_edge(n):
    """A peak at the first and at the last lag of every bin is reported in
    that bin, at that lag."""
    rng = np.random.default_rng(n)
    bs = n // 8
    H = noise(rng, (1, n))
    lags = [b * bs for b in range(8)] + [b * bs + bs - 1 for b in range(8)]
    D = np.stack([shifted(H[0], L, 50.0) + 0.01 * noise(rng, (n,)) for L in lags])
    out = run(D, H, binsize=bs)
    for i, L in enumerate(lags):
        assert out["index"][i, 0, L // bs] == L
    assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H), bs)


@pytest.mark.parametrize("n", LENGTHS)
def test_peak_at_lag_zero_and_the_last_lag(n):
    rng = np.random.default_rng(n + 1)
    H = noise(rng, (1, n))
    D = np.stack([shifted(H[0], 0, 40.0), shifted(H[0], n - 1, 40.0)])
    out = run(D, H, binsize=n)
    assert out["index"][0, 0, 0] == 0 and out["index"][1, 0, 0] == n - 1


@pytest.mark.parametrize("n", LENGTHS)
def test_window_edges(n):
    """A peak on the window's first lag and on its last lag is reported; one
    lag outside the window is not (the bin then reports its own maximum)."""
    rng = np.random.default_rng(n + 2)
    H = noise(rng, (1, n))
    ws, we = n // 8 + 3, n - n // 8 - 5
    D = np.stack([shifted(H[0], ws, 60.0), shifted(H[0], we - 1, 60.0),
                  shifted(H[0], ws - 1, 60.0), shifted(H[0], we, 60.0)])
    out = run(D, H, binsize=n, window=(ws, we))
    assert out["index"][0, 0, 0] == ws and out["index"][1, 0, 0] == we - 1
    assert out["index"][2, 0, 0] != ws - 1 and out["index"][3, 0, 0] != we
    assert ws <= out["index"][2, 0, 0] < we and ws <= out["index"][3, 0, 0] < we
    bad = parity.compare(out["index"], out["value"], oracle.correlate(D, H), n, 0.0, (ws, we))
    assert not bad, bad[:3]


@pytest.mark.parametrize("n,ws,we,bs", [(64, 3, 61, 7), (1024, 0, 1024, 100), (4096, 1, 4096, 33),
                                        (4096, 0, 4000, 64), (16384, 17, 16383, 1000),
                                        (65536, 5, 65000, 3000)])
def test_bins_that_do_not_divide_evenly(n, ws, we, bs):
    rng = np.random.default_rng(n + ws + bs)
    D, H = noise(rng, (2, n)), noise(rng, (3, n))
    out = run(D, H, binsize=bs, window=(ws, we))
    assert out.shape[-1] == -(-(we - ws) // bs)
    bad = parity.compare(out["index"], out["value"], oracle.correlate(D, H), bs, 0.0, (ws, we))
    assert not bad, bad[:3]


@pytest.mark.parametrize("n", [2048, 4096, 65536])
@pytest.mark.parametrize("amp", [1e-12, 1e-6, 1.0, 1e6, 1e12])
def test_amplitude_scale_does_not_move_the_peak(n, amp):
    """A unit-norm template planted at one lag with amplitude amp: the peak
    is at that lag with |value| = amp over twelve orders of magnitude (an
    |z|^2 that under- or overflowed would move the index)."""
    rng = np.random.default_rng(n)
    h = noise(rng, (n,)).astype(np.complex128)
    h /= np.linalg.norm(h)
    h = h.astype(np.complex64)
    lag = (733 * n) // 2048
    out = run(shifted(h, lag, amp)[None, :], h[None, :], binsize=n)
    assert out["index"][0, 0, 0] == lag
    m = abs(complex(out["value"][0, 0, 0]))
    assert np.isfinite(m) and abs(m - amp) <= 1e-3 * amp


@pytest.mark.parametrize("n", [1024, 4096])
def test_templates_of_wildly_different_scale_in_one_batch(n):
    rng = np.random.default_rng(n + 5)
    H = noise(rng, (4, n))
    H[1] *= 1e-15
    H[2] *= 1e15
    D = noise(rng, (2, n))
    out = run(D, H, binsize=n // 16)
    bad = parity.compare(out["index"], out["value"], oracle.correlate(D, H), n // 16)
    assert not bad, bad[:3]


@pytest.mark.parametrize("n", LENGTHS)
def test_zero_template_and_zero_data(n):
    """All-zero inputs report nothing (zero is never a peak), never NaN."""
    rng = np.random.default_rng(n + 6)
    H = noise(rng, (2, n))
    H[1] = 0
    D = noise(rng, (2, n))
    D[1] = 0
    out = run(D, H, binsize=n // 4)
    assert (out["index"][:, 1] == -1).all() and (out["index"][1] == -1).all()
    assert not np.isnan(out["value"]).any()
    assert (out["index"][0, 0] >= 0).all()
    pos = run(D, H, binsize=n // 4, threshold=1e-3)
    assert (pos["index"][1] == -1).all()


@pytest.mark.parametrize("n", LENGTHS)
def test_single_nonzero_frequency_bin(n):
    """A product with one nonzero frequency has |z| equal at every lag in
    exact arithmetic: which lag of a bin is reported is unspecified (the
    reference says so too), but it lies in the bin and its value is the
    oracle's at that lag."""
    D = np.zeros((1, n), np.complex64)
    H = np.zeros((1, n), np.complex64)
    D[0, 3] = 2.0
    H[0, 3] = 1.0 - 0.5j
    bs = n // 4
    out = run(D, H, binsize=bs)
    idx = out["index"][0, 0]
    assert ((idx >= np.arange(4) * bs) & (idx < np.arange(1, 5) * bs)).all()
    z = oracle.correlate(D, H)[0, 0]
    np.testing.assert_allclose(out["value"][0, 0], z[idx], rtol=1e-5)


@pytest.mark.parametrize("n", [1024, 4096, 65536])
def test_threshold_equal_to_the_peak_magnitude_is_not_a_crossing(n):
    """Crossing is strict: |z| > threshold.  A threshold a few float ulps
    above the reported peak's magnitude reports nothing in that bin; one just
    below reports the same lag."""
    rng = np.random.default_rng(n + 8)
    D, H = noise(rng, (1, n)), noise(rng, (1, n))
    out = run(D, H, binsize=n)
    mag = abs(complex(out["value"][0, 0, 0]))
    at = run(D, H, binsize=n, threshold=mag * (1 + 4e-7))
    assert at["index"][0, 0, 0] == -1 and at["value"][0, 0, 0] == 0
    below = run(D, H, binsize=n, threshold=mag * (1 - 4e-7))
    assert below["index"][0, 0, 0] == out["index"][0, 0, 0]


@pytest.mark.parametrize("n", [64, 256])
def test_binsize_one_reports_every_lag(n):
    rng = np.random.default_rng(n + 9)
    D, H = noise(rng, (2, n)), noise(rng, (2, n))
    out = run(D, H, binsize=1)
    np.testing.assert_array_equal(out["index"][:, :], np.broadcast_to(np.arange(n), (2, 2, n)))
    z = oracle.correlate(D, H)
    np.testing.assert_allclose(out["value"], z, rtol=1e-5, atol=1e-6 * np.abs(z).max())
