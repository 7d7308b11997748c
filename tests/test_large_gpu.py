"""Transforms larger than one CTA (n = 32768 ... 2^20): the two-pass four-step
path, against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu


def _mf():
    import apogee_b200 as mf
    return mf


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.mark.parametrize("n", [32768, 65536, 131072, 262144])
def test_large_parity(n):
    mf = _mf()
    rng = np.random.default_rng(n + 1)
    nd, nt = 2, 3
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    z = oracle.correlate(D, H)
    for binsize, thr, win in [(n // 16, 0.0, None), (n // 64, 0.0, None), (4096, 0.0, None),
                              (n // 100 + 7, 0.0, (13, n - 5)),
                              (n // 8, 4.0 * np.sqrt(n), (n // 3, n)), (n, 0.0, None)]:
        out, cnt = f.run(binsize=binsize, threshold=thr, window=win, counts=True)
        bad = parity.compare(out["index"], out["value"], z, binsize, thr, win)
        assert not bad, (binsize, thr, win, bad[:3])
        np.testing.assert_array_equal(cnt, (out["index"] >= 0).sum(-1))


def test_largest_length():
    mf = _mf()
    n = 1 << 20
    rng = np.random.default_rng(3)
    D, H = noise(rng, (1, n)), noise(rng, (2, n))
    f = mf.MatchedFilter(n, 1, 2)
    f.set_data(D)
    f.set_templates(H)
    out = f.run(binsize=n // 256)
    assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H), n // 256)


def test_large_known_lag_and_subrange():
    mf = _mf()
    n = 262144
    rng = np.random.default_rng(4)
    x = noise(rng, n)
    lags = (0, 1, 12345, n - 1)
    H = np.stack([x * np.exp(2j * np.pi * np.arange(n) * lag / n) for lag in lags]).astype(np.complex64)
    f = mf.MatchedFilter(n, 1, len(lags))
    f.set_data(x[None])
    f.set_templates(H)
    out = f.run(binsize=n)
    np.testing.assert_array_equal(out["index"][0, :, 0], lags)
    sub = f.run(binsize=n, templates=(1, 2))
    np.testing.assert_array_equal(sub["index"][0, :, 0], lags[1:3])


def test_large_too_many_bins_refused():
    mf = _mf()
    n = 65536
    f = mf.MatchedFilter(n, 1, 1)
    f.set_data(np.ones((1, n), np.complex64))
    f.set_templates(np.ones((1, n), np.complex64))
    with pytest.raises(ValueError):
        f.run(binsize=8)


def test_large_hierarchical_refine_is_flat():
    """Gate 0 refines every pair: the hierarchical result equals the flat one."""
    mf = _mf()
    n, nd, nt = 65536, 2, 3
    rng = np.random.default_rng(5)
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    flat = mf.MatchedFilter(n, nd, nt)
    hf = mf.HierarchicalFilter(n, nd, nt, band=n // 16, coarse="fp32")
    hf.set_coarse_threshold(0.0)
    for o in (flat, hf):
        o.set_data(D)
        o.set_templates(H)
    a = flat.run(binsize=n // 16).copy()
    b = hf.run(binsize=n // 16)
    np.testing.assert_array_equal(a, b)
    assert hf.stats == (nd * nt, nd * nt)


@pytest.mark.parametrize("n", [32768, 131072])
def test_large_run_series(n):
    """run_series for n > 16384: two-pass forward transforms of the blocks,
    then the two-pass filter, grouped by window (src/matchfilt.c:437-490)."""
    mf = _mf()
    rng = np.random.default_rng(n + 7)
    nt = 3
    H = noise(rng, (nt, n))
    series = rng.standard_normal(3 * n + n // 3).astype(np.float32)
    starts = np.array([0, n // 2, n, 2 * n, 3 * n])          # the last one runs past the end
    ws = np.array([n // 8, n // 8, 0, n // 8, n // 8])
    we = np.array([n, n, n - n // 8, n, n])
    f = mf.MatchedFilter(n, 2, nt)
    f.set_templates(H)
    bs = n // 32
    idx, val = f.run_series(series.astype(np.complex64), starts, ws, we, binsize=bs, raw=True)
    z = oracle.correlate(oracle.series_spectra(series, starts, n), H)
    for b in range(starts.size):
        bad = parity.compare(idx[b:b + 1], val[b:b + 1], z[b:b + 1], bs, 0.0,
                             (int(ws[b]), int(we[b])))
        assert not bad, (b, bad[:3])


@pytest.mark.parametrize("coarse", ["fp16x3", "bf16x3"])
@pytest.mark.parametrize("nd,nt,window", [(3, 5, None), (4, 160, (1000, 30000))])
def test_band_16384_tensor_core_coarse(coarse, nd, nt, window):
    """The split-precision tensor-core coarse pass at band 16384 (a four-step
    around the 512-point tensor-core pass, batches of 512 pairs): coarse
    maxima against FP64 over the widened coarse window, and a gated run whose
    fired rows are the flat filter's rows and whose dismissed rows are empty."""
    import apogee_b200 as mf
    n, band = 32768, 16384
    rng = np.random.default_rng(nd * 1000 + nt)
    D = (rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))).astype(np.complex64)
    H = (rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))).astype(np.complex64)
    hf = mf.HierarchicalFilter(n, nd, nt, band=band, coarse=coarse)
    hf.set_coarse_threshold(0.0)
    hf.set_data(D)
    hf.set_templates(H)
    cv = hf.coarse_values(window=window)
    cm = oracle.coarse_max(D, H, band, None, window)
    rel = np.abs(cv - cm) / cm
    assert rel.max() < 2e-5, rel.max()
    gate = float(np.quantile(cm, 0.7))
    hf.set_coarse_threshold(gate)
    bs = n // 16
    out = hf.run(binsize=bs, threshold=0.0, window=window).copy()
    flat = mf.MatchedFilter(n, nd, nt)
    flat.set_data(D)
    flat.set_templates(H)
    ref = flat.run(binsize=bs, threshold=0.0, window=window)
    fired = (out["index"] >= 0).any(-1)
    assert hf.last_refinements == int(fired.sum())
    np.testing.assert_array_equal(fired, cv >= gate)
    np.testing.assert_array_equal(out[fired], ref[fired])
    assert (out["index"][~fired] == -1).all() and (out["value"][~fired] == 0).all()
