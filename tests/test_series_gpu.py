"""run_series on the device: forward transform of caller-laid-out blocks
then the flat filter (src/matchfilt.c:437-490)."""
import os

import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu


def _mf():
    import apogee_b200 as mf
    return mf


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def test_matches_reference_golden(golden_dir):
    mf = _mf()
    g = np.load(os.path.join(golden_dir, "series.npz"))
    n, nt, bs, thr = (int(x) for x in g["par"])
    f = mf.MatchedFilter(n, 4, nt)
    f.set_templates(g["H"])
    out = f.run_series(g["series"], g["starts"], g["ws"], g["we"], binsize=bs)
    spec = oracle.series_spectra(g["series"], g["starts"], n)
    z = oracle.correlate(spec, g["H"])
    win = (int(g["ws"][0]), int(g["we"][0]))
    assert not parity.compare(out["index"], out["value"], z, bs, 0.0, win)
    diff = out["index"] != g["idx"]
    m = np.abs(z)
    for pos in zip(*np.nonzero(diff)):
        a, b = out["index"][pos], g["idx"][pos]
        assert abs(m[pos[:-1] + (a,)] - m[pos[:-1] + (b,)]) <= 1e-5 * m[pos[:-1] + (b,)]


def test_ragged_windows_grouping_and_order():
    mf = _mf()
    rng = np.random.default_rng(41)
    n, nt = 2048, 3
    H = noise(rng, (nt, n))
    series = noise(rng, 9000)
    starts = np.array([0, 1024, 2048, 3072, 4096, 5120, 6144, 7168, 8000])
    ws = np.array([0, 100, 0, 100, 0, 100, 0, 100, 50])
    we = np.array([1024, 1124, 1024, 1124, 1024, 1124, 1024, 1124, 1074])
    f = mf.MatchedFilter(n, 2, nt)
    f.set_templates(H)
    idx, val = f.run_series(series, starts, ws, we, binsize=256, raw=True)
    spec = oracle.series_spectra(series, starts, n)
    z = oracle.correlate(spec, H)
    for b in range(starts.size):
        bad = parity.compare(idx[b:b + 1], val[b:b + 1], z[b:b + 1], 256, 0.0,
                             (int(ws[b]), int(we[b])))
        assert not bad, (b, bad[:3])


def test_series_contract_errors():
    mf = _mf()
    rng = np.random.default_rng(42)
    n = 1024
    f = mf.MatchedFilter(n, 1, 1)
    f.set_templates(noise(rng, (1, n)))
    ser = noise(rng, 3000)
    with pytest.raises(ValueError):
        f.run_series(ser, [0, 10], [0, 0], [1024, 100], binsize=256)   # unequal bin counts
    with pytest.raises(ValueError):
        f.run_series(ser, [], [], [], binsize=256)
    with pytest.raises(ValueError):
        f.run_series(ser, [0], [5], [5], binsize=256)                  # empty window
    f.set_data(noise(rng, (1, n)))
    f.run_series(ser, [0], [0], [n], binsize=256)
    with pytest.raises(ValueError):
        f.run(binsize=256)                    # series consumed the data slots


def test_series_equals_block_by_block():
    """Blocks filtered through run_series agree with the flat filter on the
    same (device-computed) spectra, block by block."""
    mf = _mf()
    rng = np.random.default_rng(43)
    n, nt = 4096, 4
    H = noise(rng, (nt, n))
    series = noise(rng, 3 * n + 100)
    starts = np.array([0, n, 2 * n, 3 * n])
    f = mf.MatchedFilter(n, 4, nt)
    f.set_templates(H)
    idx, val = f.run_series(series, starts, np.zeros(4), np.full(4, n), binsize=512, raw=True)
    spec = oracle.series_spectra(series, starts, n)
    z = oracle.correlate(spec, H)
    assert not parity.compare(idx, val, z, 512)
