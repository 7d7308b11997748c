"""Flat matched filter on the device vs the FP64 oracle and the reference's
own outputs (tests/golden).  Bar: oracle/parity.py."""
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


def check(filt, D, H, binsize, threshold=0.0, window=None, **kw):
    out = filt.run(binsize=binsize, threshold=threshold, window=window, **kw)
    z = oracle.correlate(D, H)
    bad = parity.compare(out["index"], out["value"], z, binsize, threshold, window)
    assert not bad, bad[:5]
    return out


SIZES = [64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384]


@pytest.mark.parametrize("n", SIZES)
def test_parity_all_lengths(n):
    mf = _mf()
    rng = np.random.default_rng(n)
    D, H = noise(rng, (3, n)), noise(rng, (5, n))
    f = mf.MatchedFilter(n, 3, 5)
    f.set_data(D)
    f.set_templates(H)
    for binsize, thr, win in [(n, 0.0, None), (n // 16, 0.0, None), (n // 64 or 1, 0.0, None),
                              (17, 0.0, (3, n - 5)), (1, 0.0, None),
                              (n // 4, 3.0 * np.sqrt(n), (1, n)), (n + 3, 0.0, (n // 3, n))]:
        check(f, D, H, binsize, thr, win)


def test_matches_reference_golden(golden_dir):
    """Same inputs as the reference engine saw; same peaks (near ties aside)."""
    mf = _mf()
    g = np.load(os.path.join(golden_dir, "flat.npz"))
    for c in range(int(g["ncases"])):
        n, nd, nt, seed, bs, thr, w0, w1 = g["c%d_par" % c]
        n, nd, nt, bs = int(n), int(nd), int(nt), int(bs)
        win = None if w0 < 0 else (int(w0), int(w1))
        D, H = g["c%d_D" % c], g["c%d_H" % c]
        f = mf.MatchedFilter(n, nd, nt)
        f.set_data(D)
        f.set_templates(H)
        out, cnt = f.run(binsize=bs, threshold=float(thr), window=win, counts=True)
        z = oracle.correlate(D, H)
        assert not parity.compare(out["index"], out["value"], z, bs, float(thr), win)
        ri = g["c%d_idx" % c]
        diff = out["index"] != ri
        m = np.abs(z)
        for pos in zip(*np.nonzero(diff)):
            a, b = out["index"][pos], ri[pos]
            assert a >= 0 and b >= 0, (c, pos, a, b)
            assert abs(m[pos[:-1] + (a,)] - m[pos[:-1] + (b,)]) <= 1e-5 * m[pos[:-1] + (b,)]
        np.testing.assert_array_equal(cnt, g["c%d_cnt" % c])


def test_exact_ties_report_lowest_lag(golden_dir):
    """DC-only products tie at every lag (tests/test_cpu_single_peak.py)."""
    mf = _mf()
    g = np.load(os.path.join(golden_dir, "ties.npz"))
    filters = {}
    for c in range(int(g["ncases"])):
        n, lo, hi, bs, thr = g["c%d_par" % c]
        n, lo, hi, bs = int(n), int(lo), int(hi), int(bs)
        if n not in filters:
            data = np.zeros((3, n), np.complex64)
            data[:, 0] = [3 + 4j, -5j, 0]
            tm = np.zeros((5, n), np.complex64)
            tm[:, 0] = 1
            f = mf.MatchedFilter(n, 3, 5)
            f.set_data(data)
            f.set_templates(tm)
            filters[n] = f
        out = filters[n].run(binsize=bs, threshold=float(thr), window=(lo, hi))
        np.testing.assert_array_equal(out["index"], g["c%d_idx" % c])
        np.testing.assert_array_equal(out["value"], g["c%d_val" % c])


def test_period_four_tie_keeps_earliest():
    """Exact period-four correlation [0, 4, 4, 0] (test_cpu_single_peak.py:38-50)."""
    mf = _mf()
    n = 64
    data = np.zeros(n, np.complex64)
    data[[0, n // 4, 3 * n // 4]] = [2, -1 - 1j, -1 + 1j]
    f = mf.MatchedFilter(n, 1, 17)
    f.set_data(data[None, :])
    f.set_templates(np.ones((17, n), np.complex64))
    for window in [(0, 4), (1, 4), (4, 9), (5, 8), (63, 64)]:
        out = f.run(window=window, binsize=n)
        eligible = [k for k in range(*window) if k % 4 in (1, 2)]
        np.testing.assert_array_equal(out["index"], eligible[0] if eligible else -1)
        np.testing.assert_array_equal(out["value"], 4 if eligible else 0)


def test_known_lag():
    mf = _mf()
    n = 4096
    rng = np.random.default_rng(1)
    x = noise(rng, n)
    f = mf.MatchedFilter(n, 1, 5)
    f.set_data(x[None, :])
    lags = (0, 1, 37, n // 2, n - 1)
    f.set_templates(np.stack([x * np.exp(2j * np.pi * np.arange(n) * lag / n) for lag in lags])
                    .astype(np.complex64))
    out = f.run(binsize=n)
    np.testing.assert_array_equal(out["index"][0, :, 0], lags)


def test_self_correlation_and_flat_spectrum():
    mf = _mf()
    n = 1024
    rng = np.random.default_rng(2)
    h = noise(rng, n)
    f = mf.MatchedFilter(n, 1, 1)
    f.set_data(h[None])
    f.set_templates(h[None])
    out = f.run(binsize=n)
    want = float(np.sum(np.abs(h.astype(np.complex128)) ** 2))
    assert out["index"][0, 0, 0] == 0
    assert abs(abs(out["value"][0, 0, 0]) - want) <= 1e-5 * want
    g = mf.MatchedFilter(512, 1, 1)
    g.set_data(np.ones((1, 512), np.complex64))
    g.set_templates(np.ones((1, 512), np.complex64))
    m = np.abs(g.run(binsize=1)["value"][0, 0])
    assert abs(m[0] - 512) <= 1e-5 * 512 and m[1:].max() < 1e-3 * 512


def test_zero_inputs_report_nothing():
    mf = _mf()
    n = 4096
    f = mf.MatchedFilter(n, 2, 2)
    f.set_data(np.zeros((2, n), np.complex64))
    f.set_templates(np.zeros((2, n), np.complex64))
    out, cnt = f.run(binsize=256, counts=True)
    assert (out["index"] == -1).all() and (out["value"] == 0).all() and (cnt == 0).all()


def test_amplitudes_and_subnormals():
    mf = _mf()
    n = 1024
    rng = np.random.default_rng(3)
    base = noise(rng, (1, n))
    f = mf.MatchedFilter(n, 1, 1)
    f.set_templates(base)
    for scale in (1e-12, 1e-6, 1.0, 1e6, 1e12):
        D = (base * np.float32(scale)).astype(np.complex64)
        f.set_data(D)
        check(f, D, base, 128)


def test_nan_isolated_to_its_pair():
    mf = _mf()
    n = 1024
    rng = np.random.default_rng(4)
    D, H = noise(rng, (2, n)), noise(rng, (2, n))
    D[1, 5] = np.nan
    f = mf.MatchedFilter(n, 2, 2)
    f.set_data(D)
    f.set_templates(H)
    out = f.run(binsize=256)
    z = oracle.correlate(D[:1], H)
    assert not parity.compare(out["index"][:1], out["value"][:1], z, 256)


def test_window_subrange_and_raw():
    mf = _mf()
    n, nd, nt = 4096, 4, 3
    rng = np.random.default_rng(5)
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    full = f.run(binsize=1024, window=(500, 3500)).copy()
    assert ((full["index"] >= 500) & (full["index"] < 3500)).all()
    sub = f.run(binsize=1024, window=(500, 3500), data=(1, 2), templates=(0, 2))
    np.testing.assert_array_equal(sub["index"], full["index"][1:3, 0:2])
    np.testing.assert_array_equal(sub["value"], full["value"][1:3, 0:2])
    idx, val = f.run(binsize=1024, window=(500, 3500), raw=True)
    np.testing.assert_array_equal(idx, full["index"])
    np.testing.assert_array_equal(val, full["value"])


def test_threshold_is_strict_and_counts():
    mf = _mf()
    n = 256
    d = np.zeros((1, n), np.complex64)
    d[0, 0] = 3 + 4j
    t = np.zeros((1, n), np.complex64)
    t[0, 0] = 1
    f = mf.MatchedFilter(n, 1, 1)
    f.set_data(d)
    f.set_templates(t)
    for thr, expect in ((4.99, 4), (5.0, 0), (0.0, 4), (-1.0, 4)):
        out, cnt = f.run(binsize=64, threshold=thr, counts=True)
        assert cnt[0, 0] == expect


def test_single_template_and_data_setters():
    mf = _mf()
    n = 1024
    rng = np.random.default_rng(6)
    D, H = noise(rng, (2, n)), noise(rng, (3, n))
    f = mf.MatchedFilter(n, 2, 3)
    with pytest.raises(ValueError):
        f.run(binsize=n)                      # no data yet
    for i in range(2):
        f.set_data(D[i], index=i)
    with pytest.raises(ValueError):
        f.run(binsize=n)                      # no templates yet
    for i in range(3):
        f.set_templates(H[i], index=i)
    check(f, D, H, 256)
    with pytest.raises(IndexError):
        f.set_data(D[0], index=2)
    with pytest.raises(ValueError):
        f.set_data(np.zeros((2, 100), np.complex64))


def test_argument_errors():
    mf = _mf()
    with pytest.raises(ValueError):
        mf.MatchedFilter(1000, 1, 1)
    with pytest.raises(ValueError):
        mf.MatchedFilter(4096, 0, 1)
    f = mf.MatchedFilter(4096, 1, 1)
    f.set_data(np.zeros((1, 4096), np.complex64))
    f.set_templates(np.zeros((1, 4096), np.complex64))
    with pytest.raises(ValueError):
        f.run(binsize=0)
    with pytest.raises(ValueError):
        f.run(window=(10, 10))
    with pytest.raises(ValueError):
        f.run(data=(0, 2))


def test_torch_device_inputs_match_host_inputs():
    import torch
    mf = _mf()
    n = 2048
    rng = np.random.default_rng(7)
    D, H = noise(rng, (2, n)), noise(rng, (4, n))
    f = mf.MatchedFilter(n, 2, 4)
    f.set_data(torch.from_numpy(D).cuda())
    f.set_templates(torch.from_numpy(H).cuda())
    a = f.run(binsize=128).copy()
    f.set_data(D)
    f.set_templates(H)
    b = f.run(binsize=128)
    np.testing.assert_array_equal(a, b)
    idx, val = f.run_device(binsize=128)
    np.testing.assert_array_equal(idx.cpu().numpy(), b["index"])
    np.testing.assert_array_equal(val.cpu().numpy(), b["value"])


def test_batch_independence():
    """A pair's result does not depend on the rest of the batch."""
    mf = _mf()
    n, nd, nt = 4096, 5, 7
    rng = np.random.default_rng(8)
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    full = f.run(binsize=512).copy()
    g = mf.MatchedFilter(n, 1, 1)
    g.set_data(D[3:4])
    g.set_templates(H[5:6])
    one = g.run(binsize=512)
    np.testing.assert_array_equal(one[0, 0], full[3, 5])


def _same_up_to_near_ties(i1, i2, z):
    """Indices equal except where the two lags' FP64 magnitudes are within
    1e-5 relative (either kernel may then report either lag)."""
    diff = np.nonzero(i1 != i2)
    for pos in zip(*diff):
        a, b = i1[pos], i2[pos]
        assert a >= 0 and b >= 0, pos
        za, zb = abs(z[pos[:-1]][a]), abs(z[pos[:-1]][b])
        assert abs(za - zb) <= 1e-5 * max(za, zb), (pos, a, b, za, zb)


@pytest.mark.parametrize("nd,nt,binsize,threshold", [
    (16, 1024, 256, 0.0),     # the benchmark block: data rows shared by both pairs of an item
    (5, 77, 512, 3.0),        # odd nt: items straddle data rows; thresholded
    (3, 1, 64, 0.0),          # one template: every item mixes data rows; 64 bins
    (1, 3, 4096, 2.0),        # odd pair count: the last item's second pair is absent
])
def test_packed_kernel_matches_one_pair_kernel_and_oracle(nd, nt, binsize, threshold):
    """n = 4096 runs over the whole window use the kernel that carries two
    pairs per thread in packed FP32x2 arithmetic.  It must meet the oracle's
    bar and equal the one-pair kernel bit for bit (dense, listed and record
    output, counts: both form their twiddles with the same operations); listed
    rows equal the dense run's rows bit for bit."""
    import torch
    import apogee_b200 as mf
    from apogee_b200 import _lib
    n = 4096
    rng = np.random.default_rng(nd * 100 + nt)
    D = noise(rng, (nd, n))
    H = noise(rng, (nt, n))
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    L = _lib.lib()
    out = {}
    for packed in (0, 1):
        _lib.check(L.mfb_set_packed(f._plan, packed))
        r, c = f.run(binsize=binsize, threshold=threshold, counts=True)
        ri, rv = f.run(binsize=binsize, threshold=threshold, raw=True)
        out[packed] = (r.copy(), c.copy(), ri.copy(), rv.copy())
        np.testing.assert_array_equal(out[packed][0]["index"], out[packed][2])
        np.testing.assert_array_equal(out[packed][0]["value"], out[packed][3])
        np.testing.assert_array_equal(out[packed][1], (out[packed][2] >= 0).sum(-1))
    for t0 in range(0, nt, 128):
        z = oracle.correlate(D, H[t0:t0 + 128])
        for packed in (0, 1):
            r = out[packed][0][:, t0:t0 + 128]
            bad = parity.compare(r["index"], r["value"], z, binsize, threshold)
            assert not bad, (packed, bad[:3])
        _same_up_to_near_ties(out[0][2][:, t0:t0 + 128], out[1][2][:, t0:t0 + 128], z)
    np.testing.assert_array_equal(out[0][2], out[1][2])
    np.testing.assert_array_equal(out[0][3], out[1][3])
    # listed rows in arbitrary order, an odd count
    rows = np.random.default_rng(7).permutation(nd * nt)[: max(1, (nd * nt) // 2) | 1]
    rows_d = torch.as_tensor(rows.astype(np.int32), device="cuda")
    cnt_d = torch.tensor([rows.size], dtype=torch.int32, device="cuda")
    nb = n // binsize
    _lib.check(L.mfb_set_packed(f._plan, 1))
    f._bind_stream()
    idx = torch.full((nd * nt * nb,), -7, dtype=torch.int64, device="cuda")
    val = torch.zeros(nd * nt * nb, dtype=torch.complex64, device="cuda")
    _lib.check(L.mfb_run_rows(f._plan, 0, nd, 0, nt, rows_d.data_ptr(), cnt_d.data_ptr(),
                              rows.size, binsize, threshold, 0, n, idx.data_ptr(),
                              val.data_ptr(), None))
    torch.cuda.synchronize()
    got_i = idx.cpu().numpy().reshape(nd * nt, nb)
    got_v = val.cpu().numpy().reshape(nd * nt, nb)
    np.testing.assert_array_equal(got_i[rows], out[1][2].reshape(nd * nt, nb)[rows])
    np.testing.assert_array_equal(got_v[rows], out[1][3].reshape(nd * nt, nb)[rows])
    untouched = np.setdiff1d(np.arange(nd * nt), rows)
    assert (got_i[untouched] == -7).all()
