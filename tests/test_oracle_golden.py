"""The FP64 oracle against the reference's own outputs (CPU only).

The fixtures in tests/golden/ were produced by the reference engine itself
(tests/golden/make_golden.py); these tests pin the oracle that every GPU
parity test uses."""
import os

import numpy as np
import pytest

from oracle import oracle, parity


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def test_oracle_matches_reference_flat(golden_dir):
    g = _load(golden_dir, "flat.npz")
    for c in range(int(g["ncases"])):
        n, nd, nt, seed, bs, thr, w0, w1 = g["c%d_par" % c]
        win = None if w0 < 0 else (int(w0), int(w1))
        D, H = g["c%d_D" % c], g["c%d_H" % c]
        oi, ov, oc, z = oracle.flat(D, H, int(bs), float(thr), win)
        # the reference's float32 result passes the same parity bar the GPU must meet
        bad = parity.compare(g["c%d_idx" % c], g["c%d_val" % c], z, int(bs), float(thr), win)
        assert not bad, (c, bad[:3])
        # and the oracle's indices equal the reference's except at near ties
        diff = oi != g["c%d_idx" % c]
        if diff.any():
            m = np.abs(z)
            for pos in zip(*np.nonzero(diff)):
                a, b = oi[pos], g["c%d_idx" % c][pos]
                assert a >= 0 and b >= 0
                assert abs(m[pos[:-1] + (a,)] - m[pos[:-1] + (b,)]) <= 1e-5 * m[pos[:-1] + (a,)]
        np.testing.assert_array_equal(oc, g["c%d_cnt" % c])


def test_oracle_matches_reference_exact_ties(golden_dir):
    """DC-only products tie at every lag: the lowest lag wins, exactly."""
    g = _load(golden_dir, "ties.npz")
    for c in range(int(g["ncases"])):
        n, lo, hi, bs, thr = g["c%d_par" % c]
        n, lo, hi, bs = int(n), int(lo), int(hi), int(bs)
        data = np.zeros((3, n), np.complex64)
        data[:, 0] = [3 + 4j, -5j, 0]
        tm = np.zeros((5, n), np.complex64)
        tm[:, 0] = 1
        oi, ov, _, _ = oracle.flat(data, tm, bs, float(thr), (lo, hi))
        np.testing.assert_array_equal(oi, g["c%d_idx" % c])
        np.testing.assert_array_equal(ov.astype(np.complex64), g["c%d_val" % c])


def test_oracle_matches_reference_hierarchical(golden_dir):
    g = _load(golden_dir, "hier.npz")
    for c in range(int(g["ncases"])):
        n, nd, nt, band, seed, snr, fd, bs, thr, gate, pairs, trig = g["c%d_par" % c]
        D, H, P = g["c%d_D" % c], g["c%d_H" % c], g["c%d_power" % c]
        oi, ov, fired, z = oracle.hier(D, H, int(band), gate, int(bs), float(thr), None, P)
        ri, rv = g["c%d_idx" % c], g["c%d_val" % c]
        # the reference refines exactly the pairs the FP64 coarse gate fires,
        # except where the coarse max sits within float32 rounding of the gate
        cm = oracle.coarse_max(D, H, int(band), P)
        near = np.abs(cm - gate) <= 1e-5 * gate
        ref_fired = (ri >= 0).any(-1)
        assert not (ref_fired & ~fired & ~near).any()
        assert int(trig) >= ref_fired.sum()
        bad = parity.compare(ri, rv, z, int(bs), float(thr), rows_mask=fired & ~near)
        assert not bad, bad[:3]


def test_oracle_matches_reference_series(golden_dir):
    g = _load(golden_dir, "series.npz")
    n, nt, bs, thr = (int(x) for x in g["par"])
    spec = oracle.series_spectra(g["series"], g["starts"], n)
    z = oracle.correlate(spec, g["H"])
    ws, we = int(g["ws"][0]), int(g["we"][0])
    bad = parity.compare(g["idx"], g["val"], z, bs, 0.0, (ws, we))
    assert not bad, bad[:3]


def test_direct_sum_agrees_with_fft_oracle():
    rng = np.random.default_rng(5)
    d = rng.standard_normal(128) + 1j * rng.standard_normal(128)
    h = rng.standard_normal(128) + 1j * rng.standard_normal(128)
    z1 = oracle.direct_correlation(d, h)
    z2 = oracle.correlate(d[None], h[None])[0, 0]
    np.testing.assert_allclose(z1, z2, rtol=0, atol=1e-9 * np.abs(z1).max())


def test_parity_checker_catches_planted_errors():
    """A mistake planted in an oracle-derived result must be reported."""
    rng = np.random.default_rng(6)
    D = (rng.standard_normal((1, 256)) + 1j * rng.standard_normal((1, 256)))
    H = (rng.standard_normal((1, 256)) + 1j * rng.standard_normal((1, 256)))
    oi, ov, _, z = oracle.flat(D, H, 64)
    assert not parity.compare(oi, ov, z, 64)
    bad_i = oi.copy()
    bad_i[0, 0, 1] = (bad_i[0, 0, 1] + 1 - 64) % 64 + 64
    assert parity.compare(bad_i, ov, z, 64)
    bad_v = ov.copy()
    bad_v[0, 0, 2] *= (1 + 1e-4)
    assert parity.compare(oi, bad_v, z, 64)
