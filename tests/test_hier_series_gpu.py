"""HierarchicalFilter.run_series (ap_hmf_run_series, src/hmf.c:158-220):
blocks transformed on the device into the plan's data rows in runs of equal
windows, then coarse pass, gate and refine."""
import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu


def _mf():
    import apogee_b200 as mf
    return mf


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def layout(n, nblocks):
    starts = np.arange(nblocks) * (n // 2)
    ws = np.where(np.arange(nblocks) % 4 == 3, n // 8, n // 4)
    we = ws + n // 2
    return starts, ws, we


@pytest.mark.parametrize("n,band,coarse", [(4096, 512, "fp32"), (4096, 512, "bf16x3"),
                                           (65536, 4096, "fp32")])
def test_gate_zero_equals_flat_series(n, band, coarse):
    """With gate 0 every pair is refined: the result is the flat run_series'."""
    mf = _mf()
    rng = np.random.default_rng(n + band)
    nd, nt, nblk = 3, 5, 10                     # more blocks than data rows
    H = noise(rng, (nt, n))
    series = noise(rng, nblk * n // 2 + n)
    starts, ws, we = layout(n, nblk)
    bs = n // 16
    flat = mf.MatchedFilter(n, nd, nt)
    flat.set_templates(H)
    a = flat.run_series(series, starts, ws, we, binsize=bs)
    hf = mf.HierarchicalFilter(n, nd, nt, band=band, coarse=coarse)
    hf.set_coarse_threshold(0.0)
    hf.set_templates(H)
    b = hf.run_series(series, starts, ws, we, binsize=bs)
    np.testing.assert_array_equal(a["index"], b["index"])
    np.testing.assert_array_equal(a["value"], b["value"])
    assert hf.stats == (nblk * nt, nblk * nt)


def test_gated_series_matches_oracle_and_restores_data():
    mf = _mf()
    n, band, nd, nt, nblk = 4096, 512, 4, 6, 9
    rng = np.random.default_rng(3)
    H = noise(rng, (nt, n))
    series = noise(rng, nblk * n // 2 + n // 3)
    starts, ws, we = layout(n, nblk)
    for b in (1, 4, 6):                         # loud signals in some blocks
        t = int(rng.integers(nt))
        x = np.roll(np.fft.ifft(H[t]) * n * 0.05, n // 4 + 200)   # peaks at lag n/4 + 200
        series[starts[b]:starts[b] + n] += x.astype(np.complex64)
    bs, thr, gate = 256, 0.0, 60.0
    D0 = noise(rng, (nd, n))
    hf = mf.HierarchicalFilter(n, nd, nt, band=band, coarse="fp32")
    hf.set_coarse_threshold(gate)
    hf.set_templates(H)
    hf.set_data(D0)
    before = hf.run(binsize=bs).copy()
    out = hf.run_series(series, starts, ws, we, binsize=bs, threshold=thr)
    spec = oracle.series_spectra(series, starts, n)
    z = oracle.correlate(spec, H)
    fired_any = False
    for b in range(nblk):
        win = (int(ws[b]), int(we[b]))
        cm = oracle.coarse_max(spec[b:b + 1], H, band, None, win)[0]
        near = np.abs(cm - gate) <= 1e-5 * gate
        dev_fired = (out["index"][b] >= 0).any(-1)
        assert not ((dev_fired != (cm >= gate)) & ~near).any(), b
        fired = (cm >= gate) & ~near
        fired_any |= bool(fired.any())
        assert not parity.compare(out["index"][b:b + 1], out["value"][b:b + 1], z[b:b + 1],
                                  bs, thr, win, rows_mask=fired[None]), b
    assert fired_any
    after = hf.run(binsize=bs)                  # set_data's rows are back
    np.testing.assert_array_equal(before, after)
