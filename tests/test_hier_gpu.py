"""Hierarchical filter on the device: the one-sided contract
(python/matchedfilter/__init__.py:1055-1080; tests/test_api.py:163-238)."""
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


def inspiral_power(n, exponent=-7 / 3.0, knee_frac=0.0150):
    p = np.zeros(n, dtype=np.float32)
    k = np.arange(1, n // 2).astype(np.float64)
    p[1:n // 2] = (k ** exponent / ((knee_frac * n / k) ** 4 + 1.0)).astype(np.float32)
    return p / p.sum()


def template_with_power(n, power):
    h = np.sqrt(power).astype(np.complex64)
    return h / np.linalg.norm(h)


@pytest.mark.parametrize("coarse", ["fp32", "bf16x3", "fp16x3"])
def test_identical_or_absent(coarse):
    """Every reported peak is bit-identical to the flat filter's; only omissions."""
    mf = _mf()
    n, nd, nt = 4096, 4, 4
    rng = np.random.default_rng(11)
    power = inspiral_power(n)
    H = np.stack([template_with_power(n, power) for _ in range(nt)])
    D = noise(rng, (nd, n))
    for d in range(nd):
        lag = 300 + 17 * d
        D[d] += (12.0 * H[0] * np.exp(2j * np.pi * np.arange(n) * lag / n)).astype(np.complex64)
    flat = mf.MatchedFilter(n, nd, nt)
    hf = mf.HierarchicalFilter(n, nd, nt, snr=5.5, fd=1e-2, coarse=coarse)
    hf.set_reference(power)
    for o in (flat, hf):
        o.set_data(D)
        o.set_templates(H)
    a = flat.run(binsize=1024, threshold=5.5).copy()
    b = hf.run(binsize=1024, threshold=5.5)
    fired = b["index"] >= 0
    assert fired.any()
    assert not (fired & (a["index"] < 0)).any()
    np.testing.assert_array_equal(a["index"][fired], b["index"][fired])
    np.testing.assert_array_equal(a["value"][fired], b["value"][fired])
    assert (b["value"][~fired] == 0).all()


def test_matches_reference_golden(golden_dir):
    """Reference hierarchical engine, same inputs, pinned band and gate."""
    mf = _mf()
    g = np.load(os.path.join(golden_dir, "hier.npz"))
    for c in range(int(g["ncases"])):
        n, nd, nt, band, seed, snr, fd, bs, thr, gate, pairs, trig = g["c%d_par" % c]
        n, nd, nt, band, bs = int(n), int(nd), int(nt), int(band), int(bs)
        D, H, P = g["c%d_D" % c], g["c%d_H" % c], g["c%d_power" % c]
        hf = mf.HierarchicalFilter(n, nd, nt, snr=snr, fd=fd, band=band, coarse="fp32")
        hf.set_reference(P)
        hf.set_coarse_threshold(gate)
        hf.set_data(D)
        hf.set_templates(H)
        out = hf.run(binsize=bs, threshold=float(thr))
        cm = oracle.coarse_max(D, H, band, P)
        near = np.abs(cm - gate) <= 1e-5 * gate
        ri = g["c%d_idx" % c]
        dev_fired = (out["index"] >= 0).any(-1)
        ref_fired = (ri >= 0).any(-1)
        assert not ((dev_fired != ref_fired) & ~near).any()
        z = oracle.correlate(D, H)
        fired = (cm >= gate) & ~near
        assert not parity.compare(out["index"], out["value"], z, bs, float(thr), rows_mask=fired)
        assert hf.stats[0] == nd * nt
        assert abs(hf.stats[1] - int(trig)) <= near.sum()


def test_pure_noise_is_ruled_out():
    mf = _mf()
    n, nd = 4096, 64
    rng = np.random.default_rng(12)
    power = inspiral_power(n)
    hf = mf.HierarchicalFilter(n, nd, 1, snr=5.5, fd=1e-2)
    hf.set_reference(power)
    hf.set_data(noise(rng, (nd, n)))
    hf.set_templates(template_with_power(n, power)[None, :])
    peaks = hf.run(binsize=n, threshold=5.5)
    assert (peaks["index"] < 0).all()
    assert hf.refine_rate < 0.25


@pytest.mark.parametrize("coarse", ["fp32", "bf16x3"])
def test_omission_rate_meets_the_budget(coarse):
    """False dismissal within the budget fd, 16384 trials in one batched run
    (signals at exactly snr in the gate model's own complex noise).  The
    gate is the model's fd-quantile, so the measured rate is a binomial
    estimate around a true rate of at most fd: the bound allows three
    standard deviations of that estimate above fd (with ~8000 detections
    that is fd + 0.3 fd), no more."""
    mf = _mf()
    n, trials, snr, fd = 4096, 16384, 5.5, 1e-2
    rng = np.random.default_rng(13)
    power = inspiral_power(n)
    H = template_with_power(n, power)
    ph = np.exp(2j * np.pi * np.arange(n) / n)
    D = noise(rng, (trials, n))
    for i in range(trials):
        D[i] += (snr * H * ph ** ((37 * i) % n)).astype(np.complex64)
    flat = mf.MatchedFilter(n, trials, 1)
    hf = mf.HierarchicalFilter(n, trials, 1, snr=snr, fd=fd, band=512, coarse=coarse)
    hf.set_reference(power)
    for o in (flat, hf):
        o.set_data(D)
        o.set_templates(H[None, :])
    a = flat.run(binsize=n, threshold=snr).copy()
    b = hf.run(binsize=n, threshold=snr)
    det = a["index"][:, 0, 0] >= 0
    omitted = det & (b["index"][:, 0, 0] < 0)
    ndet = int(det.sum())
    assert ndet > 4000
    bound = fd * ndet + 3.0 * np.sqrt(fd * (1 - fd) * ndet)
    assert omitted.sum() <= bound, (int(omitted.sum()), ndet, bound)


def test_calibration_contract():
    mf = _mf()
    n = 1024
    hf = mf.HierarchicalFilter(n, 1, 1)
    with pytest.raises(ValueError):
        hf.set_coarse_threshold(3.0)          # explicit gate needs an explicit band
    rng = np.random.default_rng(14)
    hf.set_data(noise(rng, (1, n)))
    hf.set_templates(noise(rng, (1, n)))
    with pytest.raises(ValueError):
        hf.run(binsize=n)                     # no band, no reference
    hp = mf.HierarchicalFilter(n, 1, 1, band=128)
    hp.set_data(noise(rng, (1, n)))
    hp.set_templates(noise(rng, (1, n)))
    with pytest.raises(ValueError):
        hp.run(binsize=n)                     # pinned band, no gate and no reference
    hp.set_coarse_threshold(0.0)              # gate 0: every nonzero pair refines
    out = hp.run(binsize=256)
    assert (out["index"] >= 0).all()
    with pytest.raises(ValueError):
        mf.HierarchicalFilter(n, 1, 1, band=100)
    with pytest.raises(ValueError):
        hp.set_reference(np.zeros(n, np.float32))


@pytest.mark.parametrize("coarse,tol", [("bf16x3", 6e-5), ("fp16x3", 2e-5)])
def test_tensor_core_coarse_values_vs_fp64(coarse, tol):
    """Coarse maxima from the split-precision tensor-core contraction, against
    the FP64 coarse mirror.  Tolerance is relative to the pair's coarse
    scale (the largest |coarse z|): hi+lo BF16 keeps ~16 bits, FP16 ~22."""
    mf = _mf()
    from apogee_b200 import synthetic
    n, nd, nt, band = 4096, 5, 37, 512
    D, H, power, _ = synthetic.hier_workload(n, nd, nt, seed=5, frac=0.4)
    hf = mf.HierarchicalFilter(n, nd, nt, band=band, coarse=coarse)
    hf.set_reference(power)
    hf.set_coarse_threshold(1.0)
    hf.set_data(D)
    hf.set_templates(H)
    for window in (None, (100, 4000), (1234, 1300)):
        got = hf.coarse_values(window=window)
        want = oracle.coarse_max(D, H, band, power, window)
        err = np.abs(got - want) / np.maximum(want, 1e-30)
        assert err.max() < tol, (window, err.max())


def test_tensor_core_coarse_tail_pairs():
    """Pair counts that are not a multiple of the 8-pair tile."""
    mf = _mf()
    n, nd, nt, band = 4096, 3, 5, 512
    rng = np.random.default_rng(15)
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    hf = mf.HierarchicalFilter(n, nd, nt, band=band, coarse="bf16x3")
    hf.set_coarse_threshold(1.0)
    hf.set_data(D)
    hf.set_templates(H)
    got = hf.coarse_values()
    want = oracle.coarse_max(D, H, band)
    assert np.abs(got - want).max() < 1e-4 * want.max()


def test_band_selected_by_measured_cost():
    """band=None with a reference: every candidate band whose gate resolves is
    timed on the device with the caller's bank; the fastest is used, and the
    result keeps the hierarchical contract (reported peaks are the flat
    filter's)."""
    mf = _mf()
    n, nd, nt = 4096, 4, 64
    rng = np.random.default_rng(21)
    power = inspiral_power(n)
    H = np.stack([template_with_power(n, power) for _ in range(nt)])
    D = noise(rng, (nd, n))
    D[1] += (12.0 * H[5] * np.exp(2j * np.pi * np.arange(n) * 777 / n)).astype(np.complex64)
    hf = mf.HierarchicalFilter(n, nd, nt, snr=5.5, fd=1e-2, coarse="fp32")
    hf.set_reference(power)
    hf.set_templates(H)
    hf.set_data(D)
    b = hf.run(binsize=1024, threshold=5.5).copy()
    sel = hf.selection
    assert sel["band"] in sel["gates"] and sel["band"] == hf.config[0]
    assert set(sel["costs_us"]) == set(sel["gates"])
    if len(sel["gates"]) > 1:
        assert sel["costs_us"][sel["band"]] == min(sel["costs_us"].values())
    flat = mf.MatchedFilter(n, nd, nt)
    flat.set_data(D)
    flat.set_templates(H)
    a = flat.run(binsize=1024, threshold=5.5)
    fired = b["index"] >= 0
    assert fired[1, 5].any()
    np.testing.assert_array_equal(a["index"][fired], b["index"][fired])
    # the choice is kept until the bank or the reference changes
    hf.run(binsize=1024, threshold=5.5)
    assert hf.selection is sel
