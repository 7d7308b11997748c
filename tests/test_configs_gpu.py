"""Parity at the benchmark configurations' own shapes and generators.

Every number the benchmark reports rests on these: the flat filter at the
full 16 x 1024 bank (n = 4096, many pairs per persistent CTA, data rows
switching), the split-precision hierarchical filter at the same shape with
the model gate and the calibrated gate, a subsample of the n = 262144 bank,
and a seeded draw of uneven batched jobs (series jobs included).  The checker
is the FP64 oracle (oracle/oracle.py) and, where it runs in seconds, the
reference's own CPU engine built from its sources (oracle/_ref).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def fp64_chunks(D, H, chunk=128):
    """Yield (t0, z) with z the FP64 correlation of D against H[t0:t0+chunk]."""
    for t0 in range(0, H.shape[0], chunk):
        yield t0, oracle.correlate(D, H[t0:t0 + chunk])


def check_rows(idx, val, D, H, binsize, threshold, win=None, rows_mask=None):
    bad = []
    for t0, z in fp64_chunks(D, H):
        m = None if rows_mask is None else rows_mask[:, t0:t0 + z.shape[1]]
        bad += parity.compare(idx[:, t0:t0 + z.shape[1]], val[:, t0:t0 + z.shape[1]], z,
                              binsize, threshold, win, rows_mask=m)
        if len(bad) > 20:
            break
    return bad


def fp64_detections(D, H, binsize, threshold):
    """Per (d, t, bin): the FP64 bin maximum of |z| exceeds threshold."""
    det = np.zeros((D.shape[0], H.shape[0], D.shape[1] // binsize), bool)
    for t0, z in fp64_chunks(D, H):
        m = np.abs(z).reshape(z.shape[0], z.shape[1], -1, binsize).max(-1)
        det[:, t0:t0 + z.shape[1]] = m > threshold
    return det


# ------------------------------------------------------------------ config 0
def test_flat_full_bank_config0():
    """n = 4096, 16 x 1024 pairs, binsize 256, threshold 0, the flat
    generator (2 of 16 segments injected at SNR 8): every bin against FP64,
    and 64 templates against the reference engine."""
    import apogee_b200 as mf
    from apogee_b200 import synthetic
    D, H, inj = synthetic.flat_workload(4096, 16, 1024, seed=0)
    f = mf.MatchedFilter(4096, 16, 1024)
    f.set_data(D)
    f.set_templates(H)
    out = f.run(binsize=256, threshold=0.0).copy()
    bad = check_rows(out["index"], out["value"], D, H, 256, 0.0)
    assert not bad, bad[:5]
    # the injections are found near their lags (the template's main lobe is
    # a few lags wide, so noise moves the maximum by a lag or two) at ~SNR 8
    for d, t, lag, snr in inj:
        b = lag // 256
        assert abs(int(out["index"][d, t, b]) - lag) <= 8
        assert abs(abs(out["value"][d, t, b]) - snr) < 1.0
    from oracle import refcore
    if refcore.available():
        r = refcore.RefFlat(4096, 16, 64)
        r.set_data(D)
        r.set_templates(H[:64])
        ridx, rval, _, _ = r.run(binsize=256, threshold=0.0)
        z = oracle.correlate(D, H[:64])
        assert not parity.compare(ridx, rval, z, 256, 0.0)      # the reference meets the bar
        diff = ridx != out["index"][:, :64]
        if diff.any():
            # only FP64 near-ties may differ
            mag = np.abs(z)
            for d, t, b in zip(*np.nonzero(diff)):
                a, c = mag[d, t, ridx[d, t, b]], mag[d, t, out["index"][d, t, b]]
                assert abs(a - c) <= 1e-5 * max(a, c), (d, t, b)


@pytest.mark.parametrize("n,nd,nt,binsize,threshold,window", [
    (4096, 7, 333, 300, 3.0, (100, 3950)),    # general bin layout, many pairs per CTA
    (4096, 9, 400, 256, 4.0, None),           # whole-window fast layout with a threshold
    (1024, 9, 500, 64, 2.5, None),            # four pairs per CTA
    (16384, 3, 130, 1000, 3.5, (17, 16000)),  # one pair per CTA, odd bins
])
def test_flat_many_pairs_per_cta(n, nd, nt, binsize, threshold, window):
    """nd * nt far above the 296 persistent CTAs: each CTA walks many
    templates on one register-cached data row and switches rows."""
    import apogee_b200 as mf
    from apogee_b200 import synthetic
    rng = np.random.default_rng(n + nd + nt)
    H = synthetic.template_bank(n, nt, rng)
    D = synthetic.noise_spectra(n, nd, rng)
    for d in range(0, nd, 3):
        synthetic.inject(D, H, d, int(rng.integers(nt)), int(rng.integers(n)), 9.0)
    D = D.astype(np.complex64)
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    out = f.run(binsize=binsize, threshold=threshold, window=window)
    assert (out["index"] >= 0).any() and (out["index"] < 0).any()
    bad = check_rows(out["index"], out["value"], D, H, binsize, threshold, window)
    assert not bad, bad[:5]


# ------------------------------------------------------------------ config 1
def calibrated_gate():
    with open(os.path.join(HERE, "golden", "gate_config1.json")) as fh:
        return json.load(fh)["gate"]


@pytest.fixture(scope="module")
def config1():
    from apogee_b200 import synthetic
    D, H, power, inj = synthetic.hier_workload(4096, 16, 1024, seed=1)
    det = fp64_detections(D, H, 256, 5.5)
    cm = oracle.coarse_max(D, H, 512, power)
    return D, H, power, det, cm


@pytest.mark.parametrize("gate", ["model", "calibrated"])
@pytest.mark.parametrize("coarse", ["bf16x3", "fp16x3"])
def test_hier_full_bank_config1(config1, gate, coarse):
    """16 x 1024 pairs, band 512, split-precision tensor-core coarse pass:
    fired rows are the flat filter's rows bit for bit and meet the FP64 bar,
    dismissed rows are empty, coarse maxima match FP64, and the omission of
    FP64 detections stays within fd = 1e-2."""
    import apogee_b200 as mf
    D, H, power, det, cm64 = config1
    hf = mf.HierarchicalFilter(4096, 16, 1024, snr=5.5, fd=1e-2, band=512, coarse=coarse)
    hf.set_reference(power)
    hf.set_templates(H)
    hf.set_data(D)
    if gate == "calibrated":
        hf.set_coarse_threshold(calibrated_gate())
    g = hf._coarse_value(512)
    out = hf.run(binsize=256, threshold=5.5).copy()
    cv = hf.coarse_values()
    rel = np.abs(cv - cm64) / np.maximum(cm64, 1e-30)
    assert rel.max() < 2e-5, rel.max()
    flat = mf.MatchedFilter(4096, 16, 1024)
    flat.set_data(D)
    flat.set_templates(H)
    fout = flat.run(binsize=256, threshold=5.5)
    fired = (cv >= g) & (cv > 0)
    assert hf.last_refinements == int(fired.sum())
    np.testing.assert_array_equal(out[fired], fout[fired])
    assert (out["index"][~fired] == -1).all() and (out["value"][~fired] == 0).all()
    bad = check_rows(out["index"], out["value"], D, H, 256, 5.5, rows_mask=fired)
    assert not bad, bad[:5]
    omitted = det & (out["index"] < 0)
    assert det.sum() > 100
    assert omitted.sum() <= 1e-2 * det.sum(), (omitted.sum(), det.sum())
    # the fired set is the FP64 gate's, except within float rounding of the gate
    fired64 = cm64 >= g
    flip = fired != fired64
    assert (np.abs(cm64[flip] - g) <= 2e-5 * g).all()


def test_hier_full_bank_against_reference_engine(config1):
    """The reference's own hierarchical engine at the same shape, band and
    gate (FP32 coarse pass there, split BF16 here): identical tables except
    pairs whose coarse maximum sits within rounding of the gate."""
    from oracle import refcore
    if not refcore.available():
        pytest.skip("reference engine not built")
    import apogee_b200 as mf
    D, H, power, det, cm64 = config1
    gate = calibrated_gate()
    hf = mf.HierarchicalFilter(4096, 16, 1024, snr=5.5, fd=1e-2, band=512, coarse="bf16x3")
    hf.set_reference(power)
    hf.set_templates(H)
    hf.set_data(D)
    hf.set_coarse_threshold(gate)
    out = hf.run(binsize=256, threshold=5.5).copy()
    r = refcore.RefHier(4096, 16, 1024, 512, gate, reference=power, snr=5.5, fd=1e-2)
    r.set_templates(H)
    r.set_data(D)
    ridx, rval = r.run(binsize=256, threshold=5.5)
    rows_ours = (out["index"] >= 0).any(-1)
    rows_ref = (ridx >= 0).any(-1)
    flip = rows_ours != rows_ref
    assert (np.abs(cm64[flip] - gate) <= 2e-5 * gate).all()
    both = rows_ours & rows_ref
    assert both.sum() > 50
    # where both refined, both tables meet the FP64 bar (they may differ only
    # at FP64 near-ties)
    bad = check_rows(ridx, rval, D, H, 256, 5.5, rows_mask=both)
    assert not bad, ("reference engine", bad[:5])
    bad = check_rows(out["index"], out["value"], D, H, 256, 5.5, rows_mask=both)
    assert not bad, bad[:5]


# ------------------------------------------------------------------ config 4
def test_large_bank_subsample_config4():
    """n = 262144, 4 data rows of the 4 x 2048 bank's generator, 32 of its
    templates (the injected one included): flat against FP64, hierarchical
    (band n/16, FP32 coarse, fd 1e-3) rows equal to the flat rows where
    refined, and the injected detection kept."""
    import torch
    import apogee_b200 as mf
    from apogee_b200 import synthetic
    n, nt_bank = 262144, 2048
    # which template is injected: draw the workload once without templates
    _, _, _, inj = synthetic.large_workload(n, 4, nt_bank, seed=1, materialize=[])
    rng = np.random.default_rng(5)
    inj_t = sorted({t for _, t, _, _ in inj})
    others = [t for t in rng.choice(nt_bank, size=40, replace=False) if t not in inj_t]
    sel = sorted(inj_t + others[:32 - len(inj_t)])
    D, H, power, inj = synthetic.large_workload(n, 4, nt_bank, seed=1, materialize=sel)
    Dn, Hn, pn = D.cpu().numpy(), H.cpu().numpy(), power.cpu().numpy()
    binsize, thr = 4096, 6.0
    f = mf.MatchedFilter(n, 4, len(sel))
    f.set_data(D)
    f.set_templates(H)
    out = f.run(binsize=binsize, threshold=thr).copy()
    bad = []
    for t0 in range(0, len(sel), 8):
        z = oracle.correlate(Dn, Hn[t0:t0 + 8])
        bad += parity.compare(out["index"][:, t0:t0 + 8], out["value"][:, t0:t0 + 8], z,
                              binsize, thr)
    assert not bad, bad[:5]
    lobe = n // 2048                 # the main lobe widens with n (64 lags here)
    for d, t, lag, snr in inj:
        assert abs(int(out["index"][d, sel.index(t), lag // binsize]) - lag) <= lobe
    hf = mf.HierarchicalFilter(n, 4, len(sel), snr=6.0, fd=1e-3, band=n // 16, coarse="fp32")
    hf.set_reference(pn)
    hf.set_templates(H)
    hf.set_data(D)
    hout = hf.run(binsize=binsize, threshold=thr).copy()
    rows = (hout["index"] >= 0).any(-1)
    np.testing.assert_array_equal(hout[rows], out[rows])
    for d, t, lag, snr in inj:
        assert abs(int(hout["index"][d, sel.index(t), lag // binsize]) - lag) <= lobe
    del f, hf
    torch.cuda.empty_cache()


# ------------------------------------------------------------------ config 2
def test_batched_seeded_draw_config2():
    """A seeded 32-job draw of the batched generator (n = 2^10 .. 2^16,
    every 4th job a float32 series): a seeded subsample of each job's pairs
    against FP64."""
    import torch
    from apogee_b200 import synthetic
    from apogee_b200 import PEAK_DTYPE
    from apogee_b200.batch import BatchedFilter
    jobs = synthetic.batched_workload(njobs=32, seed=11, device="cuda")
    assert any(j.series is not None for j in jobs)
    bf = BatchedFilter(jobs)
    bf.run()
    bf.wait()
    rng = np.random.default_rng(3)
    for i, j in enumerate(jobs):
        ds = np.sort(rng.choice(j.nd, size=min(3, j.nd), replace=False))
        ts = np.sort(rng.choice(j.nt, size=min(4, j.nt), replace=False))
        Hs = j.templates[torch.as_tensor(ts, device=j.templates.device)].cpu().numpy()
        if j.data is not None:
            Ds = j.data[torch.as_tensor(ds, device=j.data.device)].cpu().numpy()
        else:
            x = j.series.cpu().numpy()
            Ds = oracle.series_spectra(x, j.starts.astype(np.int64)[ds], j.n)
        z = oracle.correlate(Ds, Hs)
        rec = bf.records(i).view(j.nd, j.nt, j.nb, 2)
        rec = rec[torch.as_tensor(ds, device=rec.device)][:, torch.as_tensor(ts, device=rec.device)]
        r = rec.contiguous().cpu().numpy().view(PEAK_DTYPE)[..., 0]
        bad = parity.compare(r["index"], r["value"], z, j.binsize, j.threshold,
                             (j.start, j.end))
        assert not bad, (i, j.n, j.nd, j.nt, bad[:3])
    bf.close()
    del jobs
    torch.cuda.empty_cache()
