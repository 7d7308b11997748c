"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Run in a container where the reference source tree is present and
oracle/_ref has been built from it (make -f oracle/Makefile.ref):

    python tests/golden/make_golden.py /path/to/reference

Outputs (small .npz files, committed):
  flat.npz    seeded inputs and the reference engine's peaks
              (python/matchedfilter/_core.c MF.run over src/matchfilt.c)
  ties.npz    exact-tie cases of tests/test_cpu_single_peak.py, answered by
              the reference engine
  hier.npz    the reference hierarchical engine (src/hmf.c) with a pinned band
              and coarse threshold
  series.npz  the reference run_series (src/matchfilt.c:437-490)
  gate.npz    gate thresholds from the reference gate model
              (python/matchedfilter/gatemodel.py:210)
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import refcore  # noqa: E402


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def inspiral_power(n, exponent=-7 / 3.0, knee_frac=0.0150):
    p = np.zeros(n, dtype=np.float32)
    k = np.arange(1, n // 2).astype(np.float64)
    p[1:n // 2] = (k ** exponent / ((knee_frac * n / k) ** 4 + 1.0)).astype(np.float32)
    return p / p.sum()


FLAT_CASES = [
    # n, nd, nt, seed, binsize, threshold, window
    (64, 2, 3, 1, 64, 0.0, None),
    (64, 2, 3, 2, 17, 0.0, (3, 60)),
    (256, 2, 3, 3, 16, 0.0, None),
    (256, 2, 3, 4, 1, 0.0, None),
    (1024, 2, 3, 5, 64, 0.0, None),
    (1024, 2, 3, 6, 100, 40.0, (7, 1000)),
    (4096, 2, 2, 7, 256, 0.0, None),
    (4096, 2, 2, 8, 4096, 0.0, None),
    (4096, 2, 2, 9, 333, 120.0, (11, 4090)),
    (16384, 1, 2, 10, 1024, 0.0, None),
]


def make_flat(out):
    arrays = {}
    for c, (n, nd, nt, seed, bs, thr, win) in enumerate(FLAT_CASES):
        rng = np.random.default_rng(seed)
        D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
        f = refcore.RefFlat(n, nd, nt)
        f.set_data(D)
        f.set_templates(H)
        idx, val, cnt, _ = f.run(binsize=bs, threshold=thr, window=win)
        arrays.update({"c%d_D" % c: D, "c%d_H" % c: H, "c%d_idx" % c: idx,
                       "c%d_val" % c: val, "c%d_cnt" % c: cnt,
                       "c%d_par" % c: np.array([n, nd, nt, seed, bs, thr,
                                                -1 if win is None else win[0],
                                                -1 if win is None else win[1]], np.float64)})
    arrays["ncases"] = np.array(len(FLAT_CASES))
    np.savez_compressed(out, **arrays)


def make_ties(out):
    """DC-only product: equal magnitude at every lag (test_cpu_single_peak.py:7-35).

    As in that test, MF_PBMAX=1024 selects the reference's pair-batched CPU
    path, whose scan reports the lowest tied lag -- the tie rule this project
    implements.  (The reference's balanced path reports the first maximum in
    its own SIMD scan order instead, which is not the lowest lag.)"""
    os.environ["MF_PBMAX"] = "1024"
    arrays, c = {}, 0
    for n in (64, 256, 1024):
        data = np.zeros((3, n), np.complex64)
        data[:, 0] = [3 + 4j, -5j, 0]
        tm = np.zeros((5, n), np.complex64)
        tm[:, 0] = 1
        f = refcore.RefFlat(n, 3, 5)
        f.set_data(data)
        f.set_templates(tm)
        for lo, hi in ((0, n), (7, n - 9), (11, 12)):
            for bs in (hi - lo, 17, n + 3):
                for thr in (0.0, 4.0, 5.0, 6.0):
                    idx, val, cnt, _ = f.run(binsize=bs, threshold=thr, window=(lo, hi))
                    arrays["c%d_idx" % c] = idx
                    arrays["c%d_val" % c] = val
                    arrays["c%d_par" % c] = np.array([n, lo, hi, bs, thr])
                    c += 1
    arrays["ncases"] = np.array(c)
    np.savez_compressed(out, **arrays)
    del os.environ["MF_PBMAX"]


HIER_CASES = [
    # n, nd, nt, band, seed, snr, fd, binsize, threshold
    (1024, 4, 4, 128, 21, 5.5, 1e-2, 256, 5.5),
    (4096, 4, 4, 512, 22, 5.5, 1e-2, 1024, 5.5),
    (4096, 3, 5, 256, 23, 5.0, 1e-3, 4096, 5.0),
]


def make_hier(out, gate_for):
    arrays = {}
    for c, (n, nd, nt, band, seed, snr, fd, bs, thr) in enumerate(HIER_CASES):
        rng = np.random.default_rng(seed)
        power = inspiral_power(n)
        h = np.sqrt(power).astype(np.complex64)
        h /= np.linalg.norm(h)
        H = np.stack([h * np.exp(2j * np.pi * rng.uniform() * np.arange(n) / n).astype(np.complex64)
                      for _ in range(nt)]).astype(np.complex64)
        D = (noise(rng, (nd, n)))
        for d in range(nd):
            if d % 2 == 0:
                lag = int(rng.integers(0, n))
                D[d] += (12.0 * H[d % nt] * np.exp(2j * np.pi * np.arange(n) * lag / n)
                         ).astype(np.complex64)
        gate = gate_for(power, n, band, snr, fd)
        r = refcore.RefHier(n, nd, nt, band, gate, reference=power, snr=snr, fd=fd)
        r.set_data(D)
        r.set_templates(H)
        idx, val = r.run(binsize=bs, threshold=thr)
        pairs, trig = r.stats()
        arrays.update({"c%d_D" % c: D, "c%d_H" % c: H, "c%d_power" % c: power,
                       "c%d_idx" % c: idx, "c%d_val" % c: val,
                       "c%d_par" % c: np.array([n, nd, nt, band, seed, snr, fd, bs, thr, gate,
                                                pairs, trig], np.float64)})
    arrays["ncases"] = np.array(len(HIER_CASES))
    np.savez_compressed(out, **arrays)


def make_series(out):
    rng = np.random.default_rng(31)
    n, nt = 1024, 3
    H = noise(rng, (nt, n))
    series = noise(rng, 5000)
    starts = np.array([0, 512, 1024, 1536, 2048, 2560, 3072, 3584, 4096], np.uintp)
    ws = np.full(starts.size, 100, np.uintp)
    we = np.full(starts.size, 900, np.uintp)
    f = refcore.RefFlat(n, 4, nt)
    f.set_templates(H)
    idx, val = f.run_series(series, starts, ws, we, binsize=200, threshold=0.0)
    np.savez_compressed(out, H=H, series=series, starts=starts, ws=ws, we=we, idx=idx, val=val,
                        par=np.array([n, nt, 200, 0.0]))


def make_gate(out, gate_for):
    rows = []
    for n in (1024, 4096):
        p = inspiral_power(n)
        for band in (n // 8, n // 4):
            for snr, fd in ((5.5, 1e-2), (5.0, 1e-3), (6.0, 1e-2)):
                g = gate_for(p, n, band, snr, fd)
                rows.append([n, band, snr, fd, np.nan if g is None else g])
    np.savez_compressed(out, rows=np.array(rows))


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference tree>")
    ref = sys.argv[1]
    spec = importlib.util.spec_from_file_location(
        "ref_gatemodel", os.path.join(ref, "python", "matchedfilter", "gatemodel.py"))
    gm = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gm)
    make_flat(os.path.join(HERE, "flat.npz"))
    make_ties(os.path.join(HERE, "ties.npz"))
    make_hier(os.path.join(HERE, "hier.npz"), gm.gate_for)
    make_series(os.path.join(HERE, "series.npz"))
    make_gate(os.path.join(HERE, "gate.npz"), gm.gate_for)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
