"""Derive the coarse threshold of the hierarchical benchmark workload from the
FP64 oracle, so that the device run and the reference engine's run can be
given the same gate.

    python tests/golden/make_gate.py            # prints the gate, writes gate_config1.json

Workload: n = 4096, 16 x 1024 pairs, band 512 (1/8), snr 5.5, fd 1e-2, the
seed-1 bank of apogee_b200.synthetic.hier_workload and its reference profile
(mean |h|^2 over the bank).

Recipe (the quantity the reference's gate model estimates,
python/matchedfilter/gatemodel.py:210-227: the fd-quantile of the coarse
maximum over pairs whose full filter reaches snr), measured instead of
modelled: 8192 independent noise segments (real N(0,1) noise, the workload's
own noise model), each carrying one template of a 128-template sample of the
bank at a uniformly random lag and amplitude snr; a pair counts when its FP64
flat maximum exceeds snr, and its FP64 coarse maximum (the band-512 filter on
H[:512]/sqrt(f) over the widened coarse window, src/hmf.c:222-300) joins the
sample.  Same draws, in the same order, as HierarchicalFilter.calibrate(),
which does this with the device filters.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N, ND, NT, BAND, SNR, FD = 4096, 16, 1024, 512, 5.5, 1e-2
SEGMENTS, TEMPLATES, CHUNK, SEED = 8192, 128, 512, 20261203


def fp64_maxima(D, H, band, power):
    """(flat max |z| over all lags, coarse max |z| over the coarse window) per pair."""
    import scipy.fft as sf
    from oracle import oracle
    n = D.shape[1]
    D128 = D.astype(np.complex128)
    H128 = H.astype(np.complex128)
    ct = oracle.coarse_templates(H, band, power).astype(np.complex128)
    cs, ce = oracle.coarse_window(n, band, 0, n)
    fm = np.empty((D.shape[0], H.shape[0]))
    cm = np.empty_like(fm)
    for t0 in range(0, H.shape[0], 16):
        z = sf.ifft(D128[:, None, :] * np.conj(H128[None, t0:t0 + 16]), axis=-1, workers=-1) * n
        fm[:, t0:t0 + 16] = np.abs(z).max(-1)
        zc = sf.ifft(D128[:, None, :band] * np.conj(ct[None, t0:t0 + 16]), axis=-1,
                     workers=-1) * band
        cm[:, t0:t0 + 16] = np.abs(zc[..., cs:ce]).max(-1)
    return fm, cm


def derive_gate():
    from apogee_b200 import synthetic
    _, H, power, _ = synthetic.hier_workload(N, ND, NT, seed=1)
    rng = np.random.default_rng(SEED)
    tsel = np.sort(rng.choice(NT, size=TEMPLATES, replace=False))
    Hs = H[tsel]
    ph = np.arange(N)
    kept = []
    for _ in range(0, SEGMENTS, CHUNK):
        D = synthetic.noise_spectra(N, CHUNK, rng)
        inj = rng.integers(0, TEMPLATES, size=CHUNK)
        lag = rng.integers(0, N, size=CHUNK)
        D += SNR * Hs[inj].astype(np.complex128) * np.exp(-2j * np.pi * np.outer(lag, ph) / N)
        D = D.astype(np.complex64)
        fm, cm = fp64_maxima(D, Hs, BAND, power)
        kept.append(cm[fm > SNR])
    kept = np.sort(np.concatenate(kept))
    i = int(np.floor(FD * kept.size))
    return float(kept[i]), int(kept.size)


def main():
    gate, det = derive_gate()
    out = {"gate": gate, "detections": det, "n": N, "band": BAND, "snr": SNR, "fd": FD,
           "segments": SEGMENTS, "templates": TEMPLATES, "seed": SEED, "bank_seed": 1,
           "how": "FP64 oracle, tests/golden/make_gate.py"}
    with open(os.path.join(HERE, "gate_config1.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
