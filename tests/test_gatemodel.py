"""The project's gate model against gate values the reference produced."""
import os

import numpy as np

from apogee_b200 import gatemodel


def test_gate_values_match_reference(golden_dir):
    rows = np.load(os.path.join(golden_dir, "gate.npz"))["rows"]
    for n, band, snr, fd, g in rows:
        n, band = int(n), int(band)
        p = np.zeros(n, np.float32)
        k = np.arange(1, n // 2).astype(np.float64)
        p[1:n // 2] = (k ** (-7 / 3.0) / ((0.015 * n / k) ** 4 + 1.0)).astype(np.float32)
        p /= p.sum()
        got = gatemodel.gate_for(p, n, band, snr, fd)
        if np.isnan(g):
            assert got is None
        else:
            assert got == g, (n, band, snr, fd, got, g)


def test_gate_validation():
    p = np.ones(1024, np.float32)
    for bad in [dict(band=100), dict(snr=-1.0), dict(fd=0.0), dict(fd=1.5)]:
        args = dict(band=128, snr=5.5, fd=1e-2)
        args.update(bad)
        try:
            gatemodel.gate_for(p, 1024, args["band"], args["snr"], args["fd"])
        except ValueError:
            continue
        raise AssertionError("accepted %r" % bad)
