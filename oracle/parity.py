"""Parity comparison between device peaks and the FP64 oracle.

TEST INFRASTRUCTURE ONLY (the checker; never part of the product).

Bar (stated by the path's specification):
  * indices identical, except where the two candidates' FP64 magnitudes
    differ by less than RTOL_TIE (1e-5) relative -- a near tie, which either
    lag may win -- or where the bin's FP64 maximum is within RTOL_TIE of the
    threshold, so crossing is undecidable in float32;
  * values within RTOL_VAL (1e-5) relative of the FP64 value at the reported
    lag, plus an absolute floor of ATOL_FLOOR (1e-6) times the pair's largest
    |z|: an FP32 FFT's error is relative to the transform's scale, not to each
    small output (the reference's own direct-sum test uses 3e-6 of the max,
    tests/test_independent.py:55).
"""
import numpy as np

RTOL_TIE = 1e-5
RTOL_VAL = 1e-5
ATOL_FLOOR = 1e-6


def oracle_bins(z, binsize, threshold=0.0, win=None):
    """FP64 (index, max |z|) per bin, vectorised."""
    from .oracle import bin_edges
    n = z.shape[-1]
    edges = bin_edges(n, binsize, win)
    thr = float(threshold)
    t2 = thr * thr if thr > 0 else 0.0
    mag = np.abs(z)
    iref = np.full(z.shape[:-1] + (len(edges),), -1, np.int64)
    mref = np.zeros(iref.shape)
    for j, (lo, hi) in enumerate(edges):
        seg = mag[..., lo:hi]
        a = seg.argmax(-1)
        mx = np.take_along_axis(seg, a[..., None], -1)[..., 0]
        mref[..., j] = mx
        iref[..., j] = np.where(mx * mx > t2, lo + a, -1)
    return iref, mref, edges


def compare(idx, val, z, binsize, threshold=0.0, win=None, *, rows_mask=None):
    """Return a list of mismatch descriptions (empty = parity).

    idx/val: device result [..., nb]; z: FP64 correlation [..., n] with the
    same leading shape.  rows_mask (optional, leading shape) restricts the
    check to those rows (e.g. fired pairs of the hierarchical filter)."""
    idx = np.asarray(idx).astype(np.int64)
    val = np.asarray(val).astype(np.complex128)
    n = z.shape[-1]
    iref, mref, edges = oracle_bins(z, binsize, threshold, win)
    thr = float(threshold)
    mag = np.abs(z)
    scale = mag.max(-1)[..., None]
    sel = np.ones(idx.shape, bool) if rows_mask is None else \
        np.broadcast_to(np.asarray(rows_mask)[..., None], idx.shape)
    bad = []
    # values at the device's lag
    safe = np.clip(idx, 0, n - 1)
    zdev = np.take_along_axis(z, safe, -1)
    mdev = np.abs(zdev)
    lo = np.array([e[0] for e in edges])
    hi = np.array([e[1] for e in edges])
    inbin = (idx >= lo) & (idx < hi)
    same = idx == iref
    tie = (idx >= 0) & (iref >= 0) & inbin & (np.abs(mdev - mref) <= RTOL_TIE * mref)
    edge_miss = (idx < 0) & (iref >= 0) & ((mref <= thr * (1 + RTOL_TIE)) |
                                          (mref * mref <= np.finfo(np.float32).tiny))
    edge_extra = (idx >= 0) & (iref < 0) & inbin & (mdev >= thr * (1 - RTOL_TIE))
    index_ok = same | tie | edge_miss | edge_extra
    for pos in zip(*np.nonzero(sel & ~index_ok)):
        bad.append("row %s bin %d: index %d, oracle %d (|z| %.9g vs %.9g)"
                   % (pos[:-1], pos[-1], idx[pos], iref[pos], mdev[pos] if idx[pos] >= 0 else -1,
                      mref[pos]))
    neg = sel & index_ok & (idx < 0) & (val != 0)
    for pos in zip(*np.nonzero(neg)):
        bad.append("row %s bin %d: index -1 with value %r" % (pos[:-1], pos[-1], val[pos]))
    vbad = sel & index_ok & (idx >= 0) & (np.abs(val - zdev) > RTOL_VAL * mdev + ATOL_FLOOR * scale)
    for pos in zip(*np.nonzero(vbad)):
        bad.append("row %s bin %d lag %d: value %r, oracle %r (rel %.3g)"
                   % (pos[:-1], pos[-1], idx[pos], val[pos], zdev[pos],
                      abs(val[pos] - zdev[pos]) / max(abs(zdev[pos]), 1e-300)))
        if len(bad) > 50:
            break
    return bad
