"""FP64 CPU oracle for the fused matched-filter hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.

Restates, in numpy float64, the reference's semantics for this path:
  * correlation z[k] = sum_f D[f] conj(H[f]) exp(+2 pi i f k/n), unnormalised
    (python/matchedfilter/matchedfilter.h:35-52; src/matchfilt.c:207-209);
  * bins nb = ceil((end-start)/binsize) over the clamped window, bin j =
    lags [start + j*binsize, min(start+(j+1)*binsize, end))
    (src/dispatch.c:62-67; python/matchedfilter/_core.c:29-43);
  * a bin reports the lag of max |z|^2 iff |z|^2 > thr^2 (thr <= 0: > 0), the
    lowest lag among exact ties, else (-1, 0) (src/balanced-inl.h:804-969);
  * hierarchical coarse pass = the same filter at length band on
    H[:band] / sqrt(f), one bin over the coarse window widened by one sample,
    fire iff the coarse max is reported and >= the coarse threshold, refine
    fired pairs with the full filter (src/hmf.c:118-156, 222-328);
  * run_series block spectra FFT(series[s:s+n] / n), zero-padded
    (src/matchfilt.c:437-490).
Pinned against the reference's own compiled CPU engine (oracle/_ref, see
oracle/Makefile.ref) and the fixtures in tests/golden/.
"""
import numpy as np


def correlate(D, H):
    """z[d, t, k] in complex128 for D [nd, n], H [nt, n]."""
    D = np.asarray(D).astype(np.complex128)
    H = np.asarray(H).astype(np.complex128)
    n = D.shape[-1]
    return np.fft.ifft(D[:, None, :] * np.conj(H[None, :, :]), axis=-1) * n


def direct_correlation(d, h):
    """O(n^2) definition, no FFT: z[k] = sum_f d[f] conj(h[f]) e^{2 pi i f k / n}."""
    d = np.asarray(d).astype(np.complex128)
    h = np.asarray(h).astype(np.complex128)
    n = d.shape[-1]
    f = np.arange(n)
    w = np.exp(2j * np.pi * np.outer(f, f) / n)
    return (d * np.conj(h)) @ w


def window(n, win):
    if win is None:
        return 0, n
    s, e = max(0, min(int(win[0]), n)), max(0, min(int(win[1]), n))
    if s >= e:
        raise ValueError("empty window")
    return s, e


def bin_edges(n, binsize, win=None):
    s, e = window(n, win)
    nb = (e - s + binsize - 1) // binsize
    return [(s + j * binsize, min(s + (j + 1) * binsize, e)) for j in range(nb)]


def binned_peaks(z, binsize, threshold=0.0, win=None):
    """Per-bin argmax of |z|^2 over the last axis with the reference's rules.

    Returns (index int64, value complex128, counts int32)."""
    n = z.shape[-1]
    edges = bin_edges(n, binsize, win)
    t2 = threshold * threshold if threshold > 0 else 0.0
    m2 = z.real ** 2 + z.imag ** 2
    idx = np.full(z.shape[:-1] + (len(edges),), -1, np.int64)
    val = np.zeros(idx.shape, np.complex128)
    for j, (lo, hi) in enumerate(edges):
        seg = m2[..., lo:hi]
        a = seg.argmax(-1)                       # first maximum = lowest lag
        mx = np.take_along_axis(seg, a[..., None], -1)[..., 0]
        ok = mx > t2
        idx[..., j] = np.where(ok, lo + a, -1)
        val[..., j] = np.where(ok, np.take_along_axis(z[..., lo:hi], a[..., None], -1)[..., 0], 0)
    return idx, val, (idx >= 0).sum(-1).astype(np.int32)


def flat(D, H, binsize=None, threshold=0.0, win=None):
    n = np.asarray(D).shape[-1]
    z = correlate(D, H)
    return binned_peaks(z, n if binsize is None else int(binsize), threshold, win) + (z,)


def band_fraction(H, band, reference=None):
    """f per template, as float32 (src/hmf.c:125-153): the reference's in-band
    fraction of its total, or each template's own, with FP64 sums."""
    H = np.asarray(H)
    if reference is not None:
        p = np.asarray(reference, np.float64)
        f = np.float32(p[:band].sum() / p.sum())
        return np.full(H.shape[0], f, np.float32)
    p = np.abs(H.astype(np.complex128)) ** 2
    tot = p.sum(-1)
    low = p[:, :band].sum(-1)
    return np.where(tot > 0, (low / np.where(tot > 0, tot, 1)), 0).astype(np.float32)


def coarse_templates(H, band, reference=None):
    """ct = (float)(H[:band] * (1/sqrt(f))) with the scale in double."""
    f = band_fraction(H, band, reference).astype(np.float64)
    sc = np.where(f > 0, 1.0 / np.sqrt(np.where(f > 0, f, 1)), 0.0)
    Hb = np.asarray(H)[:, :band]
    re = (Hb.real.astype(np.float64) * sc[:, None]).astype(np.float32)
    im = (Hb.imag.astype(np.float64) * sc[:, None]).astype(np.float32)
    return (re + 1j * im).astype(np.complex64)


def coarse_window(n, band, start, end):
    """Coarse window on the R = n/band grid, widened by one sample (src/hmf.c:233-239)."""
    R = n // band
    cs = start // R
    ce = min((end + R - 1) // R, band)
    if cs > 0:
        cs -= 1
    return cs, ce


def coarse_max(D, H, band, reference=None, win=None):
    """Maximum |coarse z| per pair over the coarse window, float64 [nd, nt]."""
    n = np.asarray(D).shape[-1]
    s, e = window(n, win)
    cs, ce = coarse_window(n, band, s, e)
    ct = coarse_templates(H, band, reference)
    zc = correlate(np.asarray(D)[:, :band], ct)
    return np.abs(zc[..., cs:ce]).max(-1)


def hier(D, H, band, coarse_threshold, binsize=None, threshold=0.0, win=None, reference=None,
         coarse=None):
    """Reference hierarchical result: (idx, val, fired, z).  `coarse` may supply
    precomputed coarse maxima (e.g. from another precision) for the gate."""
    n = np.asarray(D).shape[-1]
    idx, val, cnt, z = flat(D, H, binsize, threshold, win)
    cm = coarse_max(D, H, band, reference, win) if coarse is None else coarse
    thr = float(coarse_threshold)
    t2 = thr * thr if thr > 0 else 0.0
    fired = (cm * cm > t2) & (cm >= thr)
    idx = np.where(fired[..., None], idx, -1)
    val = np.where(fired[..., None], val, 0)
    return idx, val, fired, z


def series_spectra(series, starts, n):
    """FFT(series[s:s+n] / n) per block, zero-padded past the end (complex128)."""
    series = np.asarray(series).astype(np.complex128)
    out = np.zeros((len(starts), n), np.complex128)
    for b, s in enumerate(starts):
        blk = np.zeros(n, np.complex128)
        seg = series[int(s):int(s) + n]
        blk[:seg.size] = seg
        out[b] = np.fft.fft(blk / n)
    return out
