"""Coarse-gate threshold from the reference power profile.

Restates the reference's Monte-Carlo gate model
(python/matchedfilter/gatemodel.py:63-227), which has to stay alike because
the threshold it returns is part of the hierarchical filter's contract: the
same profile, band, snr and budget must give the same gate.

Model.  With q the normalised profile and f its in-band fraction, the
filter output at lag tau has signal rho*A(tau - L) and noise covariance
A(t1 - t2), A(d) = sum_k q_k exp(2 pi i k d / n).  The coarse stage sees
only the in-band part, A_b, of both.  For every sub-grid offset of the lag,
draw complex Gaussian noise with those covariances (Cholesky in FP64,
draws in FP32), form the coarse maximum over the coarse grid lags and the
fine maximum over nearby integer lags, keep the coarse maxima of draws
whose fine maximum reaches snr, and return their fd-quantile.

gate_for(..., device=k) runs the numerics on GPU k (FP64 sums, covariances
and Cholesky factors, FP32 transforms and maxima; gate_kernels.cuh) with the
same draws; without `device` they run here in numpy.

Noise convention: Re and Im of the output each have variance 1, so a
complex draw normalised to E|z|^2 = 1 is scaled by sqrt(2)
(gatemodel.py:26-31,40-45).
"""
from collections import OrderedDict

import numpy as np

COARSE_LAGS = 4       # coarse grid lags either side of the signal
FINE_LAGS = 3         # integer lags either side
NOISE_SCALE = np.sqrt(2.0)
SEED = 13

_cache = OrderedDict()
_CACHE_ENTRIES = 64


def _lag_table(x, n):
    """n * IFFT(x): A(d) for every integer lag d."""
    return np.fft.ifft(x) * n


def _chol32(table, lags):
    c = table[lags % len(table)]
    c = (c + c.conj().T) / 2 + 1e-9 * np.eye(c.shape[0])
    return np.linalg.cholesky(c).astype(np.complex64)


def _draw(rng, m, k):
    re = rng.standard_normal((m, k), dtype=np.float32)
    im = rng.standard_normal((m, k), dtype=np.float32)
    return (re + 1j * im) / np.float32(np.sqrt(2))


def joint_maxima(power, n, band, snr, nsamp, seed=SEED):
    """(coarse max, fine max) for nsamp draws, or None for an empty band."""
    q = np.asarray(power, dtype=np.float64)
    total = q.sum()
    if total <= 0:
        return None
    q = q / total
    f = min(max(float(q[:band].sum()), 0.0), 1.0)
    if f == 0:
        return None
    step = n // band
    in_band = np.zeros(n, dtype=np.float64)
    in_band[:band] = q[:band] / f
    A_full = _lag_table(q, n)
    A_band = _lag_table(in_band, n)
    has_out = (1.0 - f) > 1e-9
    A_out = (A_full - f * A_band) / (1.0 - f) if has_out else None
    grid = np.arange(-COARSE_LAGS, COARSE_LAGS + 1) * step
    rng = np.random.default_rng(seed)
    per = max(nsamp // step, 256)
    coarse, fine = [], []
    for off in range(step):
        taus = np.unique(np.concatenate([np.arange(-FINE_LAGS, FINE_LAGS + 1) + off, grid]))
        on_grid = np.searchsorted(taus, grid)
        lags = taus[:, None] - taus[None, :]
        noise_in = (_draw(rng, per, len(taus)) @ _chol32(A_band, lags).T) * np.float32(NOISE_SCALE)
        if has_out:
            noise_out = (_draw(rng, per, len(taus)) @ _chol32(A_out, lags).T) \
                * np.float32(NOISE_SCALE)
        else:
            noise_out = np.float32(0.0)
        s_full = A_full[(taus - off) % n].astype(np.complex64)
        s_band = A_band[(taus - off) % n].astype(np.complex64)
        fine.append(np.abs(np.float32(snr) * s_full[None, :]
                           + np.float32(np.sqrt(f)) * noise_in
                           + np.float32(np.sqrt(1 - f)) * noise_out).max(1))
        coarse.append(np.abs(np.float32(snr * np.sqrt(f)) * s_band[None, :]
                             + noise_in)[:, on_grid].max(1))
    return np.concatenate(coarse), np.concatenate(fine)


GRID_POINTS = 2 * COARSE_LAGS + 1
MAX_TAUS = 16


def joint_maxima_device(power, n, band, snr, nsamp, seed=SEED, device=0):
    """joint_maxima with its numerics on the GPU (mfb_gate_maxima): FP64
    profile sums, lag covariances and Cholesky factors, FP32 noise transforms
    and maxima.  The draws are the same seeded numpy stream, drawn here in the
    same order, so the estimator is the host one draw for draw."""
    import ctypes
    from . import _lib
    q = np.asarray(power, dtype=np.float64)
    total = q.sum()
    if total <= 0:
        return None
    q = q / total
    f = min(max(float(q[:band].sum()), 0.0), 1.0)
    if f == 0:
        return None
    step = n // band
    has_out = (1.0 - f) > 1e-9
    grid = np.arange(-COARSE_LAGS, COARSE_LAGS + 1) * step
    rng = np.random.default_rng(seed)
    per = max(nsamp // step, 256)
    taus_all = np.zeros((step, MAX_TAUS), np.int32)
    ntaus = np.zeros(step, np.int32)
    on_grid = np.zeros((step, GRID_POINTS), np.int32)
    d_in = np.zeros((step, per, MAX_TAUS), np.complex64)
    d_out = np.zeros((step, per, MAX_TAUS), np.complex64) if has_out else None
    for off in range(step):
        taus = np.unique(np.concatenate([np.arange(-FINE_LAGS, FINE_LAGS + 1) + off, grid]))
        k = len(taus)
        taus_all[off, :k] = taus
        ntaus[off] = k
        on_grid[off] = np.searchsorted(taus, grid)
        d_in[off, :, :k] = _draw(rng, per, k)
        if has_out:
            d_out[off, :, :k] = _draw(rng, per, k)
    coarse = np.empty(step * per, np.float32)
    fine = np.empty(step * per, np.float32)
    sums = np.empty(2, np.float64)
    q64 = np.ascontiguousarray(q, dtype=np.float64)
    _lib.check(_lib.lib().mfb_gate_maxima(
        int(device), q64.ctypes.data, n, band, float(snr), step, per, int(has_out),
        taus_all.ctypes.data, ntaus.ctypes.data, on_grid.ctypes.data, d_in.ctypes.data,
        None if d_out is None else d_out.ctypes.data, coarse.ctypes.data, fine.ctypes.data,
        sums.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "gate model failed")
    return coarse, fine


def kept_coarse(power, n, band, snr, nsamp, seed=SEED, device=None):
    """Sorted coarse maxima of the draws the fine stage keeps (cached);
    `device` (a CUDA ordinal) runs the numerics there."""
    p = np.asarray(power, dtype=np.float64)
    if (p.shape != (n,) or not np.isfinite(p).all() or (p < 0).any() or p.sum() <= 0):
        raise ValueError("power must be a finite nonnegative length-n profile with positive sum")
    p = p / p.sum()
    key = (p.tobytes(), n, band, float(snr), nsamp, seed, device)
    if key in _cache:
        _cache.move_to_end(key)
        return _cache[key]
    if device is None:
        got = joint_maxima(p, n, band, snr, nsamp, seed)
    else:
        got = joint_maxima_device(p, n, band, snr, nsamp, seed, device)
    if got is None:
        return None
    c, fmax = got
    kept = np.sort(c[fmax >= snr])
    _cache[key] = kept
    while len(_cache) > _CACHE_ENTRIES:
        _cache.popitem(last=False)
    return kept


def samples_for(fd):
    """Draws so that about 100 kept samples fall below the fd-quantile."""
    fd = max(float(fd), 1e-6)
    return int(min(max(2.0e4, 200.0 / fd), 3.0e6))


def _validate(n, band, snr, fd):
    if (not isinstance(n, (int, np.integer)) or n < 64 or not isinstance(band, (int, np.integer))
            or band < 1 or band > n or band & (band - 1) or n % band):
        raise ValueError("n must be divisible by a power-of-two band <= n")
    if not np.isfinite(snr) or snr <= 0:
        raise ValueError("snr must be finite and positive")
    if not np.isfinite(fd) or not 0 < fd < 1:
        raise ValueError("fd must be finite and between zero and one")


def gate_for(power, n, band, snr, fd, device=None):
    """Largest coarse threshold whose modelled dismissal meets fd, or None
    when the draws cannot resolve the budget.  With `device` (a CUDA ordinal)
    the FP64 covariance work and the FP32 draws run on that GPU."""
    _validate(n, band, snr, fd)
    nsamp = samples_for(fd)
    if fd * nsamp < 8:
        return None
    kept = kept_coarse(power, n, band, snr, nsamp, device=device)
    if kept is None or not len(kept):
        return None
    i = int(np.floor(float(fd) * len(kept)))
    if i < 8:
        return None
    return float(kept[i])


def dismissal(power, n, band, snr, gate, fd_hint=1e-3):
    """Modelled false-dismissal rate at a given coarse threshold."""
    _validate(n, band, snr, fd_hint)
    if not np.isfinite(gate) or gate < 0:
        raise ValueError("gate must be finite and nonnegative")
    kept = kept_coarse(power, n, band, snr, samples_for(fd_hint))
    if kept is None or not len(kept):
        return None
    return float(np.searchsorted(kept, float(gate)) / len(kept))
