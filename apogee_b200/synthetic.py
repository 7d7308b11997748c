"""Seeded synthetic workloads for the benchmark and tests.

No public dataset is involved: these generators stand in for the reference's
matched-profile inspiral bank (python/matchedfilter/benchmark.py:336;
tests/test_api.py:26-46) with the shapes and value distributions of the
benchmark configurations.

Templates: h_k = k^(-7/6) exp(i(2 pi k t_c / n + alpha k^(-5/3))) on bins
kmin..kmax, zero elsewhere, Hermitian-filled (h_{n-k} = conj(h_k), so the
time-domain template is real), each normalised to unit L2 over all n bins;
alpha ~ U[1e2, 1e4], t_c ~ U[0, n).

Data: spectrum of N(0,1) real white noise scaled by 1/sqrt(n), so the
filter output noise has unit variance and SNR is in units of that sigma
(the reference's own tests use per-bin complex N(0,1)+iN(0,1) instead,
tests/test_api.py:53-55).  An injection of template t* at lag tau and SNR A
adds A * h_{t*} * exp(-2 pi i k tau / n), which peaks at lag tau with value A.
Both sides are exactly Hermitian: the negative frequencies are written as
the conjugates of the positive ones.
"""
import numpy as np


def template_bank(n, nt, rng, kmin=20, kmax=None):
    kmax = n // 2 - 1 if kmax is None else int(kmax)
    k = np.arange(kmin, kmax + 1, dtype=np.float64)
    alpha = rng.uniform(1e2, 1e4, size=(nt, 1))
    tc = rng.uniform(0, n, size=(nt, 1))
    half = k ** (-7.0 / 6.0) * np.exp(1j * (2 * np.pi * k * tc / n + alpha * k ** (-5.0 / 3.0)))
    H = np.zeros((nt, n), np.complex128)
    H[:, kmin:kmax + 1] = half
    H[:, n - kmax:n - kmin + 1] = np.conj(half[:, ::-1])
    H /= np.linalg.norm(H, axis=1, keepdims=True)
    return H.astype(np.complex64)


def template_bank_torch(n, alpha, tc, kmin=20, kmax=None):
    """template_bank's formula in torch, differentiable in ``alpha`` and ``tc``
    (1-D tensors of one value per template); float64 parameters give
    complex128 templates [nt][n]."""
    import torch
    kmax = n // 2 - 1 if kmax is None else int(kmax)
    k = torch.arange(kmin, kmax + 1, dtype=alpha.dtype, device=alpha.device)
    phase = 2 * torch.pi * k * tc[:, None] / n + alpha[:, None] * k ** (-5.0 / 3.0)
    amp = k ** (-7.0 / 6.0)
    half = torch.polar(amp.expand_as(phase), phase)
    nt = alpha.shape[0]

    def zeros(width):
        return torch.zeros(nt, width, dtype=half.dtype, device=half.device)

    # bins: [0, kmin) zero | [kmin, kmax] half | (kmax, n-kmax) zero
    #       | [n-kmax, n-kmin] conjugate mirror | (n-kmin, n) zero
    mirror = torch.conj(torch.flip(half, dims=[1]))
    H = torch.cat([zeros(kmin), half, zeros(n - 2 * kmax - 1), mirror, zeros(kmin - 1)], dim=1)
    return H / torch.linalg.vector_norm(H, dim=1, keepdim=True)


def noise_spectra(n, nd, rng):
    """FFT of real N(0,1) noise / sqrt(n), exactly Hermitian."""
    x = rng.standard_normal((nd, n))
    half = np.fft.rfft(x, axis=1) / np.sqrt(n)
    D = np.zeros((nd, n), np.complex128)
    D[:, :n // 2 + 1] = half
    D[:, n // 2 + 1:] = np.conj(half[:, 1:n // 2][:, ::-1])
    D[:, 0] = D[:, 0].real
    D[:, n // 2] = D[:, n // 2].real
    return D


def inject(D, H, d, t, lag, snr):
    n = D.shape[1]
    k = np.arange(n)
    D[d] += snr * H[t].astype(np.complex128) * np.exp(-2j * np.pi * k * lag / n)


def flat_workload(n=4096, nd=16, nt=1024, seed=0, n_injected=2, snr=8.0):
    """Flat benchmark workload: noise data with `n_injected` segments carrying
    a random template at a random lag and fixed SNR."""
    rng = np.random.default_rng(seed)
    H = template_bank(n, nt, rng)
    D = noise_spectra(n, nd, rng)
    inj = []
    for d in rng.choice(nd, size=n_injected, replace=False):
        t, lag = int(rng.integers(nt)), int(rng.integers(n))
        inject(D, H, d, t, lag, snr)
        inj.append((int(d), t, lag, snr))
    return D.astype(np.complex64), H, inj


def hier_data(H, nd, rng, frac=0.10, snr_lo=5.0, snr_hi=12.0):
    """Noise data for the bank H: `frac` of the nd segments (at least one)
    carry a random template of H at a random lag and SNR U[snr_lo, snr_hi].
    Returns (D complex64 [nd][n], injections [(d, t, lag, snr)])."""
    nt, n = H.shape
    D = noise_spectra(n, nd, rng)
    k = max(1, int(round(frac * nd)))
    inj = []
    for d in rng.choice(nd, size=k, replace=False):
        t, lag = int(rng.integers(nt)), int(rng.integers(n))
        snr = float(rng.uniform(snr_lo, snr_hi))
        inject(D, H, d, t, lag, snr)
        inj.append((int(d), t, lag, snr))
    return D.astype(np.complex64), inj


def hier_workload(n=4096, nd=16, nt=1024, seed=1, frac=0.10, snr_lo=5.0, snr_hi=12.0):
    """Hierarchical benchmark workload: noise data, `frac` of the segments
    carry an injection at SNR U[snr_lo, snr_hi]; the reference profile is the
    mean |h|^2 over the bank."""
    rng = np.random.default_rng(seed)
    H = template_bank(n, nt, rng)
    D, inj = hier_data(H, nd, rng, frac, snr_lo, snr_hi)
    power = (np.abs(H.astype(np.complex128)) ** 2).mean(0).astype(np.float32)
    return D, H, power, inj


def batched_workload(njobs=256, seed=2, device="cuda", nmin_log=10, nmax_log=16, nd_max=64,
                     nt_min=16, nt_max=4096, cap_bytes=2 << 30, series_every=4, inject_every=8,
                     snr=8.0):
    """Uneven jobs for the batched launch, generated on the device.

    Job i: n = 2^U{nmin_log..nmax_log}, nd ~ U{1..nd_max}, nt ~ U{nt_min..nt_max}
    capped so that nt*n*8 <= cap_bytes, binsize n/16 or n/64; templates by the
    template_bank formula (bins 20..n/2-1) drawn from the seed; every
    `series_every`-th job is a series job (float32 N(0,1) samples cut into nd
    back-to-back blocks of n), the others take noise spectra (FFT of N(0,1)
    / sqrt(n)) with every `inject_every`-th row carrying a template at a
    random lag and SNR `snr`.  Returns a list of batch.Job on `device`.
    """
    import torch
    from .batch import Job
    rng = np.random.default_rng(seed)
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(seed)
    jobs = []
    for i in range(njobs):
        n = 1 << int(rng.integers(nmin_log, nmax_log + 1))
        nd = int(rng.integers(1, nd_max + 1))
        nt = int(min(rng.integers(nt_min, nt_max + 1), cap_bytes // (8 * n)))
        binsize = n // int(rng.choice([16, 64]))
        alpha = torch.tensor(rng.uniform(1e2, 1e4, size=nt), dtype=torch.float64, device=dev)
        tc = torch.tensor(rng.uniform(0, n, size=nt), dtype=torch.float64, device=dev)
        H = torch.empty(nt, n, dtype=torch.complex64, device=dev)
        chunk = max(1, (1 << 25) // n)
        for t0 in range(0, nt, chunk):
            H[t0:t0 + chunk] = template_bank_torch(n, alpha[t0:t0 + chunk],
                                                   tc[t0:t0 + chunk]).to(torch.complex64)
        if series_every and i % series_every == series_every - 1:
            x = torch.randn(nd * n, dtype=torch.float32, device=dev, generator=gen)
            jobs.append(Job(H, series=x, starts=np.arange(nd) * n, binsize=binsize))
        else:
            D = torch.fft.fft(torch.randn(nd, n, dtype=torch.float32, device=dev, generator=gen),
                              dim=1) / float(np.sqrt(n))
            k = torch.arange(n, device=dev, dtype=torch.float64)
            for d in range(0, nd, inject_every):
                t, lag = int(rng.integers(nt)), int(rng.integers(n))
                D[d] += (snr * H[t].to(torch.complex128) *
                         torch.exp(-2j * np.pi * k * lag / n)).to(torch.complex64)
            jobs.append(Job(H, data=D.to(torch.complex64).contiguous(), binsize=binsize))
    return jobs


def large_workload(n=262144, nd=4, nt=2048, seed=1, device="cuda", frac=0.05, snr_lo=6.0,
                   snr_hi=15.0, materialize=None, chunk=64):
    """Large-transform bank: templates by the template_bank formula on bins
    20..n/2-1, generated on the device; noise data (FFT(N(0,1))/sqrt(n)) with
    `frac` of the segments (at least one) carrying a template at a random lag
    and SNR U[snr_lo, snr_hi]; reference profile = mean |h|^2 over the bank.

    materialize: None (every template) or a sequence of template indices to
    return (a subsample of the same bank: the draws, the data and the profile
    are those of the full bank).  Returns (D [nd][n] complex64, H [k][n]
    complex64, power [n] float32, injections [(d, t, lag, snr)]) on `device`.
    """
    import torch
    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    alpha = torch.tensor(rng.uniform(1e2, 1e4, size=nt), dtype=torch.float64, device=dev)
    tc = torch.tensor(rng.uniform(0, n, size=nt), dtype=torch.float64, device=dev)
    rows = list(range(nt)) if materialize is None else [int(t) for t in materialize]
    pos = {t: i for i, t in enumerate(rows)}
    H = torch.empty(len(rows), n, dtype=torch.complex64, device=dev)
    power = torch.zeros(n, dtype=torch.float64, device=dev)
    for t0 in range(0, nt, chunk):
        blk = template_bank_torch(n, alpha[t0:t0 + chunk], tc[t0:t0 + chunk]).to(torch.complex64)
        power += (blk.abs().to(torch.float64) ** 2).sum(0)
        for t in range(t0, min(t0 + chunk, nt)):
            if t in pos:
                H[pos[t]] = blk[t - t0]
    power = (power / nt).to(torch.float32)
    D = torch.from_numpy(noise_spectra(n, nd, rng)).to(dev)
    k = torch.arange(n, device=dev, dtype=torch.float64)
    inj = []
    for d in rng.choice(nd, size=max(1, int(round(frac * nd))), replace=False):
        t, lag, snr = int(rng.integers(nt)), int(rng.integers(n)), float(rng.uniform(snr_lo, snr_hi))
        ht = template_bank_torch(n, alpha[t:t + 1], tc[t:t + 1])[0]
        D[d] += snr * ht.to(torch.complex64).to(torch.complex128) * \
            torch.exp(-2j * np.pi * k * lag / n)
        inj.append((int(d), t, lag, snr))
    return D.to(torch.complex64), H, power, inj
