"""Band selection for the hierarchical filter from costs measured on the GPU.

The reference picks the cheapest configuration whose model gate resolves the
requested budget, with costs read from tables measured on other machines
(``choose_config``, python/matchedfilter/__init__.py:1040-1054; ``cost.txt``,
``cost-<arch>.txt``; ``cost_table_for``, :807-827: "Cost is a property of the
machine").  Here the costs are measured on the device the filter runs on, at
plan time, with the caller's own template bank:

for every candidate band (a power of two, 64 <= band <= min(n/2, 16384),
that the coarse kind supports) whose gate the model resolves, a plan at that
band runs the whole hierarchical step -- coarse pass, gate at the model's
threshold, refine of what passes -- on the caller's own data bank, and CUDA
events time it.  The refine rate, and so the cost, depends on the data as much
as on the band (the model gate resolves the false-dismissal budget for signals
at snr, not a noise rate), which is why the caller's data is used.  The
fastest band wins; ties go to the wider band.

Results are cached per (device, n, ndata, ntemplates, kind, snr, fd,
reference, template bank) for the process: a choice measured on one data
bank of a stream is kept for the next ones.
"""
import hashlib

import numpy as np

_CACHE = {}

#: Timed repetitions per candidate (after one warm-up run).
REPS = 3

#: Widest coarse band: the coarse pass is the single-CTA filter at length band.
MAX_BAND = 16384


def candidate_bands(n, kind_supports_band):
    """Bands the reference's tables span at this n, narrowest first."""
    return [b for b in (n // 16, n // 8, n // 4, n // 2)
            if 64 <= b <= MAX_BAND and kind_supports_band(b)]


def pick(measured):
    """The band with the smallest measured time; ties to the wider band.

    measured: {band: microseconds}.  Raises if empty."""
    if not measured:
        raise ValueError("no candidate band to choose from")
    return min(measured, key=lambda b: (measured[b], -b))


def _key(hf, candidates):
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(hf._pending_ref).tobytes())
    t = hf._gt
    # the bank enters through its size and a sample of rows (first, middle, last)
    for r in sorted({0, t.shape[0] // 2, t.shape[0] - 1}):
        h.update(t[r].cpu().numpy().tobytes())
    return (hf.device.index, hf.n, hf.ndata, hf.ntemplates, hf._coarse,
            hf._fs_snr or hf.snr, hf.fd, tuple(candidates), h.hexdigest())


def measure(hf, gates):
    """Microseconds of one hierarchical step per candidate band.

    hf: the HierarchicalFilter being configured (templates and data set);
    gates: {band: model gate}.  Returns {band: (us, refine_rate)}."""
    import torch
    from . import HierarchicalFilter
    kind = hf._coarse
    dev = torch.device("cuda", hf.device.index)
    D = hf._gd if hf._hostdata is None else torch.from_numpy(hf._hostdata).to(dev)
    out = {}
    for band, gate in gates.items():
        p = HierarchicalFilter(hf.n, hf.ndata, hf.ntemplates, snr=hf.snr, fd=hf.fd, band=band,
                               device="gpu:%d" % hf.device.index, coarse=kind)
        p.set_coarse_threshold(float(gate))
        p.set_templates(hf._gt)
        p.set_data(D)
        p.run_device(binsize=hf.n, threshold=0.0)        # warm-up (plan, constants)
        torch.cuda.synchronize(dev)
        p0 = p.stats
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(REPS):
            p.run_device(binsize=hf.n, threshold=0.0)
        b.record()
        torch.cuda.synchronize(dev)
        p1 = p.stats
        us = a.elapsed_time(b) * 1e3 / REPS
        rate = (p1[1] - p0[1]) / max(1, p1[0] - p0[0])
        out[band] = (us, rate)
        del p
    return out


def choose(hf, gates):
    """Band for `hf` among {band: gate} (resolvable candidates), measured on
    its device and cached; returns (band, {band: (us, refine_rate)})."""
    if len(gates) == 1:
        (band,) = gates
        return band, {}
    key = _key(hf, sorted(gates))
    hit = _CACHE.get(key)
    if hit is not None:
        return hit
    costs = measure(hf, gates)
    band = pick({b: c[0] for b, c in costs.items()})
    _CACHE[key] = (band, costs)
    return band, costs
