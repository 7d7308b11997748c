"""Sharding the pair space across GPUs, one process per GPU.

Pairs are independent, so the template bank is split into contiguous slices,
one per rank: every rank holds all data rows and its own templates, filters
its slice on its own GPU, and writes the rows ``[:, t0:t0+count, :]`` of the
peak table.  Nothing crosses NVLink on the data path; assembling the full
table where a caller wants it is one all-gather of the 16-byte peak records
(NCCL between GPUs, gloo between CPU processes), and the hierarchical
filter's (pairs, triggers) statistics are summed with one all-reduce.

The reference runs one plan per process and leaves distribution to the
caller; this is the layout its multi-device use implies
(python/matchedfilter/__init__.py:253-259 picks one device per plan).
"""
import numpy as np

PEAK_DTYPE = np.dtype([("index", "<i8"), ("value", "<c8")])


def template_slice(nt, rank, world):
    """Contiguous slice ``(t0, count)`` of ``nt`` templates for ``rank``:
    sizes differ by at most one, lower ranks take the extra ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    if nt < 0:
        raise ValueError("nt must be nonnegative")
    base, extra = divmod(int(nt), int(world))
    t0 = rank * base + min(rank, extra)
    return t0, base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist
    return dist


def all_gather_records(local, nt_total, group=None):
    """Assemble the full ``(nd, nt_total, nb, 2)`` int64 record table (the
    PEAK_DTYPE bytes: index, value bits) from every rank's ``(nd, count, nb,
    2)`` slice, where the slice already lives: a CUDA tensor for NCCL groups
    (one all-gather over NVLink, the table stays on the device, no host
    copy), a CPU tensor for gloo.  Slices are padded to the largest one."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if local.dtype != torch.int64 or local.dim() != 4 or local.shape[3] != 2:
        raise TypeError("local must be an int64 (nd, count, nb, 2) record tensor")
    nd, cnt, nb, _ = local.shape
    want = template_slice(nt_total, rank, world)[1]
    if cnt != want:
        raise ValueError("rank %d holds %d templates; its slice has %d" % (rank, cnt, want))
    maxc = template_slice(nt_total, 0, world)[1]
    padded = local.new_zeros((nd, maxc, nb, 2))
    padded[:, :cnt] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([parts[r][:, :template_slice(nt_total, r, world)[1]]
                      for r in range(world)], dim=1)


def all_gather_peaks(local, nt_total, group=None):
    """all_gather_records for a numpy PEAK_DTYPE ``(nd, count, nb)`` slice
    (a host result): the exchange runs on the rank's current CUDA device for
    NCCL groups, on the CPU for gloo; returns the numpy table."""
    import torch
    dist = _dist()
    local = np.ascontiguousarray(local)
    if local.dtype != PEAK_DTYPE or local.ndim != 3:
        raise TypeError("local must be a (nd, count, nb) PEAK_DTYPE array")
    nd, cnt, nb = local.shape
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    if not local.flags.writeable:               # a hierarchical run's host table
        local = local.copy()
    words = torch.from_numpy(local.view(np.int64).reshape(nd, cnt, nb, 2)).to(dev)
    full = all_gather_records(words, nt_total, group)
    return full.cpu().numpy().view(PEAK_DTYPE).reshape(nd, nt_total, nb)


def all_reduce_stats(pairs, triggers, group=None):
    """Sum the hierarchical filters' (pairs, triggers) over the ranks."""
    import torch
    dist = _dist()
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.tensor([int(pairs), int(triggers)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, group=group)
    return int(t[0].item()), int(t[1].item())


class ShardedFilter:
    """A matched (or hierarchical) filter whose template bank is split over
    the ranks of ``group``.

    engine(n, ndata, count) builds the rank-local filter; the default is
    ``MatchedFilter`` (``kind="flat"``) or ``HierarchicalFilter``
    (``kind="hier"``, keyword arguments passed on) on this rank's current
    CUDA device.  ``set_templates`` takes the full bank (or just this rank's
    slice), ``run`` returns the full ``(nd, nt, nb)`` table on every rank.
    """

    def __init__(self, n, ndata, ntemplates, group=None, kind="flat", engine=None, **kw):
        dist = _dist()
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.n, self.ndata, self.ntemplates = int(n), int(ndata), int(ntemplates)
        self.t0, self.count = template_slice(self.ntemplates, self.rank, self.world)
        if self.count < 1:
            raise ValueError("%d templates cannot give every one of %d ranks a template"
                             % (self.ntemplates, self.world))
        if engine is None:
            import torch
            import apogee_b200 as mf
            dev = "gpu:%d" % torch.cuda.current_device()
            cls = mf.HierarchicalFilter if kind == "hier" else mf.MatchedFilter
            self.local = cls(self.n, self.ndata, self.count, device=dev, **kw)
        else:
            self.local = engine(self.n, self.ndata, self.count)

    def set_data(self, spectra):
        self.local.set_data(spectra)

    def set_templates(self, spectra):
        """The full bank (ntemplates rows) or this rank's slice (count rows)."""
        rows = spectra.shape[0]
        if rows == self.ntemplates:
            spectra = spectra[self.t0:self.t0 + self.count]
        elif rows != self.count:
            raise ValueError("expected %d (bank) or %d (slice) template rows, got %d"
                             % (self.ntemplates, self.count, rows))
        self.local.set_templates(spectra)

    def run(self, binsize=None, threshold=0.0, window=None):
        part = self.local.run(binsize=binsize, threshold=threshold, window=window)
        return all_gather_peaks(np.asarray(part), self.ntemplates, self.group)

    def run_records(self, binsize=None, threshold=0.0, window=None):
        """The full table as device records on every rank (NCCL): the rank's
        slice from ``run_records`` of its filter, gathered in place."""
        part = self.local.run_records(binsize=binsize, threshold=threshold, window=window)
        return all_gather_records(part, self.ntemplates, self.group)

    @property
    def stats(self):
        """(pairs, triggers) summed over the ranks (hierarchical filters)."""
        p, t = self.local.stats
        return all_reduce_stats(p, t, self.group)
