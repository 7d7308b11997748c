"""Many uneven matched-filter jobs in one persistent launch.

``BatchedFilter(jobs)`` plans a list of :class:`Job` -- each its own n (any
supported power of two), data rows or a time series cut into blocks,
templates, binsize, threshold and window -- for ONE persistent kernel launch
(``mfb_batch_*`` in include/mfb.h): CTAs take tickets from one queue, the
single-CTA jobs (n <= 4096) run the fused filter, the larger ones the
four-step split through L2-sized scratch slots, and series jobs first
transform their blocks.  ``run()`` enqueues that launch; ``capture()``
records it in a CUDA graph that ``replay()`` re-launches.  The split of each
large n, the pairs per ticket of each small n, come from the defaults or
from :mod:`apogee_b200.autotune`.

A job can instead run as its own launches, with the kernels specialised for
its n (the single-CTA filter with 512 or 1024 threads at n = 8192 / 16384,
the two-pass kernels above), in the same stream and the same graph, writing
the same records: ``tune={n: {"dedicated": True}}`` forces that, and the
autotuner measures both forms per n and sends a job to its own launches when
the time it saves per pair, times its pairs, exceeds the cost of a launch
(``DEDICATED_LAUNCH_US``).  The persistent launch keeps the jobs too small to
fill the GPU on their own.

Each job's result is the reference's peak table for that job
(``MatchedFilter.run`` / ``run_series``, python/matchedfilter/__init__.py:
435-514, 561-688): a ``(nd, nt, nb)`` PEAK_DTYPE array with ``(-1, 0)`` below
threshold.  The reference has no batched form; it runs one plan per shape.
"""
import ctypes

import numpy as np

from . import _lib

PEAK_DTYPE = np.dtype([("index", "<i8"), ("value", "<c8")])

#: Cost charged to a job run as its own launches: the launch itself and the
#: partial last wave of its grid, which the persistent launch would fill with
#: other jobs' work (microseconds; B200 measurement order of magnitude).
DEDICATED_LAUNCH_US = 10.0


def dedicated(job, cfg):
    """True if ``job`` runs as its own launches under configuration ``cfg``."""
    if cfg.get("dedicated"):
        return True
    pp, dp = cfg.get("pp_us"), cfg.get("dedicated_pp_us")
    if pp is None or dp is None:
        return False
    return job.pairs * (float(pp) - float(dp)) > DEDICATED_LAUNCH_US


def _torch():
    import torch
    return torch


def _device_complex(a, dev):
    """A contiguous complex64 CUDA tensor of `a` (numpy, torch, real or complex)."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a
    else:
        arr = np.asarray(a)
        if not np.iscomplexobj(arr):
            arr = arr.astype(np.float32).astype(np.complex64)
        t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.complex64))
    if not t.is_complex():
        t = t.to(torch.float32).to(torch.complex64)
    return t.to(device=dev, dtype=torch.complex64).contiguous()


class Job:
    """One job of a batch.

    templates : [nt][n] template spectra.
    data      : [nd][n] data spectra; or
    series, starts : a time series (real or complex) and the block starts;
              block b is series[starts[b] : starts[b] + n], zero past the end,
              transformed to FFT(block / n) as run_series does.
    binsize, threshold, window : as MatchedFilter.run (window shared by
              every row or block).
    """

    def __init__(self, templates, data=None, series=None, starts=None, binsize=None,
                 threshold=0.0, window=None):
        if (data is None) == (series is None):
            raise ValueError("a job takes either data spectra or a series with block starts")
        if series is not None and starts is None:
            raise ValueError("a series job needs its block starts")
        self.templates = templates
        self.data = data
        self.series = series
        shape = tuple(templates.shape)
        if len(shape) != 2:
            raise ValueError("templates must be two-dimensional (nt, n)")
        self.nt, self.n = int(shape[0]), int(shape[1])
        if self.n < 64 or self.n & (self.n - 1) or self.n > (1 << 20):
            raise ValueError("n must be a power of two from 64 to 2^20, got %d" % self.n)
        if data is not None:
            if tuple(data.shape)[1:] != (self.n,) or len(data.shape) != 2:
                raise ValueError("data must be (nd, %d)" % self.n)
            self.nd = int(data.shape[0])
            self.starts = None
        else:
            self.starts = np.ascontiguousarray(np.asarray(starts, dtype=np.int64))
            if self.starts.ndim != 1 or self.starts.size < 1 or np.any(self.starts < 0):
                raise ValueError("starts must be a nonempty 1-D array of nonnegative offsets")
            self.starts = self.starts.astype(np.uint64)
            self.nd = int(self.starts.size)
        if self.nd < 1 or self.nt < 1:
            raise ValueError("a job needs at least one data row and one template")
        self.binsize = self.n if binsize is None else int(binsize)
        if self.binsize < 1:
            raise ValueError("binsize must be >= 1")
        if window is None:
            self.start, self.end = 0, self.n
        else:
            s, e = int(window[0]), int(window[1])
            self.start, self.end = max(0, min(s, self.n)), max(0, min(e, self.n))
            if self.start >= self.end:
                raise ValueError("empty window (%d, %d)" % (self.start, self.end))
        self.threshold = float(threshold)
        b = min(self.binsize, self.n)
        self.nb = -(-(self.end - self.start) // b)
        if self.n > 4096 and self.nb > 4096:
            raise ValueError("jobs with n > 4096 take at most 4096 bins per pair (got %d)" % self.nb)

    @property
    def pairs(self):
        return self.nd * self.nt


class BatchedFilter:
    """Plan ``jobs`` for one persistent launch on a CUDA device.

    tune : False (``autotune.default``: the B200 measurements), True
           (autotune every distinct n, cached per device), or a dict
           {n: {"split": N2} | {"unit_items": k} | {"dedicated": True}}.
    slot_bytes, slots : scratch of the large-n four-step (0 = 64 MiB x 3).
    """

    def __init__(self, jobs, device=None, tune=False, slot_bytes=0, slots=0):
        from .device import parse
        torch = _torch()
        self.device = parse(device)
        self._dev = torch.device("cuda", self.device.index)
        self.jobs = list(jobs)
        if not self.jobs:
            raise ValueError("no jobs")
        from . import autotune
        if tune is True:
            self.config = {n: autotune.tune(n, device=self.device)
                           for n in sorted({j.n for j in self.jobs})}
        elif isinstance(tune, dict):
            self.config = dict(tune)
        else:
            self.config = {n: autotune.default(n) for n in sorted({j.n for j in self.jobs})}
        self._hold = []
        self._records = []
        self._plan = None
        self._graph = None
        self._own = []          # jobs on their own launches: (index, plan, device buffers)
        persist = []
        for i, j in enumerate(self.jobs):
            rec = torch.empty(j.pairs * j.nb * 2, dtype=torch.int64, device=self._dev)
            self._records.append(rec)
            if dedicated(j, self.config.get(j.n, {})):
                self._own.append(self._own_launches(i, j, rec))
            else:
                persist.append(i)
        torch.cuda.synchronize(self._dev)     # own plans' template copies are done
        for own in self._own:
            own["keep"] = []
        if not persist:
            return
        arr = (_lib.MfbJob * len(persist))()
        for slot, i in enumerate(persist):
            j = self.jobs[i]
            c = arr[slot]
            c.n, c.nd, c.nt = j.n, j.nd, j.nt
            h = _device_complex(j.templates, self._dev)
            self._hold.append(h)
            c.templates = h.data_ptr()
            if j.data is not None:
                d = _device_complex(j.data, self._dev)
                self._hold.append(d)
                c.data = d.data_ptr()
            else:
                s = _device_complex(j.series, self._dev).reshape(-1)
                self._hold.append(s)
                c.series = s.data_ptr()
                c.nseries = s.numel()
                c.starts = j.starts.ctypes.data
            c.binsize, c.threshold, c.start, c.end = j.binsize, j.threshold, j.start, j.end
            c.records = self._records[i].data_ptr()
            cfg = self.config.get(j.n, {})
            c.split = int(cfg.get("split", 0))
            c.unit_items = int(cfg.get("unit_items", 0))
        opts = _lib.MfbBatchOpts(int(slot_bytes), int(slots))
        plan = ctypes.c_void_p()
        L = _lib.lib()
        _lib.check(L.mfb_batch_create(ctypes.byref(plan), self.device.index, arr, len(persist),
                                      ctypes.byref(opts)), "batch plan failed")
        self._plan = plan

    def _own_launches(self, i, j, rec):
        """A plan of job j's own (templates and data copied in once); a series
        job keeps its samples, block starts and a spectra buffer on the device
        and transforms them at every run (mfb_forward, then mfb_set_data)."""
        torch = _torch()
        L = _lib.lib()
        plan = ctypes.c_void_p()
        _lib.check(L.mfb_create(ctypes.byref(plan), j.n, j.nd, j.nt, self.device.index),
                   "batch job plan failed")
        own = {"index": i, "plan": plan, "keep": []}
        try:
            _lib.check(L.mfb_set_stream(plan, self._stream()))
            h = _device_complex(j.templates, self._dev)
            _lib.check(L.mfb_set_templates(plan, 0, j.nt, h.data_ptr()))
            own["keep"].append(h)             # until the copy is done (constructor syncs)
            if j.data is not None:
                d = _device_complex(j.data, self._dev)
                _lib.check(L.mfb_set_data(plan, 0, j.nd, d.data_ptr()))
                own["keep"].append(d)
            else:
                ser = _device_complex(j.series, self._dev).reshape(-1)
                st = torch.from_numpy(j.starts.astype(np.int64)).to(self._dev)
                spec = torch.empty(j.nd, j.n, dtype=torch.complex64, device=self._dev)
                own["series"] = (ser, st, spec)
        except Exception:
            L.mfb_destroy(plan)
            raise
        own["rec"] = rec
        return own

    def _run_own(self, own, stream):
        L = _lib.lib()
        j = self.jobs[own["index"]]
        plan = own["plan"]
        _lib.check(L.mfb_set_stream(plan, stream))
        if "series" in own:
            ser, st, spec = own["series"]
            _lib.check(L.mfb_forward(plan, ser.data_ptr(), ser.numel(), st.data_ptr(), j.nd,
                                     spec.data_ptr()), "batch job forward failed")
            _lib.check(L.mfb_set_data(plan, 0, j.nd, spec.data_ptr()))
        _lib.check(L.mfb_run_records(plan, 0, j.nd, 0, j.nt, j.binsize, j.threshold, j.start,
                                     j.end, own["rec"].data_ptr(), None),
                   "batch job run failed")

    # ---- launching -----------------------------------------------------------
    def _stream(self):
        return _torch().cuda.current_stream(self._dev).cuda_stream

    def run(self):
        """Enqueue the persistent launch, then the jobs on their own launches,
        on torch's current stream."""
        stream = self._stream()
        if self._plan is not None:
            _lib.check(_lib.lib().mfb_batch_run(self._plan, stream), "batch run failed")
        for own in self._own:
            self._run_own(own, stream)

    def wait(self):
        """Synchronise and raise if a dependency wait of the last run ran out."""
        if self._plan is not None:
            _lib.check(_lib.lib().mfb_batch_status(self._plan, self._stream()),
                       "batch run failed")
        else:
            _torch().cuda.current_stream(self._dev).synchronize()

    def capture(self):
        """Record run() in a CUDA graph (replay() re-launches it)."""
        torch = _torch()
        if self._own:
            self.run()                        # first use sizes the own plans' workspaces
            self.wait()
        torch.cuda.synchronize(self._dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self._graph = g
        return g

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()

    # ---- results ---------------------------------------------------------------
    def records(self, i):
        """Job i's result on the device: int64 tensor [nd*nt*nb*2] in PEAK_DTYPE layout."""
        return self._records[i]

    def result(self, i):
        """Job i's (nd, nt, nb) PEAK_DTYPE result (copies; call after wait())."""
        j = self.jobs[i]
        raw = self._records[i].cpu().numpy()
        return raw.view(PEAK_DTYPE).reshape(j.nd, j.nt, j.nb)

    def results(self):
        self.run()
        self.wait()
        return [self.result(i) for i in range(len(self.jobs))]

    def info(self):
        """tickets, grid, segments, scratch batches, scratch bytes of the
        persistent launch, and how many jobs run on their own launches."""
        out = {"tickets": 0, "grid": 0, "segments": 0, "batches": 0, "scratch_bytes": 0,
               "own_launch_jobs": len(self._own)}
        if self._plan is None:
            return out
        t = ctypes.c_int64()
        g, s, q = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        b = ctypes.c_size_t()
        _lib.check(_lib.lib().mfb_batch_info(self._plan, ctypes.byref(t), ctypes.byref(g),
                                              ctypes.byref(s), ctypes.byref(q), ctypes.byref(b)))
        out.update({"tickets": t.value, "grid": g.value, "segments": s.value, "batches": q.value,
                    "scratch_bytes": b.value})
        return out

    def close(self):
        self._graph = None
        if getattr(self, "_plan", None):
            _lib.lib().mfb_batch_destroy(self._plan)
            self._plan = None
        for own in getattr(self, "_own", []):
            if own.get("plan") is not None:
                _lib.lib().mfb_destroy(own["plan"])
                own["plan"] = None
        self._own = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
