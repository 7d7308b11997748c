"""apogee_b200 -- the fused matched-filter hot path of the reference package
``matchedfilter`` (ahnitz/Apogee), rebuilt for NVIDIA B200 (CUDA sm_100a).

Drop-in API (python/matchedfilter/__init__.py:176-688, 1055-1460):

    >>> import apogee_b200 as mf
    >>> filt = mf.MatchedFilter(4096, ndata=16, ntemplates=1024, device="gpu")
    >>> filt.set_data(data_spectra)          # (16, 4096) complex64, already FFT'd
    >>> filt.set_templates(template_spectra)
    >>> peaks = filt.run(binsize=256, threshold=0.0)
    >>> peaks["index"], peaks["value"]       # (ndata, ntemplates, nbins)

Inputs are frequency-domain spectra (unnormalised forward transforms, natural
order).  For every pair the device kernel forms D*conj(H), runs the inverse
FFT and keeps the loudest lag of each bin of the window; the correlation
series never leaves the SM.  ``HierarchicalFilter`` screens pairs with a
low-band coarse pass and refines the survivors with the same kernel.

Arrays may be numpy arrays, anything that speaks DLPack, or torch tensors --
CUDA tensors are ingested device-to-device, with no host round trip.  There
is no CPU engine: if the CUDA library or device is missing, constructing a
filter raises.
"""
import math

import numpy as np

from ._errors import UnsupportedSize
from . import _lib
from .device import Device, devices, parse as _parse_device
from . import gatemodel

__version__ = "0.1.0"

#: dtype of the arrays returned by run(): where and what, as in the reference.
PEAK_DTYPE = np.dtype([("index", "<i8"), ("value", "<c8")])

#: Transform lengths the device kernels cover.
SIZES = frozenset(1 << k for k in range(6, 21))

__all__ = ["MatchedFilter", "HierarchicalFilter", "PEAK_DTYPE", "devices", "Device",
           "UnsupportedSize", "backend", "targets", "set_target", "__version__"]


def backend():
    """Name of the compute target ("CUDA sm_100a")."""
    return "CUDA sm_100a"


def targets():
    """Targets this build contains: the one CUDA architecture."""
    return ("CUDA sm_100a",)


def set_target(name):
    """Kept for API compatibility: only ``None`` or the one target is accepted."""
    if name is not None and name not in targets():
        raise ValueError("no such target in this build: %s" % name)


def _torch():
    import torch
    return torch


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _host_array(a):
    """numpy view of a host array (numpy, DLPack host producer, buffer)."""
    if isinstance(a, np.ndarray):
        return a
    if _is_torch(a):
        return a.detach().numpy()
    if hasattr(a, "__dlpack_device__"):
        try:
            return np.from_dlpack(a)
        except Exception:
            pass
    return np.asarray(a)


class _Spectra:
    """A bank of complex64 spectra ready for ingest: a torch CUDA tensor
    (device pointer) or a C-contiguous numpy array (host pointer)."""

    def __init__(self, a, shape, device_index):
        torch = None
        if _is_torch(a) and a.is_cuda:
            torch = _torch()
            t = a.detach()
            if t.dtype != torch.complex64:
                t = t.to(torch.complex64)
            if t.device.index != device_index:
                t = t.to(torch.device("cuda", device_index))
            t = t.contiguous()
            if tuple(t.shape) != shape:
                raise ValueError("expected shape %s, got %s" % (shape, tuple(t.shape)))
            self.keep, self.ptr = t, t.data_ptr()
        else:
            h = np.ascontiguousarray(_host_array(a), dtype=np.complex64)
            if h.shape != shape:
                raise ValueError("expected shape %s, got %s" % (shape, h.shape))
            self.keep, self.ptr = h, h.ctypes.data


def _repeat_key(binsize, threshold, window, data, templates):
    """The run() arguments as given, when they are immutable values that a
    later call can be compared with (None, numbers, tuples of ints); else
    None."""
    if binsize is not None and type(binsize) is not int:
        return None
    if type(threshold) not in (int, float) or threshold != threshold:
        return None
    for x in (window, data, templates):
        if x is not None and not (type(x) is tuple and all(type(v) is int for v in x)):
            return None
    return (binsize, threshold, window, data, templates)


def _check_window(n, window):
    if window is None:
        return 0, n
    start, end = int(window[0]), int(window[1])
    start = max(0, min(start, n))
    end = max(0, min(end, n))
    if start >= end:
        raise ValueError(f"empty window ({start}, {end})")
    return start, end


class MatchedFilter:
    """Correlate data segments against templates on a CUDA device.

    Every pair (d, t) gives ``IFFT(data_d * conj(template_t))``, unnormalised
    (a perfect match returns ``n * energy``), of which only the loudest sample
    per bin is reported.  Same constructor, setters, run() and run_series()
    contract as the reference's MatchedFilter
    (python/matchedfilter/__init__.py:176-688).
    """

    def __init__(self, n, ndata=1, ntemplates=1, device=None):
        self.n = int(n)
        self.ndata = int(ndata)
        self.ntemplates = int(ntemplates)
        if self.ndata < 1 or self.ntemplates < 1:
            raise ValueError("ndata and ntemplates must be >= 1")
        self.device = _parse_device(device)
        self._init_state()
        if self.n not in SIZES:
            raise ValueError(
                "device='gpu' supports n in %s; got %d" % (sorted(SIZES), self.n))
        self._plan = self._create_plan()

    # ---- plumbing -------------------------------------------------------------
    def _init_state(self):
        self._dataset = False
        self._data_ready = set()
        self._template_ready = set()
        self._bufs = {}
        self._views = {}
        self._plan = None

    def _create_plan(self):
        L = _lib.lib()
        import ctypes
        h = ctypes.c_void_p()
        _lib.check(L.mfb_create(ctypes.byref(h), self.n, self.ndata, self.ntemplates,
                                self.device.index), "mfb_create")
        return h

    def __del__(self):
        try:
            if getattr(self, "_plan", None) is not None:
                _lib.lib().mfb_destroy(self._plan)
                self._plan = None
        except Exception:
            pass

    def _stream(self):
        torch = _torch()
        return torch.cuda.current_stream(self.device.index)

    def _bind_stream(self):
        s = self._stream()
        _lib.check(_lib.lib().mfb_set_stream(self._plan, s.cuda_stream), "mfb_set_stream")
        return s

    def _buffer(self, key, shape, dtype, pinned=False):
        """Reused device (or pinned host) tensor for outputs."""
        v = self._views.get((key, shape, dtype))
        if v is not None:
            return v
        torch = _torch()
        b = self._bufs.get(key)
        numel = math.prod(shape)
        if b is None or b.numel() < numel or b.dtype != dtype:
            if pinned:
                b = torch.empty(max(numel, 1), dtype=dtype, pin_memory=True)
            else:
                b = torch.empty(max(numel, 1), dtype=dtype,
                                device=torch.device("cuda", self.device.index))
            self._bufs[key] = b
            self._views = {k: w for k, w in self._views.items() if k[0] != key}
        v = b[:numel].view(*shape)
        self._views[(key, shape, dtype)] = v
        return v

    # ---- ingest ---------------------------------------------------------------
    def _input_index(self, index, size):
        if index is None:
            return None
        index = int(index)
        if index < 0 or index >= size:
            raise IndexError("index %d out of range" % index)
        return index

    def _mark_ready(self, kind, index):
        attr = "_" + kind + "_ready"
        ready = getattr(self, attr)
        if index is None:
            setattr(self, attr, None)
        elif ready is not None:
            ready.add(index)
            if len(ready) == (self.ndata if kind == "data" else self.ntemplates):
                setattr(self, attr, None)

    def _missing(self, kind, start, count):
        ready = getattr(self, "_" + kind + "_ready")
        return ready is not None and any(i not in ready for i in range(start, start + count))

    def _require_templates(self, start, count):
        if self._missing("template", start, count):
            raise ValueError("no templates for requested rows: call set_templates() first")

    def _ingest(self, fn, spectra, index, rows):
        if index is None:
            s = _Spectra(spectra, (rows, self.n), self.device.index)
            r0, cnt = 0, rows
        else:
            a = spectra
            if _is_torch(a) and a.is_cuda:
                a = a.reshape(-1)
            else:
                a = np.ascontiguousarray(_host_array(a), dtype=np.complex64)
                if a.ndim != 1 or a.size != self.n:
                    raise ValueError("spectrum must be a 1-D complex array of %d samples, "
                                     "got shape %s" % (self.n, a.shape))
            s = _Spectra(a, (self.n,), self.device.index)
            r0, cnt = index, 1
        self._bind_stream()
        _lib.check(fn(self._plan, r0, cnt, s.ptr), "ingest")
        if not (_is_torch(spectra) and spectra.is_cuda):
            # host source: the copy is synchronous w.r.t. pageable memory, but make
            # the source's lifetime irrelevant either way
            self._stream().synchronize()
        else:
            self._ingest_keep = s.keep

    def set_data(self, spectra, index=None):
        """Set one data spectrum (with ``index``) or all from a (ndata, n) array."""
        index = self._input_index(index, self.ndata)
        self._ingest(_lib.lib().mfb_set_data, spectra, index, self.ndata)
        self._dataset = True
        self._mark_ready("data", index)

    def set_templates(self, spectra, index=None):
        """Set one template spectrum (with ``index``) or all from a (ntemplates, n) array."""
        index = self._input_index(index, self.ntemplates)
        self._ingest(_lib.lib().mfb_set_templates, spectra, index, self.ntemplates)
        self._mark_ready("template", index)

    # ---- run ------------------------------------------------------------------
    def nbins(self, binsize, window=None):
        binsize = int(binsize)
        if binsize < 1:
            raise ValueError("binsize must be >= 1")
        start, end = _check_window(self.n, window)
        return -(-(end - start) // binsize)

    def _run_args(self, binsize, window, data, templates):
        n = self.n
        binsize = n if binsize is None else int(binsize)
        if binsize < 1:
            raise ValueError("binsize must be >= 1")
        start, end = _check_window(n, window)
        d0, nd = (0, self.ndata) if data is None else (int(data[0]), int(data[1]))
        t0, nt = (0, self.ntemplates) if templates is None else (int(templates[0]),
                                                                 int(templates[1]))
        if nd < 1 or nt < 1 or d0 < 0 or t0 < 0 \
                or d0 + nd > self.ndata or t0 + nt > self.ntemplates:
            raise ValueError("data/templates sub-range out of bounds")
        if not self._dataset or self._missing("data", d0, nd):
            raise ValueError("no data: call set_data() before run()")
        self._require_templates(t0, nt)
        nb = 1 + (end - start - 1) // binsize
        return binsize, start, end, d0, nd, t0, nt, nb

    def _launch(self, records, raw_idx, raw_val, counts, d0, nd, t0, nt, binsize, thr, start, end):
        L = _lib.lib()
        cptr = counts.data_ptr() if counts is not None else None
        if records is not None:
            rc = L.mfb_run_records(self._plan, d0, nd, t0, nt, binsize, thr, start, end,
                                   records.data_ptr(), cptr)
        else:
            rc = L.mfb_run(self._plan, d0, nd, t0, nt, binsize, thr, start, end,
                           raw_idx.data_ptr(), raw_val.data_ptr(), cptr)
        _lib.check(rc, "matched filter failed")

    def run(self, binsize=None, threshold=0.0, window=None,
            data=None, templates=None, counts=False, raw=False):
        """Correlate and report the loudest sample per bin.

        Returns a structured array of shape ``(ndata, ntemplates, nbins)`` with
        fields ``index`` (int64) and ``value`` (complex64); bins that do not
        exceed ``threshold`` hold ``index == -1`` and ``value == 0``.
        ``counts=True`` also returns the per-pair crossing counts;
        ``raw=True`` returns ``(index, value)`` as two arrays.  Results live
        in buffers reused by the next call (copy what must outlive it).
        """
        binsize, start, end, d0, nd, t0, nt, nb = self._run_args(binsize, window, data, templates)
        threshold = float(threshold)
        if math.isnan(threshold):
            raise ValueError("threshold must not be NaN")
        return self._run_common(binsize, threshold, start, end, d0, nd, t0, nt, nb, counts, raw)

    def _run_common(self, binsize, threshold, start, end, d0, nd, t0, nt, nb, counts, raw):
        torch = _torch()
        stream = self._bind_stream()
        rows = nd * nt
        cnt_d = self._buffer("cnt", (rows,), torch.int32) if counts else None
        if raw:
            idx_d = self._buffer("idx", (rows * nb,), torch.int64)
            val_d = self._buffer("val", (rows * nb,), torch.complex64)
            self._launch(None, idx_d, val_d, cnt_d, d0, nd, t0, nt, binsize, threshold, start, end)
            idx_h = self._buffer("idx_h", (rows * nb,), torch.int64, pinned=True)
            val_h = self._buffer("val_h", (rows * nb,), torch.complex64, pinned=True)
            idx_h.copy_(idx_d, non_blocking=True)
            val_h.copy_(val_d, non_blocking=True)
        else:
            rec_d = self._buffer("rec", (rows * nb * 2,), torch.int64)
            self._launch(rec_d, None, None, cnt_d, d0, nd, t0, nt, binsize, threshold, start, end)
            rec_h = self._buffer("rec_h", (rows * nb * 2,), torch.int64, pinned=True)
            rec_h.copy_(rec_d, non_blocking=True)
        if counts:
            cnt_h = self._buffer("cnt_h", (rows,), torch.int32, pinned=True)
            cnt_h.copy_(cnt_d, non_blocking=True)
        self._after_launch()
        stream.synchronize()
        if raw:
            out = (idx_h.numpy().reshape(nd, nt, nb), val_h.numpy().reshape(nd, nt, nb))
        else:
            out = rec_h.numpy().view(PEAK_DTYPE).reshape(nd, nt, nb)
        if counts:
            return out, cnt_h.numpy().reshape(nd, nt)
        return out

    def _after_launch(self):
        pass

    def run_device(self, binsize=None, threshold=0.0, window=None, data=None, templates=None):
        """run() without leaving the device: returns torch CUDA tensors
        ``(index int64, value complex64)`` of shape (nd, nt, nb), enqueued on
        torch's current stream and not synchronised."""
        torch = _torch()
        binsize, start, end, d0, nd, t0, nt, nb = self._run_args(binsize, window, data, templates)
        self._bind_stream()
        dev = torch.device("cuda", self.device.index)
        idx = torch.empty(nd * nt * nb, dtype=torch.int64, device=dev)
        val = torch.empty(nd * nt * nb, dtype=torch.complex64, device=dev)
        self._launch(None, idx, val, None, d0, nd, t0, nt, binsize, float(threshold), start, end)
        return idx.view(nd, nt, nb), val.view(nd, nt, nb)

    def run_records(self, binsize=None, threshold=0.0, window=None, data=None, templates=None):
        """run() without leaving the device, as one table of PEAK_DTYPE
        records: a torch CUDA int64 tensor of shape (nd, nt, nb, 2) whose
        bytes are the structured result (index, then the complex64 value's
        bits), enqueued on torch's current stream and not synchronised.  A
        host copy viewed as PEAK_DTYPE is what run() returns."""
        torch = _torch()
        binsize, start, end, d0, nd, t0, nt, nb = self._run_args(binsize, window, data, templates)
        self._prepare_device()
        rec = torch.empty(nd * nt * nb * 2, dtype=torch.int64,
                          device=torch.device("cuda", self.device.index))
        self._launch(rec, None, None, None, d0, nd, t0, nt, binsize, float(threshold), start, end)
        return rec.view(nd, nt, nb, 2)

    def _prepare_device(self):
        self._bind_stream()

    # ---- series ---------------------------------------------------------------
    def _series_layout(self, series, starts, win_start, win_end, binsize, templates):
        from ._series import SeriesLayout
        st = np.ascontiguousarray(_host_array(starts)).astype(np.int64, copy=False)
        ws = np.ascontiguousarray(_host_array(win_start)).astype(np.int64, copy=False)
        we = np.ascontiguousarray(_host_array(win_end)).astype(np.int64, copy=False)
        if any(a.ndim != 1 for a in (st, ws, we)):
            raise ValueError("series, starts, win_start and win_end must be one-dimensional")
        if not (st.size == ws.size == we.size):
            raise ValueError("starts, win_start and win_end must be the same length")
        if st.size < 1:
            raise ValueError("run_series needs at least one block")
        if np.any(st < 0) or np.any(ws < 0) or np.any(we < 0) \
                or np.any(st > np.iinfo(np.intp).max - self.n):
            raise ValueError("starts must be nonnegative and fit in the sample index range")
        binsize = self.n if binsize is None else int(binsize)
        if binsize < 1:
            raise ValueError("binsize must be >= 1")
        t0, nt = (0, self.ntemplates) if templates is None else (int(templates[0]),
                                                                 int(templates[1]))
        if nt < 1 or t0 < 0 or t0 + nt > self.ntemplates:
            raise ValueError("templates sub-range out of bounds")
        self._require_templates(t0, nt)
        layout = SeriesLayout(self.n, st, ws, we, binsize).group()
        return layout, binsize, t0, nt

    def run_series(self, series, starts, win_start, win_end,
                   binsize=None, threshold=0.0, templates=None, raw=False):
        """Filter a time series over a caller-supplied block layout.

        Block b covers ``series[starts[b] : starts[b]+n]`` (zero-padded past
        the end); its spectrum is the forward FFT of the block divided by n,
        computed on the device.  Lags ``[win_start[b], win_end[b])`` of block
        b are searched.  Returns ``(nblocks, ntemplates, nbins)`` in caller
        order.  A later run() needs set_data() again, as in the reference.
        """
        torch = _torch()
        layout, binsize, t0, nt = self._series_layout(series, starts, win_start, win_end,
                                                      binsize, templates)
        threshold = float(threshold)
        if _is_torch(series) and series.is_cuda:
            ser = series.detach().reshape(-1).to(torch.complex64).contiguous()
            if ser.device.index != self.device.index:
                ser = ser.to(torch.device("cuda", self.device.index))
        else:
            ser_np = np.ascontiguousarray(_host_array(series), dtype=np.complex64)
            if ser_np.ndim != 1:
                raise ValueError("series, starts, win_start and win_end must be one-dimensional")
            ser = torch.from_numpy(ser_np).to(torch.device("cuda", self.device.index),
                                             non_blocking=False)
        self._dataset = False
        self._data_ready = set()
        nblk, nb = layout.starts.size, layout.nbins
        stream = self._bind_stream()
        idx_d = self._buffer("sidx", (nblk * nt * nb,), torch.int64)
        val_d = self._buffer("sval", (nblk * nt * nb,), torch.complex64)
        st = np.ascontiguousarray(layout.starts, dtype=np.uint64)
        lo = np.ascontiguousarray(layout.low, dtype=np.uint64)
        hi = np.ascontiguousarray(layout.high, dtype=np.uint64)
        rc = self._series_call(ser.data_ptr(), ser.numel(), st.ctypes.data, lo.ctypes.data,
                               hi.ctypes.data, nblk, t0, nt, binsize, threshold,
                               idx_d.data_ptr(), val_d.data_ptr())
        _lib.check(rc, "run_series failed")
        idx = idx_d.cpu().numpy().reshape(nblk, nt, nb)
        val = val_d.cpu().numpy().reshape(nblk, nt, nb)
        stream.synchronize()
        if layout.order is not None:
            ri = np.empty_like(idx)
            rv = np.empty_like(val)
            ri[layout.order], rv[layout.order] = idx, val
            idx, val = ri, rv
        if raw:
            return idx, val
        out = np.empty(idx.shape, PEAK_DTYPE)
        out["index"], out["value"] = idx, val
        return out

    def _series_call(self, *args):
        return _lib.lib().mfb_run_series(self._plan, *args, None)

    # ---- compatibility ----------------------------------------------------------
    def empty_shared(self, shape, dtype=np.complex64):
        """Pinned host array (page-locked, DMA-able), the CUDA analogue of the
        reference's host-visible shared buffers."""
        torch = _torch()
        dt = {np.dtype(np.complex64): torch.complex64, np.dtype(np.float32): torch.float32,
              np.dtype(np.uint32): torch.int32, np.dtype(np.int64): torch.int64}[np.dtype(dtype)]
        t = torch.empty(shape if isinstance(shape, tuple) else (shape,), dtype=dt,
                        pin_memory=True)
        return t.numpy().view(dtype)

    def clear_cache(self):
        """Release reused output buffers."""
        self._bufs = {}

    def set_memory_limits(self, *, cache_bytes=None, series_bytes=None):
        for value in (cache_bytes, series_bytes):
            if value is not None and int(value) < 1:
                raise ValueError("memory budgets must be positive")
        self.clear_cache()


#: Bands the split-precision tensor-core coarse pass covers: 512 directly,
#: 16384 as a four-step around the 512-point pass.
TC_BANDS = frozenset([512, 16384])
#: Bands at which coarse="auto" takes the tensor-core pass.
AUTO_TC_BANDS = frozenset([512])


def _coarse_kind(name, band=None):
    """Library coarse kind for `name` at `band` ("auto": the BF16 split
    tensor-core pass at AUTO_TC_BANDS, else the FP32 pass)."""
    kinds = {"bf16x3": _lib.COARSE_BF16X3, "fp16x3": _lib.COARSE_FP16X3, "fp32": _lib.COARSE_FP32}
    if name == "auto":
        if band is None:
            return None
        return _lib.COARSE_BF16X3 if band in AUTO_TC_BANDS else _lib.COARSE_FP32
    if name not in kinds:
        raise ValueError("coarse must be one of %s" % sorted(list(kinds) + ["auto"]))
    return kinds[name]


class HierarchicalFilter(MatchedFilter):
    """Coarse low-band screen on the device, full refinement of survivors.

    Same contract as the reference (python/matchedfilter/__init__.py:1055-1460):
    every reported peak is the flat filter's peak for that pair; pairs the
    coarse gate dismisses report (-1, 0).  ``band`` (power of two, 64 <= band
    < n) and the coarse threshold are either pinned by the caller
    (``band=...`` and ``set_coarse_threshold``) or derived: the threshold from
    the reference profile by the gate model for (snr, fd).

    ``coarse`` picks the coarse arithmetic: ``"bf16x3"`` / ``"fp16x3"``
    (split hi+lo tensor-core contraction, FP32 accumulation), ``"fp32"``
    (the flat FP32 kernel at length band, the reference's own method), or
    ``"auto"`` (default): the BF16 split tensor-core pass at AUTO_TC_BANDS,
    the FP32 pass at the others.  The tensor-core kinds cover TC_BANDS.
    """

    def __init__(self, n, ndata=1, ntemplates=1, snr=5.5, fd=1e-2,
                 band=None, taps=None, device=None, coarse="auto"):
        self.n = int(n)
        self.ndata = int(ndata)
        self.ntemplates = int(ntemplates)
        if self.ndata < 1 or self.ntemplates < 1:
            raise ValueError("ndata and ntemplates must be >= 1")
        if band is not None:
            band = int(band)
            if band < 64 or band >= self.n or band & (band - 1) or band > 16384:
                raise ValueError("band must be a power of two, >= 64, < n and <= 16384")
        if taps is not None:
            taps = int(taps)
            if taps < 2 or taps > 64 or taps % 2:
                raise ValueError("taps must be even and between 2 and 64")
        self.device = _parse_device(device)
        if self.n not in SIZES:
            raise ValueError("device='gpu' supports n in %s; got %d" % (sorted(SIZES), self.n))
        self.snr = float(snr)
        self.fd = float(fd)
        self._coarse = coarse
        self._kind = _coarse_kind(coarse, band)
        if self._kind not in (None, _lib.COARSE_FP32) and band is not None \
                and band not in TC_BANDS:
            raise ValueError("the %s coarse pass covers band in %s" % (coarse, sorted(TC_BANDS)))
        self._init_state()
        self._pinned = (band, int(taps or 8)) if band is not None else None
        self._pending_ref = None
        self._cal_thr = None
        self._fs_snr = None
        self._thr_applied = False
        self._hplan = None
        self._hband = None
        self._gate_cache = None
        self._pairs0 = 0
        self._trig0 = 0
        self._table = None     # pinned host table the device writes (run())
        self.last_d2h_bytes = 0
        self._hostdata = None  # host data bank, read by the device at run()
        self._upload_evt = None
        self._bound = None     # (plan, stream) last given to mfb_hier_set_stream
        self._tver = 0         # template bank version (band selection cache)
        self._band_sel = None  # (token, band) of the measured band selection
        self.selection = None  # the last band selection: band, gates, measured costs
        self._outview = None   # (key, read-only PEAK_DTYPE view of the host table)
        self._repeat = None    # the last host-table run's arguments, for a repeat of it
        torch = _torch()
        dev = torch.device("cuda", self.device.index)
        # Spectra are staged on the device until the band is known.
        self._gd = torch.zeros((self.ndata, self.n), dtype=torch.complex64, device=dev)
        self._gt = torch.zeros((self.ntemplates, self.n), dtype=torch.complex64, device=dev)
        self._tdirty = True
        self._ddirty = True
        if self._pinned is not None:
            self._build(self._pinned[0])

    def __del__(self):
        try:
            if getattr(self, "_hplan", None) is not None:
                _lib.lib().mfb_hier_destroy(self._hplan)
                self._hplan = None
        except Exception:
            pass

    # ---- plan ---------------------------------------------------------------
    def _build(self, band):
        import ctypes
        if self._hplan is not None and self._hband == band:
            return
        L = _lib.lib()
        if self._hplan is not None:
            p, t = self.stats
            self._pairs0, self._trig0 = p, t
            L.mfb_hier_destroy(self._hplan)
            self._hplan = None
        h = ctypes.c_void_p()
        self._kind = _coarse_kind(self._coarse, band)
        _lib.check(L.mfb_hier_create(ctypes.byref(h), self.n, self.ndata, self.ntemplates,
                                     band, self._kind, self.device.index), "mfb_hier_create")
        self._hplan = h
        self._hband = band
        self._bound = None
        self._tdirty = self._ddirty = True
        self._thr_applied = False

    def _bind_stream(self):
        s = self._stream()
        if self._hplan is not None:
            key = (self._hplan.value, s.cuda_stream)
            if key != self._bound:
                _lib.check(_lib.lib().mfb_hier_set_stream(self._hplan, s.cuda_stream))
                self._bound = key
        return s

    def _release_hostdata_event(self):
        if self._upload_evt is not None:
            self._upload_evt.synchronize()
            self._upload_evt = None

    def _release_hostdata(self):
        """Drop the held host bank once no upload from it is in flight."""
        self._release_hostdata_event()
        self._hostdata = None

    def _held_ok(self, a):
        """The held bank is still a C-contiguous complex64 (ndata, n) array."""
        return (type(a) is np.ndarray and a.dtype == np.complex64 and a.flags.c_contiguous
                and a.shape == (self.ndata, self.n))

    def set_data(self, spectra, index=None):
        """Set all data spectra (or one, with ``index``).

        A host bank is held, not copied: the device reads it when run()
        needs it, in stream order ahead of the kernels (the reference's CPU
        engine also keeps the caller's array and reads it during run,
        python/matchedfilter/__init__.py:335-351), so do not change the array
        before run() has returned.  From pinned memory the upload is one
        asynchronous copy with no host synchronisation.
        """
        if index is None and spectra is self._hostdata and self._held_ok(spectra):
            # the bank held already, refilled in place by the caller
            self._release_hostdata_event()
            self._ddirty = True
            return
        index = self._input_index(index, self.ndata)
        torch = _torch()
        if index is None:
            s = _Spectra(spectra, (self.ndata, self.n), self.device.index)
            self._release_hostdata()
            if _is_torch(s.keep):
                self._gd.copy_(s.keep)
            else:
                self._hostdata = s.keep
        else:
            if self._hostdata is not None:          # the device mirror takes the bank first
                self._gd.copy_(torch.from_numpy(self._hostdata))
                self._release_hostdata()
            a = spectra
            if not (_is_torch(a) and a.is_cuda):
                a = np.ascontiguousarray(_host_array(a), dtype=np.complex64)
                if a.ndim != 1 or a.size != self.n:
                    raise ValueError("spectrum must be a 1-D complex array of %d samples" % self.n)
                a = torch.from_numpy(a)
            self._gd[index].copy_(a.reshape(-1))
        self._ddirty = True
        self._dataset = True
        self._mark_ready("data", index)

    def set_templates(self, spectra, index=None):
        index = self._input_index(index, self.ntemplates)
        torch = _torch()
        if index is None:
            s = _Spectra(spectra, (self.ntemplates, self.n), self.device.index)
            src = s.keep if _is_torch(s.keep) else torch.from_numpy(s.keep)
            self._gt.copy_(src)
        else:
            a = spectra
            if not (_is_torch(a) and a.is_cuda):
                a = np.ascontiguousarray(_host_array(a), dtype=np.complex64)
                if a.ndim != 1 or a.size != self.n:
                    raise ValueError("spectrum must be a 1-D complex array of %d samples" % self.n)
                a = torch.from_numpy(a)
            self._gt[index].copy_(a.reshape(-1))
        self._tdirty = True
        self._tver += 1
        self._mark_ready("template", index)

    # ---- calibration -----------------------------------------------------------
    def _choose_band(self):
        """Pinned band, else the band that runs fastest on this device among
        those whose model gate resolves the budget (costmodel: the reference's
        choose_config, python/matchedfilter/__init__.py:1040-1054, with costs
        measured here on the caller's bank instead of read from a table)."""
        if self._pinned is not None:
            return self._pinned[0]
        if self._pending_ref is None:
            raise ValueError(
                "no band: pin band= (and a coarse threshold) or set_reference() so the "
                "gate model can place the threshold")
        token = (id(self._pending_ref), self._tver, self._fs_snr or self.snr, self.fd)
        # (the data bank the costs were measured on is not part of the token: a
        # choice made on one bank of the stream is kept for the next ones)
        if self._band_sel is not None and self._band_sel[0] == token:
            return self._band_sel[1]
        from . import costmodel
        tc = self._coarse in ("bf16x3", "fp16x3")
        gates = {}
        for band in costmodel.candidate_bands(self.n, (lambda b: b in TC_BANDS) if tc
                                              else (lambda b: True)):
            g = gatemodel.gate_for(self._pending_ref, self.n, band, self._fs_snr or self.snr,
                                   self.fd, device=self.device.index)
            if g is not None:
                gates[band] = g
        if not gates:
            raise ValueError("the gate model cannot resolve fd=%g at snr=%g for n=%d"
                             % (self.fd, self.snr, self.n))
        if self._template_ready is not None or not self._dataset or self._data_ready is not None:
            band, costs = max(gates), {}          # no bank or data yet to measure with: widest
        else:
            band, costs = costmodel.choose(self, gates)
            self._band_sel = (token, band)
        self.selection = {"band": band, "gates": gates,
                          "costs_us": {b: c[0] for b, c in costs.items()},
                          "refine_rates": {b: c[1] for b, c in costs.items()}}
        return band

    def _coarse_value(self, band):
        if self._cal_thr is not None:
            return float(self._cal_thr)
        if self._pending_ref is None:
            raise ValueError(
                "no calibrated coarse threshold for n=%d band=%d: provide a reference and a "
                "resolvable budget, or set both band and coarse threshold" % (self.n, band))
        key = (band, self._fs_snr or self.snr, self.fd, self._pending_ref.tobytes())
        if self._gate_cache is not None and self._gate_cache[0] == key:
            return self._gate_cache[1]
        # the model's FP64 covariance work and its draws run on this device
        v = gatemodel.gate_for(self._pending_ref, self.n, band, self._fs_snr or self.snr, self.fd,
                               device=self.device.index)
        if v is None:
            raise ValueError("no calibrated coarse threshold for n=%d band=%d" % (self.n, band))
        if not np.isfinite(v) or v < 0 or v > float(np.finfo(np.float32).max):
            raise ValueError("calibrated coarse threshold must be finite, nonnegative float32")
        self._gate_cache = (key, float(v))
        return float(v)

    def _prepare(self, defer_host=False):
        """Build the plan and push pending state; with defer_host a held host
        data bank is left for the run call to upload (returns its address)."""
        band = self._choose_band()
        self._build(band)
        L = _lib.lib()
        self._cur_stream = self._bind_stream()
        if self._tdirty:
            _lib.check(L.mfb_hier_set_templates(self._hplan, 0, self.ntemplates,
                                                self._gt.data_ptr()))
            ref = None if self._pending_ref is None else self._pending_ref
            _lib.check(L.mfb_hier_set_reference(
                self._hplan, None if ref is None else ref.ctypes.data))
            self._tdirty = False
        host = None
        if not self._thr_applied:
            _lib.check(L.mfb_hier_set_threshold(self._hplan, self._coarse_value(band)))
            self._thr_applied = True
        if self._ddirty:
            if self._hostdata is not None and defer_host:
                host = self._hostdata.ctypes.data
            elif self._hostdata is not None:
                _lib.check(L.mfb_hier_set_data(self._hplan, 0, self.ndata,
                                               self._hostdata.ctypes.data))
                if self._upload_evt is None:
                    self._upload_evt = _torch().cuda.Event()
                self._upload_evt.record(self._stream())
                self._ddirty = False
            else:
                _lib.check(L.mfb_hier_set_data(self._hplan, 0, self.ndata, self._gd.data_ptr()))
                self._ddirty = False
        return host

    def set_coarse_threshold(self, value):
        """Pin the coarse threshold (requires a pinned band); None -> model."""
        if value is None:
            self._cal_thr = None
            self._thr_applied = False
            return
        value = float(value)
        if not np.isfinite(value) or value < 0 or value > float(np.finfo(np.float32).max):
            raise ValueError("coarse threshold must be finite nonnegative float32, or None")
        if self._pinned is None:
            raise ValueError("an explicit coarse threshold requires an explicit band")
        self._cal_thr = value
        self._thr_applied = False

    def calibrate(self, snr=None, fd=None, segments=8192, templates=128, noise="real",
                  seed=20261203):
        """Measure the coarse threshold for (snr, fd) on the device and pin it.

        The reference's gate model (gatemodel.gate_for) assumes complex filter
        output with Re and Im each of unit variance; data whose output noise is
        distributed differently (real-valued output from Hermitian spectra, for
        instance) gets a gate that is right for the model, not for the data.
        This measures the same quantity the model computes -- the fd-quantile
        of the coarse maximum over pairs whose full filter reaches `snr` --
        from signals injected at `snr` into independent noise, with this
        filter's own coarse pass and the flat filter as the fine stage.

        noise: "real" (spectrum of real N(0,1) noise / sqrt(n), Hermitian) or
        "complex" (per-bin complex normal, unit output variance).  A sample of
        `templates` templates of the bank is used, `segments` noise segments,
        one injection each at a uniformly random lag.  Needs a pinned band.
        Returns the threshold, which is also applied.
        """
        if self._pinned is None:
            raise ValueError("calibrate() needs an explicit band")
        if self._template_ready is not None:
            raise ValueError("calibrate() needs the template bank: call set_templates() first")
        snr = self.snr if snr is None else float(snr)
        fd = self.fd if fd is None else float(fd)
        if not (np.isfinite(snr) and snr > 0 and np.isfinite(fd) and 0 < fd < 1):
            raise ValueError("snr must be positive and fd in (0, 1)")
        from . import synthetic
        band, n = self._pinned[0], self.n
        rng = np.random.default_rng(seed)
        k = min(int(templates), self.ntemplates)
        tsel = np.sort(rng.choice(self.ntemplates, size=k, replace=False))
        Hs = self._gt[tsel].cpu().numpy()
        kind = self._coarse
        chunk = 512
        kept = []
        flat = MatchedFilter(n, chunk, k, device=self.device)
        coarse = HierarchicalFilter(n, chunk, k, band=band, device=self.device, coarse=kind)
        coarse.set_coarse_threshold(0.0)
        flat.set_templates(Hs)
        coarse.set_templates(Hs)
        if self._pending_ref is not None:
            coarse.set_reference(self._pending_ref)
        ph = np.arange(n)
        for c0 in range(0, int(segments), chunk):
            if noise == "real":
                D = synthetic.noise_spectra(n, chunk, rng)
            elif noise == "complex":
                D = (rng.standard_normal((chunk, n)) + 1j * rng.standard_normal((chunk, n))) \
                    / np.sqrt(2)
            else:
                raise ValueError("noise must be 'real' or 'complex'")
            inj = rng.integers(0, k, size=chunk)
            lag = rng.integers(0, n, size=chunk)
            D += snr * Hs[inj].astype(np.complex128) * np.exp(-2j * np.pi * np.outer(lag, ph) / n)
            D = D.astype(np.complex64)
            flat.set_data(D)
            coarse.set_data(D)
            det = flat.run(binsize=n, threshold=snr)["index"][:, :, 0] >= 0
            cv = coarse.coarse_values()
            kept.append(cv[det])
        kept = np.sort(np.concatenate(kept))
        i = int(np.floor(fd * kept.size))
        if i < 8:
            raise ValueError("too few detections (%d) to place fd=%g; raise segments"
                             % (kept.size, fd))
        gate = float(kept[i])
        self.set_coarse_threshold(gate)
        self.calibration = {"gate": gate, "detections": int(kept.size), "snr": snr, "fd": fd,
                            "noise": noise, "segments": int(segments), "templates": k}
        return gate

    def set_first_stage(self, snr):
        """Calibrate the coarse gate at ``snr`` instead of the constructor's."""
        self._fs_snr = float(snr) if snr is not None and float(snr) > 0 else None
        self._thr_applied = False

    def set_reference(self, power):
        """Expected output power per frequency bin (length n, any scale)."""
        if power is not None:
            p = np.ascontiguousarray(_host_array(power), dtype=np.float32)
            if p.shape != (self.n,):
                raise ValueError("reference must be a one-dimensional array of length %d" % self.n)
            if not np.isfinite(p).all() or np.any(p < 0) or not np.any(p > 0):
                raise ValueError("reference must be finite, nonnegative, with positive total power")
            self._pending_ref = p
        else:
            self._pending_ref = None
        self._tdirty = True
        self._thr_applied = False

    # ---- run ----------------------------------------------------------------
    def _launch(self, records, raw_idx, raw_val, counts, d0, nd, t0, nt, binsize, thr, start, end):
        L = _lib.lib()
        cptr = counts.data_ptr() if counts is not None else None
        if records is not None:
            rc = L.mfb_hier_run_records(self._hplan, d0, nd, t0, nt, binsize, thr, start, end,
                                        records.data_ptr(), cptr)
        else:
            rc = L.mfb_hier_run(self._hplan, d0, nd, t0, nt, binsize, thr, start, end,
                                raw_idx.data_ptr(), raw_val.data_ptr(), cptr)
        _lib.check(rc, "hierarchical filter failed")

    def run(self, binsize=None, threshold=0.0, window=None,
            data=None, templates=None, counts=False, raw=False):
        """Hierarchical run; the table as ``MatchedFilter.run``.

        The default structured table is kept in pinned host memory between
        calls and only the refined rows cross the host link (every row the
        gate dismisses is all empty records), written by the device straight
        into the host table.  As in the reference ("Results may reuse
        buffers ... The next run on this filter overwrites it in place;
        .copy() anything that must outlive that call",
        python/matchedfilter/__init__.py:463-466), the next call updates it in
        place; it is returned read-only because the device tracks which of its
        rows hold refined results.
        """
        if not counts and not raw:
            rep = self._repeat
            if rep is not None and rep[0] == (binsize, threshold, window, data, templates) \
                    and self._repeat_ok(rep):
                return self._run_repeat(rep)
        binsize_a, threshold_a, window_a, data_a, templates_a = (binsize, threshold, window,
                                                                 data, templates)
        binsize, start, end, d0, nd, t0, nt, nb = self._run_args(binsize, window, data, templates)
        threshold = float(threshold)
        if math.isnan(threshold):
            raise ValueError("threshold must not be NaN")
        if not counts and not raw:
            host = self._prepare(defer_host=True)
            out = self._run_host(binsize, threshold, start, end, d0, nd, t0, nt, nb, host)
            key = _repeat_key(binsize_a, threshold_a, window_a, data_a, templates_a)
            self._repeat = None if key is None else (key, self._hplan.value, self._last_args)
            return out
        self._prepare()
        return self._run_common(binsize, threshold, start, end, d0, nd, t0, nt, nb, counts, raw)

    def _repeat_ok(self, rep):
        """The plan state a repeat of the last host-table run relies on is
        unchanged: same plan, templates and reference pushed, threshold
        applied, and the data rows current or held as a host bank."""
        return (self._hplan is not None and self._hplan.value == rep[1] and not self._tdirty
                and self._thr_applied and (not self._ddirty or self._hostdata is not None))

    def _run_repeat(self, rep):
        """run() with the arguments of the previous host-table run, which
        _run_args validated then (argument checks and plan set-up skipped)."""
        stream = self._bind_stream()
        host = self._hostdata.ctypes.data if self._ddirty else None
        fn, args, tail, _ = rep[2]
        _lib.check(fn(self._hplan, *args, host, *tail), "hierarchical filter failed")
        stream.synchronize()
        if host is not None:
            self._ddirty = False
        out, info = self._outview[1], self._outview[2]
        self.last_d2h_bytes = int(info[1])
        return out

    def _run_host(self, binsize, threshold, start, end, d0, nd, t0, nt, nb, host=None):
        torch = _torch()
        stream = self._cur_stream                 # bound by _prepare
        need = nd * nt * nb * 2                   # int64 words of the table
        rec_d = self._buffer("rec", (need,), torch.int64)
        tab = self._table
        if tab is None or tab.numel() < need:
            tab = self._table = torch.empty(need, dtype=torch.int64, pin_memory=True)
        info = self._buffer("info", (2,), torch.int64, pinned=True)
        fn = _lib.lib().mfb_hier_run_host
        args = (d0, nd, t0, nt, binsize, threshold, start, end)
        tail = (rec_d.data_ptr(), tab.data_ptr(), info.data_ptr())
        self._last_args = (fn, args, tail, (rec_d, tab, info))   # the tensors stay alive
        _lib.check(fn(self._hplan, *args, host, *tail), "hierarchical filter failed")
        stream.synchronize()
        if host is not None:
            self._ddirty = False
        key = (tab.data_ptr(), info.data_ptr(), nd, nt, nb)
        if self._outview is None or self._outview[0] != key:
            out = tab.numpy()[:need].view(PEAK_DTYPE).reshape(nd, nt, nb)
            out.flags.writeable = False
            self._outview = (key, out, info.numpy())
        self.last_d2h_bytes = int(self._outview[2][1])
        return self._outview[1]

    def _prepare_device(self):
        self._prepare()

    def run_device(self, binsize=None, threshold=0.0, window=None, data=None, templates=None):
        torch = _torch()
        binsize, start, end, d0, nd, t0, nt, nb = self._run_args(binsize, window, data, templates)
        self._prepare()
        dev = torch.device("cuda", self.device.index)
        idx = torch.empty(nd * nt * nb, dtype=torch.int64, device=dev)
        val = torch.empty(nd * nt * nb, dtype=torch.complex64, device=dev)
        self._launch(None, idx, val, None, d0, nd, t0, nt, binsize, float(threshold), start, end)
        return idx.view(nd, nt, nb), val.view(nd, nt, nb)

    def coarse_values(self, window=None, data=None, templates=None):
        """Maximum |coarse z| per pair (tensor-core coarse kinds), (nd, nt) float32."""
        torch = _torch()
        _, start, end, d0, nd, t0, nt, _ = self._run_args(None, window, data, templates)
        self._prepare()
        out = torch.empty(nd * nt, dtype=torch.float32,
                          device=torch.device("cuda", self.device.index))
        _lib.check(_lib.lib().mfb_hier_coarse_values(self._hplan, d0, nd, t0, nt, start, end,
                                                     out.data_ptr()))
        return out.cpu().numpy().reshape(nd, nt)

    def run_series(self, series, starts, win_start, win_end,
                   binsize=None, threshold=0.0, templates=None, raw=False):
        """Hierarchical filter over a caller-supplied block layout
        (ap_hmf_run_series, src/hmf.c:158-220): runs of blocks with equal
        windows, at most ndata at a time, are transformed on the device into
        the plan's data rows and run through coarse pass, gate and refine.
        The data set with set_data() is restored before the next run()."""
        self._prepare()
        kept = (self._dataset,
                None if self._data_ready is None else set(self._data_ready))
        try:
            return MatchedFilter.run_series(self, series, starts, win_start, win_end,
                                            binsize=binsize, threshold=threshold,
                                            templates=templates, raw=raw)
        finally:
            self._dataset, self._data_ready = kept
            self._ddirty = True

    def _series_call(self, *args):
        return _lib.lib().mfb_hier_run_series(self._hplan, *args, None)

    @property
    def config(self):
        """``(band, taps)`` pinned or selected."""
        if self._pinned is not None:
            return self._pinned
        return (self._choose_band(), 8)

    @property
    def stats(self):
        """``(pairs, triggers)`` accumulated since construction."""
        import ctypes
        if self._hplan is None:
            return (self._pairs0, self._trig0)
        p, t = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.lib().mfb_hier_stats(self._hplan, ctypes.byref(p), ctypes.byref(t)))
        return (self._pairs0 + p.value, self._trig0 + t.value)

    @property
    def refine_rate(self):
        """Fraction of pairs that needed the full correlation (lifetime)."""
        pairs, trig = self.stats
        return trig / pairs if pairs else 0.0

    @property
    def last_refinements(self):
        """Survivors of the most recent run()."""
        import ctypes
        t = ctypes.c_int64()
        _lib.check(_lib.lib().mfb_hier_last_triggers(self._hplan, ctypes.byref(t)))
        return t.value
