"""Loader for the reference's own CPU engine, built into oracle/_ref.

TEST INFRASTRUCTURE ONLY.  This module is imported by the tests, by
``__graft_entry__.smoke()`` and by ``bench.py``'s CPU-baseline leg, as the
checker and the reported baseline.  The product (``apogee_b200``) never
imports anything under ``oracle/``.

``oracle/Makefile.ref`` compiles the reference's unmodified sources
(``src/matchfilt.c``, ``src/hmf.c``, ``src/dispatch.c``, ``src/kernel.cc``
and the binding ``python/matchedfilter/_core.c``) against the project's
single-target Highway shim.  The resulting extension exposes the reference's
``_core.MF`` / ``_core.HMF`` types with their own argument conventions
(``_core.c:119-147,273-301``).  This module wraps them in the small amount of
Python that the reference's ``MatchedFilter.run`` adds on top
(``python/matchedfilter/__init__.py:435-514``): window clamping, bin count,
buffer allocation and conversion to ``(index int64, value complex64)``.
"""
import importlib.machinery
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def _has_avx512():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= flags
    except OSError:
        pass
    return False


_CORE = None


def path():
    """Path of the variant this host can run, or None if not built."""
    names = (["refcore_avx512.so"] if _has_avx512() else []) + ["refcore_avx2.so"]
    for name in names:
        p = os.path.join(REF_DIR, name)
        if os.path.exists(p):
            return p
    return None


def available():
    return path() is not None


def core():
    """The reference's compiled ``_core`` module (MF, HMF, backend())."""
    global _CORE
    if _CORE is None:
        p = path()
        if p is None:
            raise RuntimeError("reference CPU engine not built: run "
                               "make -f oracle/Makefile.ref")
        loader = importlib.machinery.ExtensionFileLoader("_core", p)
        spec = importlib.util.spec_from_file_location("_core", p, loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _CORE = mod
    return _CORE


def _window(n, window):
    if window is None:
        return 0, n
    s, e = max(0, min(int(window[0]), n)), max(0, min(int(window[1]), n))
    if s >= e:
        raise ValueError("empty window")
    return s, e


class RefFlat:
    """The reference flat filter (``_core.MF``) with run() returning arrays."""

    def __init__(self, n, ndata, ntemplates):
        self.n, self.nd, self.nt = int(n), int(ndata), int(ntemplates)
        self.mf = core().MF(self.n, self.nd, self.nt)

    def set_data(self, D):
        D = np.ascontiguousarray(D, np.complex64)
        self._held = D
        for i in range(D.shape[0]):
            self.mf.set_data(i, D[i])

    def set_templates(self, H):
        H = np.ascontiguousarray(H, np.complex64)
        for i in range(H.shape[0]):
            self.mf.set_template(i, H[i])

    def run(self, binsize=None, threshold=0.0, window=None, data=None, templates=None):
        """Returns (index int64 [nd,nt,nb], value complex64, counts int32 [nd,nt], total)."""
        n = self.n
        binsize = n if binsize is None else int(binsize)
        s, e = _window(n, window)
        d0, nd = (0, self.nd) if data is None else data
        t0, nt = (0, self.nt) if templates is None else templates
        nb = 1 + (e - s - 1) // binsize
        idx = np.empty(nd * nt * nb, np.int64)
        val = np.empty(nd * nt * nb, np.complex64)
        mag = np.empty(0, np.float32)
        cnt = np.empty(nd * nt, np.int32)
        tot = self.mf.run(d0, nd, t0, nt, binsize, float(threshold), s, e, idx, val, mag, cnt)
        return (idx.reshape(nd, nt, nb), val.reshape(nd, nt, nb),
                cnt.reshape(nd, nt), tot)

    def run_series(self, series, starts, wstart, wend, binsize, threshold=0.0, templates=None):
        """Blocks must already be grouped by window (the reference C contract)."""
        ser = np.ascontiguousarray(series, np.complex64)
        st = np.ascontiguousarray(starts, np.uintp)
        ws = np.ascontiguousarray(wstart, np.uintp)
        we = np.ascontiguousarray(wend, np.uintp)
        t0, nt = (0, self.nt) if templates is None else templates
        nblk = st.size
        lo, hi = min(int(ws[0]), self.n), min(int(we[0]), self.n)
        nb = 1 + (hi - lo - 1) // int(binsize)
        idx = np.empty(nblk * nt * nb, np.int64)
        val = np.empty(nblk * nt * nb, np.complex64)
        cnt = np.empty(nblk * nt, np.int32)
        self.mf.run_series(ser, st, ws, we, t0, nt, int(binsize), float(threshold),
                           idx, val, np.empty(0, np.float32), cnt)
        return idx.reshape(nblk, nt, nb), val.reshape(nblk, nt, nb)


class RefHier:
    """The reference hierarchical filter (``_core.HMF``) with a pinned band."""

    def __init__(self, n, ndata, ntemplates, band, coarse_threshold, reference=None,
                 snr=5.5, fd=1e-2):
        self.n, self.nd, self.nt = int(n), int(ndata), int(ntemplates)
        self.hmf = core().HMF(self.n, self.nd, self.nt, float(snr), float(fd),
                              int(band), 1, 8)
        if reference is not None:
            self._ref = np.ascontiguousarray(reference, np.float32)
            self.hmf.set_reference(self._ref)
        self.hmf.set_threshold(float(coarse_threshold))

    def set_data(self, D):
        # The reference plan keeps the caller's pointer (hmf.c:141): hold it.
        self._held = np.ascontiguousarray(D, np.complex64)
        for i in range(self._held.shape[0]):
            self.hmf.set_data(i, self._held[i])

    def set_templates(self, H):
        H = np.ascontiguousarray(H, np.complex64)
        for i in range(H.shape[0]):
            self.hmf.set_template(i, H[i])

    def run(self, binsize=None, threshold=0.0, window=None):
        n = self.n
        binsize = n if binsize is None else int(binsize)
        s, e = _window(n, window)
        nb = 1 + (e - s - 1) // binsize
        rows = self.nd * self.nt
        idx = np.empty(rows * nb, np.int64)
        val = np.empty(rows * nb, np.complex64)
        cnt = np.empty(rows, np.int32)
        self.hmf.run(0, self.nd, 0, self.nt, binsize, float(threshold), s, e,
                     idx, val, np.empty(0, np.float32), cnt)
        return idx.reshape(self.nd, self.nt, nb), val.reshape(self.nd, self.nt, nb)

    def stats(self):
        return self.hmf.stats()
