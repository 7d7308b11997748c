"""Block-layout validation and window grouping for run_series.

Same contract as the reference's SeriesLayout (python/matchedfilter/
_series.py:5-62): windows are clamped to [0, n]; every block needs a
nonempty window; every block's window must give the same bin count;
blocks with equal windows are grouped (stable, so the caller's order is
restored through ``order``).
"""
import numpy as np


class SeriesLayout:
    def __init__(self, n, starts, low, high, binsize):
        limit = np.iinfo(np.intp).max
        if np.any(low > limit) or np.any(high > limit):
            raise ValueError("window offsets must be nonnegative and fit in the index range")
        self.order = None
        self.starts = starts
        self.low = np.minimum(low, n)
        self.high = np.minimum(high, n)
        if np.any(self.low >= self.high):
            raise ValueError("every block must have a nonempty search window")
        widths = (self.high - self.low).astype(np.int64)
        bins = np.ones_like(widths) if binsize >= n else 1 + (widths - 1) // binsize
        self.nbins = int(bins[0])
        if np.any(bins != self.nbins):
            raise ValueError("every block's window must give the same bin count; "
                             "call run_series once per distinct bin count")
        self.groups = None

    def group(self):
        """Sort blocks by window (stable) so equal windows are adjacent."""
        lo, hi = self.low, self.high
        if lo.size > 1 and not (np.all(lo == lo[0]) and np.all(hi == hi[0])):
            change = (lo[1:] != lo[:-1]) | (hi[1:] != hi[:-1])
            runs = np.r_[0, np.flatnonzero(change) + 1]
            keys = list(zip(lo[runs].tolist(), hi[runs].tolist()))
            if len(set(keys)) != len(keys):          # a window recurs non-adjacently
                self.order = np.lexsort((hi, lo))
                self.starts = self.starts[self.order]
                self.low = lo[self.order]
                self.high = hi[self.order]
        lo, hi = self.low, self.high
        cuts = np.flatnonzero((lo[1:] != lo[:-1]) | (hi[1:] != hi[:-1])) + 1
        edges = np.r_[0, cuts, lo.size]
        self.groups = [(int(lo[a]), int(hi[a]), int(a), int(b))
                       for a, b in zip(edges[:-1], edges[1:])]
        return self
