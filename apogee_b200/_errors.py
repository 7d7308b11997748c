"""Errors shared with the reference API (python/matchedfilter/_errors.py:13)."""


class UnsupportedSize(RuntimeError):
    """This device cannot run this transform length. Use a shorter one."""
