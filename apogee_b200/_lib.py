"""ctypes binding of libmfb.so, the C ABI declared in include/mfb.h.

The library is built in-tree (``apogee_b200/build.py``).  There is no CPU
fallback: if the shared library or a CUDA device is missing, creating a
filter raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmfb.so")

MFB_OK = 0
MFB_ERR_ARG = -1
MFB_ERR_INDEX = -2
MFB_ERR_CUDA = -3
MFB_ERR_UNSUPPORTED = -4
MFB_ERR_STATE = -5

COARSE_FP32 = 0
COARSE_BF16X3 = 1
COARSE_FP16X3 = 2

#: Every symbol include/mfb.h declares, with (restype, argtypes).
_P = ctypes.c_void_p
_I = ctypes.c_int
_SZ = ctypes.c_size_t
_F = ctypes.c_float
_PP = ctypes.POINTER(ctypes.c_void_p)
_I64P = ctypes.POINTER(ctypes.c_int64)
_SZP = ctypes.POINTER(ctypes.c_size_t)
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)


class MfbJob(ctypes.Structure):
    """struct mfb_job of include/mfb.h (field order and types as declared)."""
    _fields_ = [
        ("n", ctypes.c_size_t),
        ("nd", ctypes.c_int),
        ("nt", ctypes.c_int),
        ("data", ctypes.c_void_p),
        ("templates", ctypes.c_void_p),
        ("series", ctypes.c_void_p),
        ("nseries", ctypes.c_size_t),
        ("starts", ctypes.c_void_p),
        ("binsize", ctypes.c_size_t),
        ("threshold", ctypes.c_float),
        ("start", ctypes.c_size_t),
        ("end", ctypes.c_size_t),
        ("records", ctypes.c_void_p),
        ("split", ctypes.c_int),
        ("unit_items", ctypes.c_int),
    ]


class MfbBatchOpts(ctypes.Structure):
    """struct mfb_batch_opts of include/mfb.h."""
    _fields_ = [("slot_bytes", ctypes.c_size_t), ("slots", ctypes.c_int)]


SIGNATURES = {
    "mfb_batch_create": (_I, [_PP, _I, ctypes.POINTER(MfbJob), _I, ctypes.POINTER(MfbBatchOpts)]),
    "mfb_batch_run": (_I, [_P, _P]),
    "mfb_batch_status": (_I, [_P, _P]),
    "mfb_batch_test_wait_limit": (_I, [_P, _I]),
    "mfb_batch_info": (_I, [_P, _I64P, _IP, _IP, _IP, _SZP]),
    "mfb_batch_destroy": (_I, [_P]),
    "mfb_create": (_I, [_PP, _SZ, _I, _I, _I]),
    "mfb_destroy": (_I, [_P]),
    "mfb_set_stream": (_I, [_P, _P]),
    "mfb_set_packed": (_I, [_P, _I]),
    "mfb_set_cluster": (_I, [_P, _I]),
    "mfb_set_data": (_I, [_P, _I, _I, _P]),
    "mfb_set_templates": (_I, [_P, _I, _I, _P]),
    "mfb_run": (_I, [_P, _I, _I, _I, _I, _SZ, _F, _SZ, _SZ, _P, _P, _P]),
    "mfb_run_records": (_I, [_P, _I, _I, _I, _I, _SZ, _F, _SZ, _SZ, _P, _P]),
    "mfb_run_rows": (_I, [_P, _I, _I, _I, _I, _P, _P, _I, _SZ, _F, _SZ, _SZ, _P, _P, _P]),
    "mfb_run_series": (_I, [_P, _P, _SZ, _P, _P, _P, _I, _I, _I, _SZ, _F, _P, _P, _P]),
    "mfb_forward": (_I, [_P, _P, _SZ, _P, _I, _P]),
    "mfb_nbins": (_SZ, [_SZ, _SZ, _SZ, _SZ]),
    "mfb_last_error": (ctypes.c_char_p, []),
    "mfb_supported": (_I, [_SZ]),
    "mfb_hier_create": (_I, [_PP, _SZ, _I, _I, _SZ, _I, _I]),
    "mfb_hier_destroy": (_I, [_P]),
    "mfb_hier_set_stream": (_I, [_P, _P]),
    "mfb_hier_set_packed": (_I, [_P, _I]),
    "mfb_hier_set_cluster": (_I, [_P, _I]),
    "mfb_hier_set_data": (_I, [_P, _I, _I, _P]),
    "mfb_hier_set_templates": (_I, [_P, _I, _I, _P]),
    "mfb_hier_set_reference": (_I, [_P, _P]),
    "mfb_hier_set_threshold": (_I, [_P, _F]),
    "mfb_hier_run": (_I, [_P, _I, _I, _I, _I, _SZ, _F, _SZ, _SZ, _P, _P, _P]),
    "mfb_hier_run_records": (_I, [_P, _I, _I, _I, _I, _SZ, _F, _SZ, _SZ, _P, _P]),
    "mfb_hier_run_host": (_I, [_P, _I, _I, _I, _I, _SZ, _F, _SZ, _SZ, _P, _P, _P, _P]),
    "mfb_hier_run_phase": (_I, [_P, _I, _I, _I, _I, _I, _SZ, _F, _SZ, _SZ, _P, _P, _P]),
    "mfb_hier_last_triggers": (_I, [_P, _I64P]),
    "mfb_hier_stats": (_I, [_P, _I64P, _I64P]),
    "mfb_hier_config": (_I, [_P, _SZP, _IP]),
    "mfb_hier_coarse_values": (_I, [_P, _I, _I, _I, _I, _SZ, _SZ, _P]),
    "mfb_fp32_peak": (_I, [_I, _DP]),
    "mfb_hier_run_series": (_I, [_P, _P, _SZ, _P, _P, _P, _I, _I, _I, _SZ, _F, _P, _P, _P]),
    "mfb_gate_maxima": (_I, [_I, _P, _SZ, _SZ, _F, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _DP]),
    "mfb_adjoint": (_I, [_I, _SZ, _P, _I, _P, _I, _SZ, _P, _P, _P, _P, _P]),
    "mfb_run_large_static": (_I, [_I, _SZ, _P, _I, _P, _I, _SZ, _F, _SZ, _SZ, _P, _P, _P, _P]),
}

_LIB = None


class LibraryMissing(RuntimeError):
    """libmfb.so is not built (run apogee_b200.build.build())."""


def lib():
    """The loaded library; raises LibraryMissing rather than falling back."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                "apogee_b200/libmfb.so is not built; run python -c "
                "'import apogee_b200.build as b; b.build()'")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc, what="matchedfilter"):
    """Map an MFB status to the reference binding's exception types
    (python/matchedfilter/_core.c:90-145)."""
    if rc >= 0:
        return rc
    msg = lib().mfb_last_error().decode(errors="replace") or what
    if rc in (MFB_ERR_ARG, MFB_ERR_UNSUPPORTED):
        raise ValueError(msg)
    if rc == MFB_ERR_INDEX:
        raise IndexError(msg)
    raise RuntimeError("%s: %s" % (what, msg))
