"""Differentiable peak values.

``peak_values(data, templates, binsize, threshold, window)`` runs the fused
filter and returns ``(index, value, power)`` with ``power = |value|^2``; it is
a ``torch.autograd.Function`` whose backward is the hand-written adjoint
kernel (``mfb_adjoint`` in include/mfb.h).  Gradients are taken at the fixed
argmax lags: a change of input that would move a bin's argmax is not
differentiated through (the peak lag is piecewise constant).  Backward
recomputes the lags by running the filter again on the saved spectra; no
correlation series is stored or written.

The reference has no gradients; the peak values themselves are the
reference's (``MatchedFilter.run``, python/matchedfilter/__init__.py:435-514).
"""
import torch

from . import _lib

_PLANS = {}


def _plan(n, nd, nt, device_index):
    from . import MatchedFilter
    key = (n, nd, nt, device_index)
    f = _PLANS.get(key)
    if f is None:
        f = _PLANS[key] = MatchedFilter(n, nd, nt, device="gpu:%d" % device_index)
    return f


def clear_plans():
    """Release the cached filter plans."""
    _PLANS.clear()


def _check(data, templates):
    for name, a in (("data", data), ("templates", templates)):
        if not isinstance(a, torch.Tensor) or not a.is_cuda:
            raise TypeError("%s must be a CUDA torch tensor" % name)
        if a.dtype != torch.complex64:
            raise TypeError("%s must be complex64, got %s" % (name, a.dtype))
        if a.dim() != 2:
            raise ValueError("%s must be two-dimensional (rows, n)" % name)
    if data.shape[1] != templates.shape[1]:
        raise ValueError("data and templates have different lengths")
    if data.device != templates.device:
        raise ValueError("data and templates are on different devices")


def _peaks(data, templates, binsize, threshold, window):
    n = data.shape[1]
    f = _plan(n, data.shape[0], templates.shape[0], data.device.index)
    f.set_data(data)
    f.set_templates(templates)
    return f.run_device(binsize=binsize, threshold=threshold, window=window)


class PeakValues(torch.autograd.Function):
    """Peaks of the fused filter with the adjoint kernel as backward."""

    @staticmethod
    def forward(ctx, data, templates, binsize, threshold, window):
        idx, val = _peaks(data, templates, binsize, threshold, window)
        ctx.save_for_backward(data, templates)
        ctx.args = (binsize, threshold, window)
        ctx.mark_non_differentiable(idx)
        power = val.real.square() + val.imag.square()
        return idx, val, power

    @staticmethod
    def backward(ctx, g_idx, g_val, g_pow):
        data, templates = ctx.saved_tensors
        need_d, need_t = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_d or need_t):
            return None, None, None, None, None
        idx, val = _peaks(data, templates, *ctx.args)
        gz = torch.zeros_like(val)
        if g_val is not None:
            gz = gz + g_val.to(torch.complex64)
        if g_pow is not None:
            gz = gz + 2.0 * g_pow.to(torch.float32) * val
        gz = gz.contiguous()
        gd = torch.empty_like(data) if need_d else None
        gt = torch.empty_like(templates) if need_t else None
        n, nd, nt, nb = data.shape[1], data.shape[0], templates.shape[0], val.shape[2]
        stream = torch.cuda.current_stream(data.device).cuda_stream
        rc = _lib.lib().mfb_adjoint(
            data.device.index, n, data.data_ptr(), nd, templates.data_ptr(), nt, nb,
            idx.data_ptr(), gz.data_ptr(), gd.data_ptr() if gd is not None else None,
            gt.data_ptr() if gt is not None else None, stream)
        _lib.check(rc, "adjoint failed")
        return gd, gt, None, None, None


def peak_values(data, templates, binsize, threshold=0.0, window=None):
    """``(index, value, power)`` of shape (nd, nt, nb), differentiable in
    ``value`` and ``power`` with respect to ``data`` and ``templates``
    (complex64 CUDA tensors [rows][n], spectra as ``MatchedFilter`` takes
    them).  Bins below threshold have index -1, value 0 and zero gradient."""
    _check(data, templates)
    data = data.contiguous()
    templates = templates.contiguous()
    return PeakValues.apply(data, templates, int(binsize), float(threshold),
                            None if window is None else (int(window[0]), int(window[1])))
