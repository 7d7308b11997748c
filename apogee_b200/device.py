"""Where a filter runs: CUDA devices only.

The spelling follows the reference (python/matchedfilter/device.py:145-199):
``"gpu"``, ``"gpu:N"``, ``"auto"`` and ``None`` (``MF_DEVICE`` or the
default), plus torch's ``"cuda"`` / ``"cuda:N"``.  This build has no CPU
engine: ``"cpu"`` is refused with a ValueError rather than silently served
by something else.
"""
import os


class Device:
    """One CUDA device.  Compares equal to ``"gpu:N"`` / ``"cuda:N"``."""

    __slots__ = ("kind", "index", "name", "backend", "is_software", "arch")

    def __init__(self, index, name="", arch=()):
        self.kind = "gpu"
        self.index = int(index)
        self.name = name
        self.backend = "cuda"
        self.is_software = False
        self.arch = tuple(arch)

    def __str__(self):
        return "gpu:%d" % self.index

    def __repr__(self):
        return "Device('%s', %r, backend='cuda')" % (self, self.name)

    def __eq__(self, other):
        if isinstance(other, str):
            try:
                other = parse(other)
            except (ValueError, RuntimeError, TypeError):
                return False
        return isinstance(other, Device) and self.index == other.index

    def __hash__(self):
        return hash(("gpu", self.index))


def devices():
    """Every CUDA device torch can see."""
    import torch
    out = []
    if torch.cuda.is_available():
        for i in range(torch.cuda.device_count()):
            p = torch.cuda.get_device_properties(i)
            out.append(Device(i, p.name, ("sm_%d%d" % (p.major, p.minor),)))
    return out


def parse(spec):
    """``None`` / string / Device -> Device; raises if no such CUDA device."""
    if isinstance(spec, Device):
        return spec
    if spec is None:
        spec = os.environ.get("MF_DEVICE") or "gpu"
    if not isinstance(spec, str):
        raise TypeError("device must be a string or Device, got %r" % (spec,))
    text = spec.strip().lower()
    if text == "auto":
        text = "gpu"
    kind, _, ordinal = text.partition(":")
    if kind == "cpu":
        raise ValueError("this build runs on CUDA devices only; device='cpu' has no engine "
                         "here (use the reference package for CPU filtering)")
    if kind not in ("gpu", "cuda"):
        raise ValueError("unknown device %r -- expected 'gpu', 'gpu:<n>', 'cuda:<n>' or 'auto'"
                         % spec)
    if ordinal and not ordinal.isdigit():
        raise ValueError("device ordinal must be an integer, got %r" % spec)
    found = devices()
    if not found:
        raise RuntimeError("no CUDA device available")
    want = int(ordinal) if ordinal else 0
    for d in found:
        if d.index == want:
            return d
    raise ValueError("no gpu with index %d; available: %s"
                     % (want, ", ".join(str(d) for d in found)))
