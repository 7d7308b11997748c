"""Autotuner for the batched launch.

For one transform length n it times every candidate configuration of the
batched kernel on the device, in a one-job batch with a probe workload of
that n, and keeps the fastest:

* n <= 4096 (single-CTA fused filter): pairs per ticket -- 1, 2, 4 or 8
  items of 4096/n pairs (longer tickets take fewer queue atomics, shorter
  ones balance the tail better);
* n >= 8192 (four-step): the factorisation n = N1 * N2 with N2 in
  {64, 128, 256} and 64 <= N1 <= 4096, i.e. which radix-16 transform sizes
  the two passes run, and so the column tile width 4096/N2 of the first pass.

It also times the same probe job on its own launches (the kernels
specialised for n, as one plan per job runs them) and records both costs per
pair (``pp_us``, ``dedicated_pp_us``): ``batch.dedicated`` sends a job of
that n to its own launches when the difference times its pairs exceeds the
cost of a launch.

Results are cached per (device name, n) for the process, and in a JSON file
when ``MFB_TUNE_CACHE`` names one.
"""
import json
import os

_CACHE = {}


def candidates(n):
    """Configurations the batched kernel accepts for transform length n."""
    if n <= 4096:
        return [{"unit_items": k} for k in (1, 2, 4, 8)]
    out = []
    for n2 in (64, 128, 256):
        if 64 <= n // n2 <= 4096:
            out.append({"split": n2})
    return out


#: What tune(n) found on a B200 (CUDA events, probe workload of probe_shape):
#: the kernel configuration and the cost per pair (us) in the persistent launch
#: and on the job's own launches.  Used when a batch is not tuned.
B200 = {
    1024: ({"unit_items": 8}, 0.0046, 0.0037),
    2048: ({"unit_items": 8}, 0.0094, 0.0076),
    4096: ({"unit_items": 8}, 0.0198, 0.0148),
    8192: ({"split": 64}, 0.131, 0.038),
    16384: ({"split": 64}, 0.235, 0.086),
    32768: ({"split": 128}, 0.477, 0.335),
    65536: ({"split": 256}, 0.940, 0.661),
}


def default(n):
    """The configuration the library uses without tuning: the B200
    measurement where there is one, else the kernel's own defaults."""
    if n in B200:
        cfg, pp, dp = B200[n]
        out = dict(cfg)
        out["pp_us"], out["dedicated_pp_us"] = pp, dp
        return out
    if n <= 4096:
        return {"unit_items": 1}
    return {"split": 256 if n >= 16384 else 128}


def _load_file():
    path = os.environ.get("MFB_TUNE_CACHE")
    if not path or not os.path.exists(path):
        return {}
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_file(key, cfg):
    path = os.environ.get("MFB_TUNE_CACHE")
    if not path:
        return
    data = _load_file()
    data[key] = cfg
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def probe_shape(n, points=1 << 25):
    """(nd, nt) of the probe workload: about `points` correlation samples."""
    nd = 8
    nt = int(max(16, min(4096, points // (n * nd))))
    return nd, nt


def tune(n, device=None, reps=3, warmup=2):
    """Fastest configuration for n on `device` (a Device, spec or None)."""
    import torch
    from .batch import BatchedFilter, Job
    from .device import parse
    dev = parse(device)
    key = "%s|%d" % (dev.name or str(dev), n)
    if key in _CACHE:
        return dict(_CACHE[key])
    stored = _load_file().get(key)
    if stored is not None:
        _CACHE[key] = stored
        return dict(stored)
    nd, nt = probe_shape(n)
    tdev = torch.device("cuda", dev.index)
    g = torch.Generator(device=tdev).manual_seed(n)
    D = torch.randn(nd, n, dtype=torch.complex64, device=tdev, generator=g)
    H = torch.randn(nt, n, dtype=torch.complex64, device=tdev, generator=g)

    def time_cfg(cfg):
        bf = BatchedFilter([Job(H, data=D, binsize=max(1, n // 16))], device=dev,
                           tune={n: cfg})
        for _ in range(warmup):
            bf.run()
        bf.wait()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            bf.run()
        b.record()
        bf.wait()
        bf.close()
        return a.elapsed_time(b) / reps

    best, best_ms = None, float("inf")
    for cfg in candidates(n):
        ms = time_cfg(cfg)
        if ms < best_ms:
            best, best_ms = cfg, ms
    best = dict(best)
    pairs = nd * nt
    best["pp_us"] = best_ms * 1e3 / pairs
    best["dedicated_pp_us"] = time_cfg({"dedicated": True}) * 1e3 / pairs
    _CACHE[key] = best
    _store_file(key, best)
    return dict(best)


def tuned():
    """The configurations tuned so far in this process: {key: config}."""
    return dict(_CACHE)
