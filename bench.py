#!/usr/bin/env python
"""Benchmark: filter pairs/sec at n=4096 -- mixed-precision hierarchical
filter vs FP32 flat filter, at the same false-dismissal rate.

Workload (one GPU): n=4096, 16 data segments x 1024 templates = 16384 pairs,
binsize 256 (16 bins), hierarchical band 512 (1/8), snr 5.5, fd 1e-2,
threshold 5.5, reference profile = mean |h|^2 of the bank; synthetic seeded
inputs (apogee_b200/synthetic.py), 10% of segments injected at SNR U[5,12].
Both arms use the same coarse threshold (CAL_GATE below); the gate model's
own threshold is reported beside it.  With --gpus N each rank filters its own
16 x 1024 block (its own template slice), so per-GPU work is fixed (weak
scaling) and nothing is exchanged.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload hier|batched|large] [--no-sub]

Prints ONE JSON line (rank 0).  `value` is device throughput with inputs
resident in HBM, timed with CUDA events per step (L2 flushed between steps),
max over ranks; `e2e` is the same metric through the public API
(HierarchicalFilter.set_data from pinned host memory holding fresh data every
step + run() returning the numpy structured result).  At one GPU the line also
carries `configs`: the flat generator's workload, the adjoint, the n=262144
bank and the batched jobs, each with its time and a parity summary.
`--impl reference` times the reference's own CPU engine (built from its
sources into oracle/_ref) on the same workload and gate, on every host thread,
with the one-thread figure beside it.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N, ND, NT, BINSIZE, BAND = 4096, 16, 1024, 256, 512
SNR, FD, THRESHOLD = 5.5, 1e-2, 5.5
FLOPS_PER_PAIR = lambda n: 5 * n * int(np.log2(n)) + 9 * n   # the reference's own convention
# Tensor-core flops the coarse pass executes per pair at band 512: per 8 pairs,
# stage 1 = 12 MMAs of M128 x N32 x K16 and stage 2 = 12 MMAs of M128 x N64 x K16
# (hi*hi + hi*lo + lo*hi included), 2 flops per multiply-add.
TC_FLOPS_PER_PAIR = (12 * 128 * 32 * 16 * 2 + 12 * 128 * 64 * 16 * 2) / 8
# DRAM bytes per launch from one ncu capture of the same kernels on this workload
# (profiles/coarse_tc_ws_band512_16x1024.md, profiles/flat_kernel_n4096_16x1024.md).
TRAFFIC_COARSE_TC = 4.347e6
TRAFFIC_FLAT = 34.18e6


def measured_peaks():
    """(bf16 TFLOP/s, HBM GB/s, source) from MEASURED_PEAKS.json, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["bf16_tflops"]), float(m["hbm_gbs"]), "MEASURED_PEAKS.json (burst)"
    except (OSError, ValueError, KeyError):
        return 1590.0, 6650.0, "fallback (no MEASURED_PEAKS.json)"


# Coarse threshold of the benchmark workload, shared by both arms: the
# fd = 1e-2 quantile of the band-512 coarse maximum over pairs whose full
# filter reaches snr 5.5, measured with FP64 correlations on 8192 independent
# noise segments with injections (tests/golden/make_gate.py, which writes
# tests/golden/gate_config1.json).  The gate model's own value for this
# profile is reported beside it (model_gate).
CAL_GATE = 3.7228326885529683
GATE_DESC = ("fd=1e-2 quantile of the coarse maximum of detectable signals, FP64, "
             "8192 independent noise segments (tests/golden/make_gate.py)")
METRIC = "filter pairs/sec at n=4096: mixed-precision hier vs FP32 flat, same FD rate"
WORKLOAD = ("hierarchical n=4096 ndata=16 ntemplates=1024 binsize=256 band=512 snr=5.5 "
            "fd=1e-2 threshold=5.5, 10% of segments injected at SNR U[5,12]")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--coarse", default=os.environ.get("MFB_COARSE", "bf16x3"),
                    choices=["fp32", "bf16x3", "fp16x3"])
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--workload", default="hier", choices=["hier", "batched", "large"],
                    help="hier: the headline n=4096 workload (default); batched: 256 uneven "
                         "jobs in one persistent launch; large: n=262144 bank, flat and "
                         "hierarchical")
    ap.add_argument("--jobs", type=int, default=256, help="batched workload: number of jobs")
    ap.add_argument("--large-coarse", default="fp16x3", choices=["fp32", "bf16x3", "fp16x3"],
                    help="large workload: coarse arithmetic of the hierarchical filter")
    ap.add_argument("--no-tune", action="store_true", help="batched workload: default configs")
    ap.add_argument("--no-sub", action="store_true",
                    help="headline only: skip the per-configuration sub-records")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of this GPU's clocks and throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ reference arm
def host_threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except (AttributeError, OSError):
        return max(1, os.cpu_count() or 1)


class RefHierThreads:
    """The reference hierarchical engine on `threads` host threads: one plan
    per thread over a contiguous slice of the template bank (the reference
    parallelises by separate plans; its binding releases the GIL while a
    plan runs, python/matchedfilter/_core.c)."""

    def __init__(self, refcore, H, power, gate, threads):
        from concurrent.futures import ThreadPoolExecutor
        from apogee_b200.shard import template_slice
        self.threads = max(1, min(int(threads), NT))
        self.plans = []
        for i in range(self.threads):
            t0, cnt = template_slice(NT, i, self.threads)
            r = refcore.RefHier(N, ND, cnt, BAND, gate, reference=power, snr=SNR, fd=FD)
            r.set_templates(H[t0:t0 + cnt])
            self.plans.append(r)
        self.pool = ThreadPoolExecutor(self.threads)

    def step(self, D):
        def one(r):
            r.set_data(D)
            return r.run(binsize=BINSIZE, threshold=THRESHOLD)
        return [f.result() for f in [self.pool.submit(one, r) for r in self.plans]]

    def close(self):
        self.pool.shutdown()


def workload_config():
    """The `config` both arms print: workload, gate and pairs (identical)."""
    return {"workload": WORKLOAD, "gate": GATE_DESC, "gate_value": CAL_GATE,
            "pairs_per_gpu": ND * NT}


def ref_single_thread(refcore, H, power, D, gate, seconds=2.0):
    """The reference hierarchical engine as it runs by default: one plan on
    one thread, warm run() calls over the whole 16 x 1024 workload."""
    r = refcore.RefHier(N, ND, NT, BAND, gate, reference=power, snr=SNR, fd=FD)
    r.set_templates(H)
    r.set_data(D)
    r.run(binsize=BINSIZE, threshold=THRESHOLD)
    reps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds or reps < 3:
        r.run(binsize=BINSIZE, threshold=THRESHOLD)
        reps += 1
    return reps * ND * NT / (time.perf_counter() - t0), reps


def reference_arm(args):
    """The reference's own CPU engine (oracle/_ref) on all host threads, at
    the same gate as our arm; the one-thread figure beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    try:
        from oracle import refcore
        if not refcore.available():
            raise RuntimeError("oracle/_ref not built")
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU engine: %s" % e}))
        return
    from apogee_b200 import synthetic, gatemodel
    D, H, power, _ = synthetic.hier_workload(N, ND, NT, seed=args.seed)
    eng = RefHierThreads(refcore, H, power, CAL_GATE, host_threads())
    for _ in range(args.warmup):
        eng.step(D)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.step(D)
    dt = (time.perf_counter() - t0) / args.steps
    eng.close()
    v = ND * NT / dt
    st_value, st_reps = ref_single_thread(refcore, H, power, D, CAL_GATE)
    gate_model = gatemodel.gate_for(power, N, BAND, SNR, FD)
    engm = RefHierThreads(refcore, H, power, gate_model, host_threads())
    engm.step(D)
    t0 = time.perf_counter()
    for _ in range(max(3, args.steps // 4)):
        engm.step(D)
    model_v = max(3, args.steps // 4) * ND * NT / (time.perf_counter() - t0)
    engm.close()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(),
        "engine": "reference CPU engine built from its sources, %d threads (one plan per "
                  "thread over a template slice), HierarchicalFilter band=512" % eng.threads,
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": eng.threads,
                         "kind": "reference",
                         "sample": "the full 16x1024 workload per step, %d steps" % args.steps,
                         "cpu": cpu_model(), "simd": refcore.core().backend(),
                         "single_thread": {"value": st_value, "unit": "pairs/s", "cores": 1,
                                           "sample": "one plan, %d warm runs of the full "
                                                     "workload" % st_reps}},
        "model_gate": {"gate_value": gate_model, "value": model_v, "unit": "pairs/s",
                       "cores": eng.threads},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# --------------------------------------------------------------- our arm
def cpu_baseline_leg(D, H, power, gate, hier_idx):
    """Rank 0, N=1: the reference CPU engine on a bounded sample at the
    headline's gate (all host threads, and one thread), and the false
    dismissal of each device hierarchical result against FP64."""
    out = {}
    try:
        from oracle import refcore, oracle
    except Exception as e:
        return {"unavailable": str(e)}, None
    if refcore.available():
        eng = RefHierThreads(refcore, H, power, gate, host_threads())
        eng.step(D)
        reps, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 3.0 or reps < 3:
            eng.step(D)
            reps += 1
        hier_v = reps * ND * NT / (time.perf_counter() - t0)
        eng.close()
        st_value, st_reps = ref_single_thread(refcore, H, power, D, gate)
        f = refcore.RefFlat(N, ND, NT)
        f.set_templates(H)
        f.set_data(D)
        t0 = time.perf_counter()
        f.run(binsize=BINSIZE, threshold=THRESHOLD)
        flat_v = ND * NT / (time.perf_counter() - t0)
        out = {"value": hier_v, "unit": "pairs/s", "cores": eng.threads, "kind": "reference",
               "sample": "full 16x1024 hierarchical workload at the headline gate, %d runs "
                         "(~3 s), one plan per thread over a template slice" % reps,
               "single_thread": {"value": st_value, "unit": "pairs/s", "cores": 1,
                                 "sample": "one plan, %d warm runs of the full workload"
                                           % st_reps},
               "flat_value": flat_v, "flat_sample": "flat filter, 1 run on 1 thread",
               "cpu": cpu_model(), "simd": refcore.core().backend()}
    # false dismissal vs the FP64 flat filter, for each hierarchical result
    det = 0
    omit = {k: 0 for k in hier_idx}
    for t0 in range(0, NT, 128):
        z = oracle.correlate(D, H[t0:t0 + 128])
        m = np.abs(z).reshape(ND, -1, N // BINSIZE, BINSIZE).max(-1)
        hit = m > THRESHOLD
        det += int(hit.sum())
        for k, hidx in hier_idx.items():
            omit[k] += int((hit & (hidx[:, t0:t0 + 128, :] < 0)).sum())
    fd = {"fp64_detections": det}
    for k in hier_idx:
        fd[k] = {"omitted": omit[k], "rate": omit[k] / det if det else 0.0}
    return out, fd


def graph_of(dev, step, bind):
    """One CUDA graph of `step` (after `bind`), warmed outside the capture."""
    import torch
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        bind()
        step()
    torch.cuda.current_stream(dev).wait_stream(s)
    torch.cuda.synchronize(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        bind()
        step()
    return g


def timed_replays(dev, g, steps, warm, flush, world=1, sampler=None):
    """Device milliseconds of `steps` replays of g (CUDA events per replay, L2
    flushed before each, outside the events), max over ranks."""
    import torch
    import torch.distributed as dist
    for _ in range(warm):
        flush.zero_()
        g.replay()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    if sampler:
        # sustained load so that the clock samples see the GPU busy
        sampler.start()
        t_end = time.perf_counter() + 1.5
        while time.perf_counter() < t_end:
            for _ in range(50):
                g.replay()
            torch.cuda.synchronize(dev)
    evs = []
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        g.replay()
        b.record()
        evs.append((a, b))
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = sampler.stop() if sampler else None
    ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item()), clk


def fp32_peak(local):
    import ctypes
    from apogee_b200 import _lib
    peak = ctypes.c_double()
    _lib.check(_lib.lib().mfb_fp32_peak(local, ctypes.byref(peak)))
    return peak.value


def our_arm(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import apogee_b200 as mf
    from apogee_b200 import synthetic, _lib
    dev = torch.device("cuda", local)
    seed = args.seed + 1000 * rank
    D, H, power, inj = synthetic.hier_workload(N, ND, NT, seed=seed)
    gdev = "gpu:%d" % local

    def make_hier(gate):
        hf = mf.HierarchicalFilter(N, ND, NT, snr=SNR, fd=FD, band=BAND, device=gdev,
                                   coarse=args.coarse)
        hf.set_reference(power)
        hf.set_templates(H)
        if gate is not None:
            hf.set_coarse_threshold(gate)
        hf.set_data(D)
        return hf

    hf_cal = make_hier(CAL_GATE)
    hf_mod = make_hier(None)
    first_cal = hf_cal.run(binsize=BINSIZE, threshold=THRESHOLD).copy()
    first_mod = hf_mod.run(binsize=BINSIZE, threshold=THRESHOLD).copy()
    gate_model = hf_mod._coarse_value(BAND)
    flat = mf.MatchedFilter(N, ND, NT, device=gdev)
    flat.set_data(D)
    flat.set_templates(H)
    L = _lib.lib()
    nb = N // BINSIZE
    rows = ND * NT
    idx = torch.empty(rows * nb, dtype=torch.int64, device=dev)
    val = torch.empty(rows * nb, dtype=torch.complex64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    def hier_step(hf):
        _lib.check(L.mfb_hier_run(hf._hplan, 0, ND, 0, NT, BINSIZE, THRESHOLD, 0, N,
                                  idx.data_ptr(), val.data_ptr(), None))

    def flat_step():
        _lib.check(L.mfb_run(flat._plan, 0, ND, 0, NT, BINSIZE, THRESHOLD, 0, N,
                             idx.data_ptr(), val.data_ptr(), None))

    g_cal = graph_of(dev, lambda: hier_step(hf_cal), hf_cal._bind_stream)
    g_mod = graph_of(dev, lambda: hier_step(hf_mod), hf_mod._bind_stream)
    g_flat = graph_of(dev, flat_step, flat._bind_stream)

    sampler = ClockSampler(local)
    ms_cal, clocks = timed_replays(dev, g_cal, args.steps, args.warmup, flush, world, sampler)
    ms_mod, _ = timed_replays(dev, g_mod, args.steps, args.warmup, flush, world)
    flat_steps = max(3, args.steps // 2)
    ms_flat, _ = timed_replays(dev, g_flat, flat_steps, args.warmup, flush, world)
    hier_ms_step = ms_cal / args.steps
    model_ms_step = ms_mod / args.steps
    flat_ms_step = ms_flat / flat_steps
    value = world * rows / (hier_ms_step * 1e-3)
    model_value = world * rows / (model_ms_step * 1e-3)
    flat_value = world * rows / (flat_ms_step * 1e-3)

    # per-kernel durations of the hierarchical step (coarse+gate, refine)
    def phase_ms(hf, phase, reps=10):
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            hf._bind_stream()
            if phase == 2:
                _lib.check(L.mfb_hier_run_phase(hf._hplan, 1, 0, ND, 0, NT, BINSIZE, THRESHOLD,
                                                0, N, idx.data_ptr(), val.data_ptr(), None))
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            _lib.check(L.mfb_hier_run_phase(hf._hplan, phase, 0, ND, 0, NT, BINSIZE, THRESHOLD,
                                            0, N, idx.data_ptr(), val.data_ptr(), None))
            b.record()
            torch.cuda.synchronize(dev)
            tot += a.elapsed_time(b)
        return tot / reps
    coarse_ms = phase_ms(hf_cal, 1)
    refine_ms = phase_ms(hf_cal, 2)
    trig = hf_cal.last_refinements
    phase_ms(hf_mod, 1, 1)
    trig_mod = hf_mod.last_refinements

    # End to end through the public API (host buffers both ways), fresh data
    # every step: banks of the same templates with new noise and injections,
    # copied into the step's pinned input outside the timed region; the
    # result comes back as the rows of the table that changed.
    banks = [synthetic.hier_data(H, ND, np.random.default_rng(seed * 7919 + 17 + i))[0]
             for i in range(8)]
    D_pin = torch.empty(D.shape, dtype=torch.complex64, pin_memory=True)
    D_host = D_pin.numpy()

    def e2e_step(i):
        D_host[:] = banks[i % len(banks)]
        t0 = time.perf_counter()
        hf_cal.set_data(D_host)
        hf_cal.run(binsize=BINSIZE, threshold=THRESHOLD)
        return time.perf_counter() - t0, hf_cal.last_d2h_bytes
    for i in range(args.warmup):
        e2e_step(i)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    e2e_s, d2h_total = 0.0, 0
    for i in range(args.steps):
        dt, nbytes = e2e_step(i)
        e2e_s += dt
        d2h_total += nbytes
    last = hf_cal.run(binsize=BINSIZE, threshold=THRESHOLD).copy()
    ridx, rval = hf_cal.run(raw=True, binsize=BINSIZE, threshold=THRESHOLD)
    if not ((last["index"] == ridx).all() and (last["value"] == rval).all()):
        raise RuntimeError("end-to-end table differs from the device table of the same data")
    t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * rows * args.steps / float(t.item())

    peak = fp32_peak(local)
    flat_flops = rows * FLOPS_PER_PAIR(N)
    flat_achieved = flat_flops / (flat_ms_step * 1e-3) / 1e12
    # coarse kernel: the reference's algorithmic flops of a band-point filter per pair
    coarse_flops = rows * FLOPS_PER_PAIR(BAND)
    refine_flops = trig * FLOPS_PER_PAIR(N)
    dominant = "coarse" if coarse_ms >= refine_ms else "refine"
    dom_flops, dom_ms = (coarse_flops, coarse_ms) if dominant == "coarse" else (refine_flops,
                                                                                refine_ms)
    bf16_peak, hbm_peak, peak_src = measured_peaks()
    if dominant == "coarse" and args.coarse != "fp32":
        tc_flops = rows * TC_FLOPS_PER_PAIR
        roofline_line = {
            "bound": "tensor", "kernel": "coarse_tc_ws_kernel",
            "achieved": tc_flops / (coarse_ms * 1e-3) / 1e12, "peak": bf16_peak,
            "unit": "TFLOP/s", "frac": tc_flops / (coarse_ms * 1e-3) / (bf16_peak * 1e12),
            "traffic": TRAFFIC_COARSE_TC,
            "flops_per_pair": TC_FLOPS_PER_PAIR,
            "hbm_frac": TRAFFIC_COARSE_TC / (coarse_ms * 1e-3) / (hbm_peak * 1e9),
            "fp32_equivalent": {"achieved": coarse_flops / (coarse_ms * 1e-3) / 1e12,
                                "frac": coarse_flops / (coarse_ms * 1e-3) / peak,
                                "flops_per_pair": FLOPS_PER_PAIR(BAND)},
            "peak_source": "bf16 dense GEMM " + peak_src + " (of measured); traffic from an "
                           "ncu capture"}
    else:
        roofline_line = {
            "bound": "fp32", "kernel": dominant,
            "achieved": dom_flops / (dom_ms * 1e-3) / 1e12, "peak": peak / 1e12,
            "unit": "TFLOP/s", "frac": dom_flops / (dom_ms * 1e-3) / peak,
            "traffic": TRAFFIC_FLAT if dominant == "refine" else None,
            "peak_source": "measured FP32 FMA loop on this GPU (mfb_fp32_peak)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": hier_ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "bf16x3": "bf16x3+f32", "fp16x3": "f16x3+f32"}[args.coarse],
            "data": "synthetic",
            "config": workload_config(),
            "method": {"coarse": args.coarse,
                       "l2": "flushed (256 MiB write) between timed steps",
                       "timing": "CUDA events per step around a CUDA-graph replay"},
            "flat": {"value": flat_value, "unit": "pairs/s", "ms_per_step": flat_ms_step},
            "speedup_hier_vs_flat": value / flat_value,
            "refine_rate": trig / rows,
            "model_gate": {"gate_value": gate_model, "value": model_value,
                           "ms_per_step": model_ms_step, "refine_rate": trig_mod / rows,
                           "speedup_vs_flat": model_value / flat_value},
            "kernels_ms": {"coarse_gate": coarse_ms, "refine": refine_ms,
                           "how": "each phase alone (mfb_hier_run_phase), CUDA events around "
                                  "its launches, L2 flushed; the graph step overlaps their "
                                  "launch latencies"},
            "roofline": roofline_line,
            "roofline_flat": {"bound": "fp32", "achieved": flat_achieved,
                              "peak": peak / 1e12, "unit": "TFLOP/s",
                              "frac": flat_achieved * 1e12 / peak,
                              "flops_per_pair": FLOPS_PER_PAIR(N),
                              "traffic": TRAFFIC_FLAT,
                              "hbm_frac": TRAFFIC_FLAT / (flat_ms_step * 1e-3) / (hbm_peak * 1e9),
                              "peak_source": "measured FP32 FMA loop on this GPU (mfb_fp32_peak, "
                                             "of measured); %.1f TFLOP/s theoretical at the "
                                             "median SM clock" % (
                                                 148 * 128 * 2 * (clocks.get("sm_mhz") or 1965)
                                                 * 1e6 / 1e12)},
            "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": ND * N * 8,
                    "d2h_bytes_per_step": d2h_total // args.steps,
                    "result": "full (%d, %d, %d) peak table on the host; the refined rows "
                              "cross the link, every other row is empty" % (ND, NT, nb),
                    "data": "fresh every step: %d banks of the same templates with new noise "
                            "and injections, copied into the pinned input outside the timed "
                            "region" % len(banks)},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
        }
        if world == 1:
            cb, fd = cpu_baseline_leg(D, H, power, CAL_GATE,
                                      {"calibrated": first_cal["index"],
                                       "model": first_mod["index"]})
            line["cpu_baseline"] = cb
            line["false_dismissal"] = fd
    del g_cal, g_mod, g_flat, hf_cal, hf_mod, flat
    if world == 1 and not args.no_sub:
        torch.cuda.empty_cache()
        line["configs"] = sub_records(args, dev, local, flush, peak)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------- per-configuration records
def sub_records(args, dev, local, flush, peak):
    """The other benchmark configurations at one GPU, each with its time,
    roofline and a parity or false-dismissal summary (a failure is reported
    in its record and does not stop the others)."""
    import torch
    out = {}
    for name, fn in (("config0_flat", sub_config0), ("config3_adjoint", sub_config3),
                     ("config4_large", sub_config4), ("config2_batched", sub_config2)):
        t0 = time.perf_counter()
        try:
            out[name] = fn(args, dev, local, flush, peak)
        except Exception as e:     # reported in the record
            out[name] = {"error": "%s: %s" % (type(e).__name__, e)}
        out[name]["wall_s"] = time.perf_counter() - t0
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
    return out


def sub_config0(args, dev, local, flush, peak):
    """Flat FP32 filter on its own generator: n=4096, 16 x 1024, binsize 256,
    threshold 0, 2 of 16 segments injected at SNR 8."""
    import apogee_b200 as mf
    from apogee_b200 import synthetic, _lib
    import torch
    D, H, inj = synthetic.flat_workload(N, ND, NT, seed=0)
    f = mf.MatchedFilter(N, ND, NT, device="gpu:%d" % local)
    f.set_data(D)
    f.set_templates(H)
    L = _lib.lib()
    rows, nb = ND * NT, N // BINSIZE
    rec = torch.empty(rows * nb * 2, dtype=torch.int64, device=dev)

    def step():
        _lib.check(L.mfb_run_records(f._plan, 0, ND, 0, NT, BINSIZE, 0.0, 0, N,
                                     rec.data_ptr(), None))
    g = graph_of(dev, step, f._bind_stream)
    steps = max(5, args.steps // 2)
    ms, _ = timed_replays(dev, g, steps, max(3, args.warmup), flush)
    ms /= steps
    out = f.run(binsize=BINSIZE, threshold=0.0).copy()
    from oracle import oracle, parity
    bad = parity.compare(out["index"][:, :128], out["value"][:, :128],
                         oracle.correlate(D, H[:128]), BINSIZE, 0.0)
    found = sum(int(abs(int(out["index"][d, t, lag // BINSIZE]) - lag) <= 8)
                for d, t, lag, _ in inj)
    flops = rows * FLOPS_PER_PAIR(N)
    return {"workload": "flat n=4096 ndata=16 ntemplates=1024 binsize=256 threshold=0, 2 of 16 "
                        "segments injected at SNR 8",
            "value": rows / (ms * 1e-3), "unit": "pairs/s", "ms_per_step": ms,
            "roofline": {"bound": "fp32", "achieved": flops / (ms * 1e-3) / 1e12,
                         "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": flops / (ms * 1e-3) / peak, "traffic": TRAFFIC_FLAT,
                         "peak_source": "measured FP32 FMA loop (mfb_fp32_peak), of measured"},
            "parity": {"pairs_checked_fp64": ND * 128, "mismatches": len(bad),
                       "injections_found": "%d/%d within 8 lags" % (found, len(inj))},
            "timing": "CUDA events per CUDA-graph replay, L2 flushed, %d steps" % steps}


def sub_config3(args, dev, local, flush, peak):
    """Differentiable peak values: n=16384, 8 x 256, binsize 1024; forward +
    backward of sum |peak|^2 through the adjoint kernel, and the gradient's
    error against an FP64 torch.fft dense-correlation gradient."""
    import torch
    from apogee_b200 import synthetic
    from apogee_b200.adjoint import peak_values
    n, nd, nt, bs = 16384, 8, 256, 1024
    rng = np.random.default_rng(3)
    Hn = synthetic.template_bank(n, nt, rng)
    Dn = synthetic.noise_spectra(n, nd, rng)
    for d in range(0, nd, 3):
        synthetic.inject(Dn, Hn, d, int(rng.integers(nt)), int(rng.integers(n)), 8.0)
    D = torch.from_numpy(Dn.astype(np.complex64)).to(dev).requires_grad_(True)
    H = torch.from_numpy(Hn).to(dev).requires_grad_(True)

    def fwd_bwd():
        D.grad = None
        H.grad = None
        _, _, power = peak_values(D, H, bs)
        power.sum().backward()
    for _ in range(3):
        fwd_bwd()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(max(5, args.steps // 4)):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fwd_bwd()
        b.record()
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    idx, _, _ = peak_values(D, H, bs)
    D64 = D.detach().to(torch.complex128).requires_grad_(True)
    H64 = H.detach().to(torch.complex128).requires_grad_(True)
    z = torch.fft.ifft(D64[:, None, :] * torch.conj(H64[None]), dim=-1) * n
    zb = torch.gather(z, 2, idx.clamp(min=0))
    ((zb.real ** 2 + zb.imag ** 2) * (idx >= 0)).sum().backward()
    err = {}
    for name, ours, ref in (("grad_data", D.grad, D64.grad), ("grad_templates", H.grad, H64.grad)):
        ref = ref.resolve_conj()
        diff = ours.to(torch.complex128) - ref
        err[name] = {"rel_l2": (diff.norm() / ref.norm()).item(),
                     "max_rel": (diff.abs().max() / ref.abs().max()).item()}
    del z, zb
    return {"workload": "adjoint n=16384 ndata=8 ntemplates=256 binsize=1024: forward + "
                        "backward of sum |peak value|^2",
            "ms_per_step": float(np.median(ms)), "unit": "ms",
            "value": nd * nt / (float(np.median(ms)) * 1e-3), "value_unit": "pairs/s",
            "gradient_vs_fp64_torch_fft": err,
            "timing": "CUDA events around forward + backward, median of %d" % len(ms)}


def sub_config4(args, dev, local, flush, peak):
    rec = large_record(dev, local, args.seed, steps=3, warmup=2, coarse="fp16x3",
                       cpu_sample=False, compare="fp32")
    rec.pop("clocks", None)
    return rec


def sub_config2(args, dev, local, flush, peak):
    rec = batched_record(dev, local, args.seed, 256, steps=2, warmup=1, tune=False,
                         peak=peak)
    rec.pop("clocks", None)
    return rec


# ------------------------------------------------------- batched workload
BATCH_METRIC = "filter pairs/sec, uneven jobs in one persistent launch"
BATCH_WORKLOAD = ("%d jobs: n = 2^U{10..16}, nd ~ U{1..64}, nt ~ U{16..4096} (nt*n*8 <= 2 GB), "
                  "binsize n/16 or n/64, every 4th job a float32 series cut into nd blocks, "
                  "templates by the config-0 formula generated on the device")


def per_job_plans(jobs, dev_index):
    """Device time of the same jobs run one plan per job (mfb_run / mfb_run_series),
    the way the reference runs one plan per shape.  Plan creation and template
    upload are outside the timed region; each job is warmed once."""
    import ctypes
    import torch
    from apogee_b200 import _lib
    from apogee_b200.batch import _device_complex
    L = _lib.lib()
    dev = torch.device("cuda", dev_index)
    stream = torch.cuda.current_stream(dev).cuda_stream
    total_ms = 0.0
    for j in jobs:
        plan = ctypes.c_void_p()
        _lib.check(L.mfb_create(ctypes.byref(plan), j.n, j.nd, j.nt, dev_index))
        try:
            _lib.check(L.mfb_set_stream(plan, stream))
            H = _device_complex(j.templates, dev)
            _lib.check(L.mfb_set_templates(plan, 0, j.nt, H.data_ptr()))
            idx = torch.empty(j.pairs * j.nb, dtype=torch.int64, device=dev)
            val = torch.empty(j.pairs * j.nb, dtype=torch.complex64, device=dev)
            if j.data is not None:
                D = _device_complex(j.data, dev)
                _lib.check(L.mfb_set_data(plan, 0, j.nd, D.data_ptr()))

                def run():
                    _lib.check(L.mfb_run(plan, 0, j.nd, 0, j.nt, j.binsize, j.threshold, j.start,
                                         j.end, idx.data_ptr(), val.data_ptr(), None))
            else:
                ser = _device_complex(j.series, dev).reshape(-1)
                st = np.ascontiguousarray(j.starts, dtype=np.uint64)
                ws = np.full(j.nd, j.start, np.uint64)
                we = np.full(j.nd, j.end, np.uint64)

                def run():
                    _lib.check(L.mfb_run_series(plan, ser.data_ptr(), ser.numel(), st.ctypes.data,
                                                ws.ctypes.data, we.ctypes.data, j.nd, 0, j.nt,
                                                j.binsize, j.threshold, idx.data_ptr(),
                                                val.data_ptr(), None))
            run()
            torch.cuda.synchronize(dev)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            run()
            b.record()
            torch.cuda.synchronize(dev)
            total_ms += a.elapsed_time(b)
        finally:
            L.mfb_destroy(plan)
    return total_ms


def batched_record(dev, local, seed, njobs, steps, warmup, tune, peak, world=1, rank=0):
    """Time the config-2 generator's first `njobs` jobs in the batched engine
    (one CUDA graph: the persistent launch plus the jobs' own launches)
    against the same jobs one plan per job."""
    import torch
    import torch.distributed as dist
    from apogee_b200 import synthetic, autotune
    from apogee_b200.batch import BatchedFilter
    t0 = time.perf_counter()
    jobs = synthetic.batched_workload(njobs=njobs, seed=seed + 1000 * rank, device=str(dev))
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    pairs = sum(j.pairs for j in jobs)
    flops = float(sum(j.pairs * FLOPS_PER_PAIR(j.n) for j in jobs))
    tmpl_bytes = sum(j.nt * j.n * 8 for j in jobs)
    t0 = time.perf_counter()
    bf = BatchedFilter(jobs, device="gpu:%d" % local, tune=tune)
    plan_s = time.perf_counter() - t0
    bf.capture()
    for _ in range(max(warmup, 1)):
        bf.replay()
    torch.cuda.synchronize(dev)
    bf.wait()
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for a, b in ev:
        a.record()
        bf.replay()
        b.record()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    bf.wait()
    ms_step = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    if world > 1:
        tmax = torch.tensor([ms_step], device=dev)
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        ms_step = float(tmax.item())
    info = bf.info()
    bf.close()
    base_ms = per_job_plans(jobs, local)
    return {
        "workload": BATCH_WORKLOAD % njobs, "value": pairs * world / (ms_step * 1e-3),
        "unit": "pairs/s", "ms_per_step": ms_step, "pairs_per_gpu": pairs,
        "templates_gb": tmpl_bytes / 1e9, "tuned": autotune.tuned() if tune else False,
        "plan": info, "generate_s": gen_s, "plan_s": plan_s,
        "l2": "inputs (%.0f GB) far larger than L2" % (tmpl_bytes / 1e9),
        "timing": "CUDA events around each CUDA-graph replay",
        "per_job_plans": {"value": pairs / (base_ms * 1e-3), "unit": "pairs/s", "ms": base_ms,
                          "how": "one mfb plan per job (mfb_run / mfb_run_series), "
                                 "device time summed over jobs"},
        "speedup_vs_per_job_plans": base_ms / ms_step,
        "roofline": {"bound": "fp32", "achieved": flops / (ms_step * 1e-3) / 1e12,
                     "peak": peak / 1e12, "unit": "TFLOP/s",
                     "frac": flops / (ms_step * 1e-3) / peak, "traffic": None,
                     "flops": "5 n log2 n + 9 n per pair, summed over jobs",
                     "peak_source": "measured FP32 FMA loop on this GPU (mfb_fp32_peak)"},
        "clocks": clocks,
    }


def batched_arm(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    peak = fp32_peak(local)
    rec = batched_record(dev, local, args.seed, args.jobs, args.steps, args.warmup,
                         not args.no_tune, peak, world, rank)
    if rank == 0:
        line = {"metric": BATCH_METRIC, "value": rec.pop("value"), "unit": "pairs/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": rec.pop("ms_per_step"), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded, generated on the device)",
                "config": {"workload": rec.pop("workload")},
                "gpu_launches": args.steps, "clocks": rec.pop("clocks")}
        line.update(rec)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------- large workload
LN, LND, LNT, LBIN, LBAND = 262144, 4, 2048, 4096, 262144 // 16
LSNR, LFD, LTHR = 6.0, 1e-3, 6.0
LARGE_METRIC = "filter pairs/sec at n=262144: flat and hierarchical (band n/16, fd=1e-3)"
LARGE_WORKLOAD = ("n=262144 ndata=4 ntemplates=2048 (4.3 GB of complex64 templates) binsize=4096; "
                  "templates by the config-0 formula on bins 20..n/2-1, data FFT(N(0,1))/sqrt(n), "
                  "5% of segments (at least one) injected at SNR U[6,15]; hierarchical band "
                  "n/16 with the FP32 coarse pass, snr=6, fd=1e-3, threshold=6")


def fp64_detections(D, H, thr):
    """FP64 dense correlation on the device: per (d, t, bin) whether max |z| >= thr."""
    import torch
    nb = LN // LBIN
    det = torch.zeros(LND, LNT, nb, dtype=torch.bool, device=D.device)
    D64 = D.to(torch.complex128)
    for t0 in range(0, LNT, 32):
        Hc = H[t0:t0 + 32].to(torch.complex128)
        z = torch.fft.ifft(D64[:, None, :] * torch.conj(Hc[None]), dim=-1) * LN
        m = z.abs().reshape(LND, Hc.shape[0], nb, LBIN).amax(-1)
        det[:, t0:t0 + 32] = m >= thr
        del z
    return det


def large_record(dev, local, seed, steps, warmup, coarse, cpu_sample=True, rank=0,
                 compare=None):
    """Config 4: the n = 262144 bank, flat and hierarchical, with the false
    dismissal of both against an FP64 dense correlation; `compare` names
    another coarse kind whose hierarchical run is timed beside it."""
    import torch
    import apogee_b200 as mf
    from apogee_b200 import synthetic, _lib
    D, H, power, inj = synthetic.large_workload(LN, LND, LNT, seed=seed + 1000 * rank,
                                                device=str(dev))
    gdev = "gpu:%d" % local
    flat = mf.MatchedFilter(LN, LND, LNT, device=gdev)
    flat.set_data(D)
    flat.set_templates(H)

    def make_hier(kind):
        h = mf.HierarchicalFilter(LN, LND, LNT, snr=LSNR, fd=LFD, band=LBAND, device=gdev,
                                  coarse=kind)
        h.set_reference(power.cpu().numpy())
        h.set_templates(H)
        h.set_data(D)
        return h
    hf = make_hier(coarse)
    pairs = LND * LNT
    L = _lib.lib()
    nbl = LN // LBIN
    pidx = torch.empty(pairs * nbl, dtype=torch.int64, device=dev)
    pval = torch.empty(pairs * nbl, dtype=torch.complex64, device=dev)

    def coarse_ms(h, reps=3):
        """The coarse pass and gate alone (mfb_hier_run_phase 1), CUDA events."""
        h.run_device(binsize=LBIN, threshold=LTHR)
        tot = 0.0
        for _ in range(reps):
            h._bind_stream()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            _lib.check(L.mfb_hier_run_phase(h._hplan, 1, 0, LND, 0, LNT, LBIN, LTHR, 0, LN,
                                            pidx.data_ptr(), pval.data_ptr(), None))
            b.record()
            torch.cuda.synchronize(dev)
            tot += a.elapsed_time(b)
        return tot / reps

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(dev)
        ms = []
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize(dev)
            ms.append(a.elapsed_time(b))
        return float(np.mean(ms))

    sampler = ClockSampler(local)
    sampler.start()
    flat_ms = timed(lambda: flat.run_device(binsize=LBIN, threshold=LTHR), steps,
                    max(warmup, 2))
    hier_ms = timed(lambda: hf.run_device(binsize=LBIN, threshold=LTHR), steps, max(warmup, 2))
    clocks = sampler.stop()
    hidx, _ = hf.run_device(binsize=LBIN, threshold=LTHR)
    fidx, _ = flat.run_device(binsize=LBIN, threshold=LTHR)
    det = fp64_detections(D, H, LTHR)
    n_det = int(det.sum().item())
    missed_h = int((det & (hidx < 0)).sum().item())
    missed_f = int((det & (fidx < 0)).sum().item())
    refine = hf.refine_rate
    gate = hf._coarse_value(LBAND)
    hier_coarse_ms = coarse_ms(hf)
    other = None
    if compare:
        del hf
        torch.cuda.empty_cache()
        h2 = make_hier(compare)
        h2_ms = timed(lambda: h2.run_device(binsize=LBIN, threshold=LTHR), steps,
                      max(warmup, 2))
        i2, _ = h2.run_device(binsize=LBIN, threshold=LTHR)
        other = {"coarse": compare, "value": pairs / (h2_ms * 1e-3), "ms_per_step": h2_ms,
                 "coarse_gate_ms": coarse_ms(h2), "refine_rate": h2.refine_rate,
                 "speedup_vs_flat": flat_ms / h2_ms,
                 "fp64_detections_missed": int((det & (i2 < 0)).sum().item())}
        del h2
    else:
        del hf
    del flat
    peak = fp32_peak(local)
    flops = FLOPS_PER_PAIR(LN) * pairs
    cb = None
    if cpu_sample and rank == 0:
        try:
            from oracle import refcore
            if refcore.available():
                k = 4
                r = refcore.RefFlat(LN, 1, k)
                r.set_data(D[:1].cpu().numpy())
                r.set_templates(H[:k].cpu().numpy())
                r.run(binsize=LBIN, threshold=LTHR)
                t0 = time.perf_counter()
                reps = 3
                for _ in range(reps):
                    r.run(binsize=LBIN, threshold=LTHR)
                dt = (time.perf_counter() - t0) / reps
                cb = {"value": k / dt, "unit": "pairs/s", "cores": 1, "kind": "reference",
                      "sample": "flat filter, 1 data row x %d templates of the workload, "
                                "%d runs" % (k, reps), "cpu": cpu_model()}
        except Exception as e:   # reported, not fatal
            cb = {"unavailable": str(e)}
    return {
        "workload": LARGE_WORKLOAD.replace("FP32 coarse pass", {
            "fp32": "FP32 coarse pass", "fp16x3": "FP16 split-precision tensor-core coarse "
                                                  "pass", "bf16x3": "BF16 split-precision "
                                                                    "tensor-core coarse pass"}[
            coarse]),
        "value": pairs / (hier_ms * 1e-3), "unit": "pairs/s", "ms_per_step": hier_ms,
        "gate": gate,
        "timing": "CUDA events per step, %d steps; the refine of the survivors reads their "
                  "count on the host at this n" % steps,
        "flat": {"value": pairs / (flat_ms * 1e-3), "unit": "pairs/s", "ms_per_step": flat_ms,
                 "fp64_detections_missed": missed_f},
        "hier": {"value": pairs / (hier_ms * 1e-3), "ms_per_step": hier_ms, "coarse": coarse,
                 "coarse_gate_ms": hier_coarse_ms,
                 "refine_rate": refine, "speedup_vs_flat": flat_ms / hier_ms},
        "hier_other_coarse": other,
        "false_dismissal": {"fp64_detections": n_det, "missed": missed_h,
                            "rate": missed_h / n_det if n_det else 0.0, "injections": inj},
        "roofline_flat": {"bound": "fp32", "achieved": flops / (flat_ms * 1e-3) / 1e12,
                          "peak": peak / 1e12, "unit": "TFLOP/s",
                          "frac": flops / (flat_ms * 1e-3) / peak,
                          "flops_per_pair": FLOPS_PER_PAIR(LN),
                          "peak_source": "measured FP32 FMA loop on this GPU, of measured"},
        "cpu_baseline": cb,
        "clocks": clocks,
    }


def large_arm(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rec = large_record(dev, local, args.seed, args.steps, args.warmup, args.large_coarse,
                       rank=rank, compare="fp32" if args.large_coarse != "fp32" else None)
    if rank == 0:
        line = {"metric": LARGE_METRIC, "value": rec.pop("value"), "unit": "pairs/s",
                "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": rec.pop("ms_per_step"), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded, generated on the device)",
                "config": {"workload": rec.pop("workload"), "gate": rec.pop("gate")}}
        line.update(rec)
        print(json.dumps(line))


def main():
    args = parse()
    if args.workload == "large":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the large workload's line carries the reference CPU engine "
                              "as cpu_baseline"}))
            return
        large_arm(args)
        return
    if args.workload == "batched":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no batched form; per_job_plans in our line "
                              "times the same jobs one plan per job"}))
            return
        batched_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
