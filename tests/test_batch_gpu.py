"""Batched uneven jobs in one persistent launch, against the FP64 oracle:
mixed n (single-CTA and four-step), binsizes, thresholds, windows and series
jobs; every four-step split; repeated runs and CUDA-graph replays."""
import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def make_jobs(seed=0):
    from apogee_b200.batch import Job
    rng = np.random.default_rng(seed)
    spec = [  # n, nd, nt, binsize, threshold, window
        (64, 3, 50, 16, 0.0, None),
        (256, 2, 33, 7, 0.0, (5, 250)),
        (1024, 5, 40, 64, 0.0, None),
        (2048, 1, 17, 2048, 0.0, None),
        (4096, 4, 30, 256, 3.0 * 64, None),
        (8192, 3, 7, 128, 0.0, None),
        (16384, 2, 9, 1024, 0.0, (100, 16000)),
        (32768, 2, 5, 512, 0.0, None),
        (65536, 3, 4, 1024, 0.0, None),
        (65536, 1, 3, 4096, 2.0 * 256, (1000, 60000)),
    ]
    jobs, refs = [], []
    for n, nd, nt, bs, thr, win in spec:
        D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
        jobs.append(Job(H, data=D, binsize=bs, threshold=thr, window=win))
        refs.append((oracle.correlate(D, H), bs, thr, win))
    # series jobs: real time series cut into overlapping blocks
    for n, nblk, nt, bs in [(1024, 6, 11, 64), (32768, 3, 4, 2048)]:
        x = rng.standard_normal(nblk * n // 2 + n // 3).astype(np.float32)
        starts = np.arange(nblk) * (n // 2)
        H = noise(rng, (nt, n))
        win = (n // 8, n)
        jobs.append(Job(H, series=x, starts=starts, binsize=bs, window=win))
        D = oracle.series_spectra(x, starts, n)
        refs.append((oracle.correlate(D, H), bs, 0.0, win))
    return jobs, refs


def check(bf, refs):
    for i, (z, bs, thr, win) in enumerate(refs):
        r = bf.result(i)
        bad = parity.compare(r["index"], r["value"], z, bs, thr, win)
        assert not bad, (i, bf.jobs[i].n, bad[:3])


def test_mixed_batch_parity_and_repeats():
    from apogee_b200.batch import BatchedFilter
    jobs, refs = make_jobs()
    bf = BatchedFilter(jobs)
    info = bf.info()
    assert info["tickets"] > 0 and info["grid"] >= 148
    bf.run()
    bf.wait()
    check(bf, refs)
    first = [bf.result(i).copy() for i in range(len(jobs))]
    bf.run()
    bf.wait()
    for i in range(len(jobs)):
        np.testing.assert_array_equal(bf.result(i), first[i])


def test_graph_replay_matches():
    import torch
    from apogee_b200.batch import BatchedFilter
    jobs, refs = make_jobs(seed=1)
    bf = BatchedFilter(jobs, slot_bytes=1 << 20, slots=2)   # many small batches, slot reuse
    assert bf.info()["batches"] > 10
    bf.capture()
    for _ in range(2):
        for r in bf._records:
            r.fill_(7)
        bf.replay()
        torch.cuda.synchronize()
        bf.wait()
        check(bf, refs)


@pytest.mark.parametrize("split", [64, 128, 256])
def test_every_split(split):
    from apogee_b200.batch import BatchedFilter, Job
    rng = np.random.default_rng(split)
    n = 16384
    D, H = noise(rng, (2, n)), noise(rng, (6, n))
    bf = BatchedFilter([Job(H, data=D, binsize=n // 64)], tune={n: {"split": split}})
    (r,) = bf.results()
    assert not parity.compare(r["index"], r["value"], oracle.correlate(D, H), n // 64)


@pytest.mark.parametrize("items", [1, 3, 8])
def test_small_unit_sizes(items):
    from apogee_b200.batch import BatchedFilter, Job
    rng = np.random.default_rng(items)
    n = 512
    D, H = noise(rng, (3, n)), noise(rng, (45, n))
    bf = BatchedFilter([Job(H, data=D, binsize=32)], tune={n: {"unit_items": items}})
    (r,) = bf.results()
    assert not parity.compare(r["index"], r["value"], oracle.correlate(D, H), 32)


def test_autotuner_picks_a_valid_config():
    from apogee_b200 import autotune
    from apogee_b200.batch import BatchedFilter, Job
    for n in (2048, 32768):
        cfg = autotune.tune(n)
        kernel_cfg = {k: v for k, v in cfg.items() if k in ("split", "unit_items")}
        assert kernel_cfg in autotune.candidates(n)
        assert cfg["pp_us"] > 0 and cfg["dedicated_pp_us"] > 0
    rng = np.random.default_rng(5)
    n = 32768
    D, H = noise(rng, (2, n)), noise(rng, (3, n))
    bf = BatchedFilter([Job(H, data=D, binsize=n // 16)], tune=True)
    (r,) = bf.results()
    assert not parity.compare(r["index"], r["value"], oracle.correlate(D, H), n // 16)


def test_plan_errors():
    from apogee_b200.batch import BatchedFilter, Job
    rng = np.random.default_rng(0)
    n = 8192
    D, H = noise(rng, (1, n)), noise(rng, (1, n))
    with pytest.raises(ValueError):
        BatchedFilter([Job(H, data=D, binsize=64)], tune={n: {"split": 256}})   # N1 = 32
    with pytest.raises(ValueError):
        Job(H, data=D, binsize=1)   # 8192 bins > 4096 for the four-step


def test_own_launch_jobs_beside_the_persistent_launch():
    """Jobs forced onto their own launches (single-CTA 8192/16384, two-pass
    65536, a series job) next to persistent ones: same results, also replayed
    from a graph."""
    import torch
    from apogee_b200.batch import BatchedFilter
    jobs, refs = make_jobs(seed=2)
    own_n = {8192, 16384, 65536, 1024}
    tune = {n: {"dedicated": True} for n in own_n}
    bf = BatchedFilter(jobs, tune=tune)
    info = bf.info()
    assert info["own_launch_jobs"] == sum(1 for j in jobs if j.n in own_n)
    assert info["tickets"] > 0
    bf.run()
    bf.wait()
    check(bf, refs)
    bf.capture()
    for r in bf._records:
        r.fill_(7)
    bf.replay()
    torch.cuda.synchronize()
    bf.wait()
    check(bf, refs)
    # every job on its own launches: no persistent launch at all
    solo = BatchedFilter(jobs[:3], tune={j.n: {"dedicated": True} for j in jobs[:3]})
    assert solo.info()["tickets"] == 0
    solo.run()
    solo.wait()
    for i in range(3):
        z, bs, thr, win = refs[i]
        r = solo.result(i)
        assert not parity.compare(r["index"], r["value"], z, bs, thr, win)



def test_dependency_wait_runs_out_and_is_reported():
    """Failure detection without a GPU fault: pass B of the first four-step
    batch is made to wait for a pass-A unit that never comes.  The bounded
    wait runs out, the launch stops and returns, wait() raises, and the same
    plan runs correctly once restored."""
    import time
    from apogee_b200 import _lib
    from apogee_b200.batch import BatchedFilter, Job
    rng = np.random.default_rng(31)
    n = 32768
    D, H = noise(rng, (2, n)), noise(rng, (3, n))
    d2, h2 = noise(rng, (2, 1024)), noise(rng, (5, 1024))
    bf = BatchedFilter([Job(H, data=D, binsize=1024), Job(h2, data=d2, binsize=64)],
                       tune={n: {"split": 128}, 1024: {"unit_items": 2}})
    L = _lib.lib()
    _lib.check(L.mfb_batch_test_wait_limit(bf._plan, 1))
    t0 = time.perf_counter()
    bf.run()
    with pytest.raises(RuntimeError, match="dependency wait ran out"):
        bf.wait()
    assert time.perf_counter() - t0 < 60
    _lib.check(L.mfb_batch_test_wait_limit(bf._plan, -1))
    bf.run()
    bf.wait()
    r = bf.result(0)
    assert not parity.compare(r["index"], r["value"], oracle.correlate(D, H), 1024)
    r = bf.result(1)
    assert not parity.compare(r["index"], r["value"], oracle.correlate(d2, h2), 64)
