"""The thread-block-cluster kernel (n = 32768 and 65536: one cluster per
pair, the spectrum held in distributed shared memory between the passes)
against the two-pass kernels it replaces (same arithmetic: identical outputs)
and against the FP64 oracle: dense blocks with more pairs than clusters,
windows, thresholds, ragged bins, listed rows and the hierarchical refine."""
import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _modes(f, **kw):
    """Run with the two cluster geometries and with the two-pass kernels."""
    from apogee_b200 import _lib
    L = _lib.lib()
    outs = []
    for mode in (1, 2, 0):
        _lib.check(L.mfb_set_cluster(f._plan, mode))
        out, cnt = f.run(counts=True, **kw)     # buffers reused by the next run
        outs.append((out.copy(), cnt.copy()))
    _lib.check(L.mfb_set_cluster(f._plan, 0))
    return outs


@pytest.mark.parametrize("n", [32768, 65536])
def test_cluster_equals_two_pass_and_oracle(n):
    import apogee_b200 as mf
    rng = np.random.default_rng(n + 11)
    nd, nt = 6, 40                       # 240 pairs: more than the GPU's clusters
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    # a few loud pairs so thresholds leave some bins empty and some full
    for d, t, lag in [(0, 3, 17), (4, 39, n - 2), (5, 0, n // 2 + 1)]:
        D[d] += (30 * H[t].astype(np.complex128) *
                 np.exp(-2j * np.pi * np.arange(n) * lag / n)).astype(np.complex64)
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    sel_t = [0, 3, 39]
    z = oracle.correlate(D, H[sel_t])
    for binsize, thr, win in [(n // 16, 0.0, None), (n // 64, 0.0, None),
                              (n // 100 + 7, 0.0, (13, n - 5)),
                              (n // 8, 5.0 * np.sqrt(n), (n // 3, n)), (n, 0.0, None),
                              (1000, 0.0, (n // 2 - 20000, n // 2 + 20000)),
                              (n // 16, 0.0, (n // 16, n)),        # window on a bin edge
                              (16, 0.0, None)]:                    # 2048 / 4096 bins
        (a, ca), (a2, ca2), (b, cb) = _modes(f, binsize=binsize, threshold=thr, window=win)
        for x, cx in ((a, ca), (a2, ca2)):
            np.testing.assert_array_equal(x["index"], b["index"])
            np.testing.assert_array_equal(x["value"], b["value"])
            np.testing.assert_array_equal(cx, cb)
        np.testing.assert_array_equal(ca, (a["index"] >= 0).sum(-1))
        bad = parity.compare(a["index"][:, sel_t], a["value"][:, sel_t], z, binsize, thr, win)
        assert not bad, (binsize, thr, win, bad[:3])
    out = f.run(binsize=n // 16)
    assert out["index"][0, 3, 0] == 17 and out["index"][4, 39, 15] == n - 2


@pytest.mark.parametrize("n", [32768, 65536])
def test_cluster_listed_rows(n):
    """Listed runs read their row count on the device; rows not listed keep
    what the caller put there."""
    import torch
    import apogee_b200 as mf
    from apogee_b200 import _lib
    rng = np.random.default_rng(n + 12)
    nd, nt, binsize = 3, 20, n // 64
    D, H = noise(rng, (nd, n)), noise(rng, (nt, n))
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(D)
    f.set_templates(H)
    L = _lib.lib()
    nb = n // binsize
    rows = np.sort(rng.choice(nd * nt, size=23, replace=False)).astype(np.int32)
    dev = torch.device("cuda")
    res = []
    for mode in (1, 2, 0):
        _lib.check(L.mfb_set_cluster(f._plan, mode))
        f._bind_stream()
        idx = torch.full((nd * nt * nb,), -7, dtype=torch.int64, device=dev)
        val = torch.zeros(nd * nt * nb, dtype=torch.complex64, device=dev)
        r = torch.tensor(rows, device=dev)
        cnt = torch.tensor([len(rows)], dtype=torch.int32, device=dev)
        _lib.check(L.mfb_run_rows(f._plan, 0, nd, 0, nt, r.data_ptr(), cnt.data_ptr(), len(rows),
                                  binsize, 0.0, 0, n, idx.data_ptr(), val.data_ptr(), None))
        torch.cuda.synchronize()
        res.append((idx.view(nd * nt, nb).cpu().numpy(), val.view(nd * nt, nb).cpu().numpy()))
    _lib.check(L.mfb_set_cluster(f._plan, 0))
    for other in res[1:]:
        np.testing.assert_array_equal(res[0][0], other[0])
        np.testing.assert_array_equal(res[0][1], other[1])
    listed = np.zeros(nd * nt, bool)
    listed[rows] = True
    assert (res[0][0][~listed] == -7).all()
    dense = f.run(binsize=binsize)
    np.testing.assert_array_equal(res[0][0][listed], dense["index"].reshape(nd * nt, nb)[listed])
    np.testing.assert_array_equal(res[0][1][listed], dense["value"].reshape(nd * nt, nb)[listed])


def test_cluster_hierarchical_refine_and_host_table():
    """Hierarchical filter at n = 32768 with the cluster refine: its table
    equals the two-pass refine's, and the host-table run (replayed as one
    CUDA graph at this length, since no step reads the survivor count on the
    host) matches the device table over changing data."""
    import apogee_b200 as mf
    from apogee_b200 import _lib
    n, nd, nt = 32768, 4, 64
    rng = np.random.default_rng(21)
    H = noise(rng, (nt, n))
    power = (np.abs(H.astype(np.complex128)) ** 2).mean(0).astype(np.float32)
    hf = mf.HierarchicalFilter(n, nd, nt, snr=6.0, fd=1e-2, band=2048)
    hf.set_reference(power)
    hf.set_templates(H)
    hf.set_coarse_threshold(2.5)
    L = _lib.lib()
    hf._prepare()
    _lib.check(L.mfb_hier_set_cluster(hf._hplan, 1))
    for step in range(4):
        D = noise(rng, (nd, n))
        t, lag = int(rng.integers(nt)), int(rng.integers(n))
        D[step % nd] += (20 * H[t].astype(np.complex128) *
                         np.exp(-2j * np.pi * np.arange(n) * lag / n)).astype(np.complex64)
        hf.set_data(D)
        tab = hf.run(binsize=n // 16, threshold=0.0).copy()
        ridx, rval = (x.copy() for x in hf.run(raw=True, binsize=n // 16, threshold=0.0))
        np.testing.assert_array_equal(tab["index"], ridx)
        np.testing.assert_array_equal(tab["value"], rval)
        hf._prepare()
        _lib.check(L.mfb_hier_set_cluster(hf._hplan, 0))
        oidx, oval = hf.run(raw=True, binsize=n // 16, threshold=0.0)
        _lib.check(L.mfb_hier_set_cluster(hf._hplan, 1))
        np.testing.assert_array_equal(ridx, oidx)
        np.testing.assert_array_equal(rval, oval)
        assert tab["index"][step % nd, t, lag // (n // 16)] == lag


def test_cluster_mode_argument_checked():
    """Modes 0, 1 and 2 are accepted at any length (they select nothing below
    n = 32768); anything else is an argument error."""
    import apogee_b200 as mf
    from apogee_b200 import _lib
    L = _lib.lib()
    for n in (4096, 32768):
        f = mf.MatchedFilter(n, 1, 1)
        for mode in (0, 1, 2):
            assert L.mfb_set_cluster(f._plan, mode) == 0
        for mode in (-1, 3):
            assert L.mfb_set_cluster(f._plan, mode) == _lib.MFB_ERR_ARG
            assert "cluster mode" in L.mfb_last_error().decode()
