"""HierarchicalFilter.run writes its table from the device straight into a
pinned host table (mfb_hier_run_host): only the rows that change since the
previous call cross the host link.  Every call must equal the dense table
of the same run (mfb_hier_run, raw output), whatever the previous call left
in the host table."""
import numpy as np
import pytest

from oracle import oracle, parity

pytestmark = pytest.mark.gpu


def noise(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _filter(n, nd, nt, band, coarse, gate):
    import apogee_b200 as mf
    hf = mf.HierarchicalFilter(n, nd, nt, band=band, coarse=coarse)
    hf.set_coarse_threshold(gate)
    return hf


def _dense(hf, **kw):
    idx, val = hf.run(raw=True, **kw)
    return idx.copy(), val.copy()


@pytest.mark.parametrize("coarse", ["fp32", "bf16x3"])
def test_host_table_equals_dense_over_changing_survivors(coarse):
    n, nd, nt, band, bs, thr = 4096, 4, 64, 512, 256, 330.0
    rng = np.random.default_rng(11)
    H = noise(rng, (nt, n))
    hf = _filter(n, nd, nt, band, coarse, 0.0)
    hf.set_templates(H)
    hf.set_data(noise(rng, (nd, n)))
    # a gate that about one pair in ten passes
    hf.set_coarse_threshold(float(np.quantile(hf.coarse_values(), 0.9)))
    seen = set()
    for _ in range(6):
        D = noise(rng, (nd, n))
        hf.set_data(D)
        out = hf.run(binsize=bs, threshold=thr)
        seen.add(hf.last_refinements)
        idx, val = _dense(hf, binsize=bs, threshold=thr)
        assert out.shape == (nd, nt, n // bs)
        np.testing.assert_array_equal(out["index"], idx)
        np.testing.assert_array_equal(out["value"], val)
        hit = (out["index"] >= 0).any(-1)
        assert 0 < hit.sum() < nd * nt
        bad = parity.compare(out["index"], out["value"], oracle.correlate(D, H), bs, thr,
                             rows_mask=hit)
        assert not bad, bad[:3]
    assert len(seen) > 1                          # the survivor sets really changed


def test_host_table_gate_extremes_and_shape_changes():
    n, nd, nt, band = 4096, 3, 40, 512
    rng = np.random.default_rng(12)
    H = noise(rng, (nt, n))
    D = noise(rng, (nd, n))
    hf = _filter(n, nd, nt, band, "bf16x3", 0.0)
    hf.set_templates(H)
    hf.set_data(D)
    z = oracle.correlate(D, H)
    # gate 0: every row refines, more than the first prefix guess (256 rows)
    big = _filter(n, 8, 64, band, "bf16x3", 0.0)
    Hb, Db = noise(rng, (64, n)), noise(rng, (8, n))
    big.set_templates(Hb)
    big.set_data(Db)
    out = big.run(binsize=512)
    assert big.last_refinements == 8 * 64
    bad = parity.compare(out["index"], out["value"], oracle.correlate(Db, Hb), 512, 0.0)
    assert not bad, bad[:3]
    # all rows refine, then none: the host copy must drop every old row
    a = hf.run(binsize=256, threshold=0.0)
    assert not parity.compare(a["index"], a["value"], z, 256, 0.0)
    hf.set_coarse_threshold(1e30)
    b = hf.run(binsize=256, threshold=0.0)
    assert hf.last_refinements == 0
    assert (b["index"] == -1).all() and (b["value"] == 0).all()
    # a window and a sub-block change the table's shape; then back again
    hf.set_coarse_threshold(0.0)
    c = hf.run(binsize=300, threshold=0.0, window=(100, 3000), data=(1, 2), templates=(5, 30))
    idx, val = _dense(hf, binsize=300, threshold=0.0, window=(100, 3000), data=(1, 2),
                      templates=(5, 30))
    np.testing.assert_array_equal(c["index"], idx)
    np.testing.assert_array_equal(c["value"], val)
    d = hf.run(binsize=256, threshold=0.0)
    assert not parity.compare(d["index"], d["value"], z, 256, 0.0)


def test_host_table_result_is_read_only():
    n, nd, nt = 4096, 2, 8
    rng = np.random.default_rng(13)
    hf = _filter(n, nd, nt, 512, "fp32", 0.0)
    hf.set_templates(noise(rng, (nt, n)))
    hf.set_data(noise(rng, (nd, n)))
    out = hf.run(binsize=1024)
    with pytest.raises(ValueError):
        out["index"][0, 0, 0] = 5
    keep = out.copy()
    keep["index"][0, 0, 0] = 5                    # a copy is the caller's


def test_host_table_bytes_and_unpinned_table_rejected():
    import ctypes
    from apogee_b200 import _lib
    n, nd, nt, nb = 4096, 2, 16, 4
    rng = np.random.default_rng(14)
    hf = _filter(n, nd, nt, 512, "bf16x3", 0.0)
    hf.set_templates(noise(rng, (nt, n)))
    hf.set_data(noise(rng, (nd, n)))
    hf.run(binsize=n // nb)
    full = nd * nt * nb * 16
    assert hf.last_d2h_bytes == full              # a new table is copied whole
    hf.run(binsize=n // nb)
    assert hf.last_d2h_bytes == full              # the same rows again: each written once
    hf.set_coarse_threshold(1e30)
    hf.run(binsize=n // nb)
    assert hf.last_d2h_bytes == full              # reset only
    hf.run(binsize=n // nb)
    assert hf.last_d2h_bytes == 0                 # nothing changes
    # a pageable host table is refused before anything is enqueued
    import torch
    rec = torch.empty(nd * nt * nb * 2, dtype=torch.int64, device="cuda")
    pageable = np.empty(nd * nt * nb * 2 + 2, np.int64)
    ptr = (pageable.ctypes.data + 15) // 16 * 16
    L = _lib.lib()
    rc = L.mfb_hier_run_host(hf._hplan, 0, nd, 0, nt, n // nb, 0.0, 0, n, None, rec.data_ptr(),
                             ctypes.c_void_p(ptr), None)
    assert rc == -1 and b"pinned" in L.mfb_last_error()


def test_held_host_bank_then_row_update():
    """set_data keeps a host bank and the device reads it at run(); a later
    single-row set_data lands on top of that bank."""
    import torch
    n, nd, nt, bs = 4096, 3, 8, 1024
    rng = np.random.default_rng(15)
    H = noise(rng, (nt, n))
    A = noise(rng, (nd, n))
    hf = _filter(n, nd, nt, 512, "bf16x3", 0.0)
    hf.set_templates(H)
    pin = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True)
    pin.numpy()[:] = A
    hf.set_data(pin.numpy())                     # pinned: one asynchronous upload at run()
    out = hf.run(binsize=bs)
    assert not parity.compare(out["index"], out["value"], oracle.correlate(A, H), bs)
    B = noise(rng, (n,))
    hf.set_data(B, index=1)
    A2 = A.copy()
    A2[1] = B
    out = hf.run(binsize=bs)
    assert not parity.compare(out["index"], out["value"], oracle.correlate(A2, H), bs)
    C = noise(rng, (nd, n))
    hf.set_data(C.astype(np.complex128))         # converted: the filter holds its own copy
    out = hf.run(binsize=bs)
    assert not parity.compare(out["index"], out["value"], oracle.correlate(C, H), bs)


def test_host_data_upload_overlapped_with_coarse_pass():
    """A held host bank reaches the device inside the run call: the band
    ahead of the coarse pass, the rest on a second stream joined before the
    refine.  Every refined row must see the whole spectrum (gate 0: all)."""
    import torch
    n, nd, nt, band, bs = 4096, 5, 24, 512, 256
    rng = np.random.default_rng(16)
    H = noise(rng, (nt, n))
    hf = _filter(n, nd, nt, band, "bf16x3", 0.0)
    hf.set_templates(H)
    for k in range(3):
        D = noise(rng, (nd, n))
        if k == 1:                                # pageable source, the same path
            src = D
        else:
            pin = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True)
            pin.numpy()[:] = D
            src = pin.numpy()
        hf.set_data(src)
        out = hf.run(binsize=bs)
        assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H), bs)
        # a sub-block run after it reads the same uploaded rows
        sub = hf.run(binsize=bs, data=(2, 3), templates=(4, 10))
        assert not parity.compare(sub["index"], sub["value"],
                                  oracle.correlate(D[2:5], H[4:14]), bs)


def test_repeated_calls_replay_one_graph_with_fresh_inputs():
    """Identical arguments from the third call on replay one captured graph
    (upload, coarse pass, refine, table update); new contents of the same
    pinned bank and other arguments in between must all come out right."""
    import torch
    n, nd, nt, band = 4096, 4, 32, 512
    rng = np.random.default_rng(17)
    H = noise(rng, (nt, n))
    hf = _filter(n, nd, nt, band, "bf16x3", 0.0)
    hf.set_templates(H)
    hf.set_data(noise(rng, (nd, n)))
    hf.set_coarse_threshold(float(np.quantile(hf.coarse_values(), 0.8)))
    pin = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True)
    for k, bs in enumerate((256, 256, 256, 256, 512, 256, 256, 256)):
        D = noise(rng, (nd, n))
        pin.numpy()[:] = D
        hf.set_data(pin.numpy())
        out = hf.run(binsize=bs, threshold=300.0)
        idx, val = _dense(hf, binsize=bs, threshold=300.0)
        np.testing.assert_array_equal(out["index"], idx)
        np.testing.assert_array_equal(out["value"], val)
        hit = (out["index"] >= 0).any(-1)
        assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H), bs, 300.0,
                                  rows_mask=hit)
    pairs, _ = hf.stats
    assert pairs == 16 * nd * nt                  # replays count their pairs once each


@pytest.mark.parametrize("n,band,coarse", [(4096, 512, "fp16x3"), (4096, 1024, "fp32"),
                                           (65536, 4096, "fp32")])
def test_host_table_other_kinds_and_lengths(n, band, coarse):
    """The host-table run for the other coarse kinds and for the two-pass
    large-n refine (no graph there: its batches are sized on the host)."""
    import torch
    nd, nt, bs = 3, 12, n // 16
    rng = np.random.default_rng(n + band)
    H = noise(rng, (nt, n))
    hf = _filter(n, nd, nt, band, coarse, 0.0)
    hf.set_templates(H)
    hf.set_data(noise(rng, (nd, n)))
    hf.set_coarse_threshold(float(np.quantile(hf.coarse_values(), 0.6)))
    pin = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True)
    for _ in range(4):
        D = noise(rng, (nd, n))
        pin.numpy()[:] = D
        hf.set_data(pin.numpy())
        out = hf.run(binsize=bs, window=(n // 32, n - 7))
        idx, val = _dense(hf, binsize=bs, window=(n // 32, n - 7))
        np.testing.assert_array_equal(out["index"], idx)
        np.testing.assert_array_equal(out["value"], val)
        hit = (out["index"] >= 0).any(-1)
        assert hit.any()
        assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H), bs, 0.0,
                                  (n // 32, n - 7), rows_mask=hit)


def _injected(rng, n, nd, H, pairs, amp=50.0):
    """Complex unit-variance noise plus `amp` * H[t] at a random lag on data
    row d for every (d, t) in pairs: with a coarse gate of 10 only those
    pairs fire (their coarse maximum is about amp * sqrt(band/n))."""
    D = (rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))) / np.sqrt(2)
    k = np.arange(n)
    for d, t in pairs:
        lag = int(rng.integers(n))
        D[d] += amp * H[t].astype(np.complex128) * np.exp(-2j * np.pi * k * lag / n)
    return D.astype(np.complex64)


def test_row_marks_over_survivor_sets():
    """Survivor sets A, A|B, B, A, then A, A|B, B again through the replayed
    graph (same pinned bank, new contents): every table equals the dense run,
    and the bytes written are (rows reset + rows refined) * nb * 16 -- a row
    refined in consecutive runs is written each time it is refined and never
    reset in between; a row refined, dropped and refined again is reset once
    and written again."""
    import torch
    n, nd, nt, band, bs = 4096, 4, 32, 512, 512
    nb = n // bs
    rng = np.random.default_rng(31)
    H = noise(rng, (nt, n))
    H /= np.linalg.norm(H, axis=1, keepdims=True)
    hf = _filter(n, nd, nt, band, "bf16x3", 10.0)
    hf.set_templates(H)
    A = {(0, 1), (1, 5), (2, 7)}
    B = {(0, 3), (3, 9), (2, 20)}
    pin = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True)
    sequence = [A, A | B, B, A, A, A | B, B]
    prev = None
    for k, S in enumerate(sequence):
        D = _injected(rng, n, nd, H, sorted(S))
        if k >= 4:                                 # same pinned bank: graph capture and replay
            pin.numpy()[:] = D
            hf.set_data(pin.numpy())
        else:
            hf.set_data(D.copy())
        out = hf.run(binsize=bs, threshold=5.0)
        assert hf.last_refinements == len(S)
        fired = {(int(d), int(t)) for d, t in zip(*np.nonzero((out["index"] >= 0).any(-1)))}
        assert fired == S, (k, fired, S)
        idx, val = _dense(hf, binsize=bs, threshold=5.0)
        np.testing.assert_array_equal(out["index"], idx)
        np.testing.assert_array_equal(out["value"], val)
        if prev is None:
            assert hf.last_d2h_bytes == nd * nt * nb * 16     # first table: copied whole
        else:
            assert hf.last_d2h_bytes == (len(prev - S) + len(S)) * nb * 16, (k, hf.last_d2h_bytes)
        prev = S


def test_replayed_run_follows_template_and_reference_changes():
    """After identical calls have captured the run as a graph, changing the
    template bank, the reference profile or the gate between two calls with
    the same arguments must give the new answer."""
    import torch
    import apogee_b200 as mf
    n, nd, nt, band, bs = 4096, 3, 24, 512, 256
    rng = np.random.default_rng(32)
    H1, H2 = noise(rng, (nt, n)), noise(rng, (nt, n))
    hf = _filter(n, nd, nt, band, "bf16x3", 0.0)
    hf.set_templates(H1)
    pin = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True)
    D = noise(rng, (nd, n))
    pin.numpy()[:] = D
    for _ in range(3):                            # direct, capture, replay
        hf.set_data(pin.numpy())
        out = hf.run(binsize=bs)
    assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H1), bs)
    hf.set_templates(H2)
    for _ in range(3):
        hf.set_data(pin.numpy())
        out = hf.run(binsize=bs)
        assert not parity.compare(out["index"], out["value"], oracle.correlate(D, H2), bs)
    # a gate that dismisses some pairs, then a reference profile that rescales
    # the coarse templates: the fired set must follow both
    cv = hf.coarse_values()
    g = float(np.quantile(cv, 0.5))
    hf.set_coarse_threshold(g)
    for _ in range(3):
        hf.set_data(pin.numpy())
        out = hf.run(binsize=bs)
    fired = (out["index"] >= 0).any(-1)
    np.testing.assert_array_equal(fired, (cv >= g))
    power = np.ones(n, np.float32)
    power[:band] = 4.0                            # in-band fraction 4/11 instead of each row's own
    hf.set_reference(power)
    cv2 = hf.coarse_values()
    assert not np.allclose(cv2, cv)
    for _ in range(2):
        hf.set_data(pin.numpy())
        out = hf.run(binsize=bs)
        fired = (out["index"] >= 0).any(-1)
        np.testing.assert_array_equal(fired, (cv2 >= g))
    flat = mf.MatchedFilter(n, nd, nt)
    flat.set_data(D)
    flat.set_templates(H2)
    ref = flat.run(binsize=bs)
    np.testing.assert_array_equal(out[fired], ref[fired])


def test_kept_results_follow_the_reuse_contract():
    """run() reuses its result table, as the reference's run does
    (python/matchedfilter/__init__.py:463-466, "The next run on this filter
    overwrites it in place; .copy() anything that must outlive that call"):
    a kept result shows the latest run, a copy keeps its own."""
    n, nd, nt, bs = 4096, 2, 8, 1024
    rng = np.random.default_rng(33)
    H = noise(rng, (nt, n))
    hf = _filter(n, nd, nt, 512, "bf16x3", 0.0)
    hf.set_templates(H)
    D1, D2 = noise(rng, (nd, n)), noise(rng, (nd, n))
    hf.set_data(D1)
    first = hf.run(binsize=bs)
    first_copy = first.copy()
    hf.set_data(D2)
    second = hf.run(binsize=bs)
    assert not parity.compare(second["index"], second["value"], oracle.correlate(D2, H), bs)
    assert not parity.compare(first_copy["index"], first_copy["value"],
                              oracle.correlate(D1, H), bs)
    np.testing.assert_array_equal(first, second)          # the reused table
    assert not (first_copy["index"] == second["index"]).all()


def test_repeated_run_skips_set_up_but_follows_every_change():
    """A run() with the arguments of the previous one and a bank held in
    place takes the short path (no argument checks or plan set-up); every
    change in between -- the bank refilled in place, another binsize or
    threshold, one data row set, new templates, a new gate -- is still seen."""
    import torch
    n, nd, nt, band = 4096, 4, 64, 512
    rng = np.random.default_rng(31)
    H = noise(rng, (nt, n))
    hf = _filter(n, nd, nt, band, "bf16x3", 0.0)
    hf.set_templates(H)
    bank = torch.empty((nd, n), dtype=torch.complex64, pin_memory=True).numpy()
    bank[:] = noise(rng, (nd, n))
    hf.set_data(bank)
    hf.set_coarse_threshold(float(np.quantile(hf.coarse_values(), 0.8)))

    def check(**kw):
        tab = hf.run(**kw).copy()
        assert hf._repeat is not None
        idx, val = _dense(hf, **kw)
        np.testing.assert_array_equal(tab["index"], idx)
        np.testing.assert_array_equal(tab["value"], val)
        return tab

    kw = dict(binsize=256, threshold=0.0)
    check(**kw)
    for step in range(3):
        bank[:] = noise(rng, (nd, n))
        bank[step % nd] += (50 * H[7 * step + 1].astype(np.complex128) *
                            np.exp(-2j * np.pi * np.arange(n) * (100 + step) / n)).astype(np.complex64)
        hf.set_data(bank)                      # the same array: refilled in place
        tab = check(**kw)
        assert tab["index"][step % nd, 7 * step + 1, 0] == 100 + step
    check(binsize=512, threshold=0.0)
    check(binsize=512, threshold=20.0)
    hf.set_data(noise(rng, n), index=2)        # one row: the bank goes to the device mirror
    check(binsize=512, threshold=20.0)
    hf.set_templates(noise(rng, (nt, n)))
    check(binsize=512, threshold=20.0)
    hf.set_coarse_threshold(0.0)               # every pair refined
    tab = check(binsize=512, threshold=20.0)
    assert (tab["index"] >= 0).any()
    bank[:] = noise(rng, (nd, n))
    hf.set_data(bank)
    check(binsize=512, threshold=20.0)
    check(binsize=512, threshold=20.0, window=(0, n))    # a tuple window: same result
