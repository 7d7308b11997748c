"""mfb_run_large_static, the entry point that allocates nothing, called through
the C ABI and compared with mfb_run (through MatchedFilter) on two calls in a
row.  The file name sorts last so that it also runs after every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_run(L, D, H, binsize, threshold, start, end):
    import torch
    n = D.shape[1]
    nd, nt = D.shape[0], H.shape[0]
    nb = L.mfb_nbins(n, binsize, start, end)
    idx = torch.full((nd * nt * nb,), -7, dtype=torch.int64, device=D.device)
    val = torch.zeros(nd * nt * nb, dtype=torch.complex64, device=D.device)
    cnt = torch.full((nd * nt,), 99, dtype=torch.int32, device=D.device)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(D.device)[0]
    rc = L.mfb_run_large_static(D.device.index, n, D.data_ptr(), nd, H.data_ptr(), nt, binsize,
                                threshold, start, end, idx.data_ptr(), val.data_ptr(),
                                cnt.data_ptr(), torch.cuda.current_stream(D.device).cuda_stream)
    assert rc == 0, L.mfb_last_error().decode()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(D.device)[0]
    return (idx.cpu().numpy().reshape(nd, nt, nb), val.cpu().numpy().reshape(nd, nt, nb),
            cnt.cpu().numpy().reshape(nd, nt), free0 - free1)


@pytest.mark.parametrize("n", [65536, 262144, 524288])
def test_static_matches_planned_twice(n):
    import torch
    import apogee_b200 as mf
    from apogee_b200._lib import lib
    L = lib()
    rng = np.random.default_rng(n + 11)
    nd, nt = 2, 5
    Dn = (rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))).astype(np.complex64)
    Hn = (rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))).astype(np.complex64)
    D = torch.from_numpy(Dn).to("cuda:0")
    H = torch.from_numpy(Hn).to("cuda:0")
    f = mf.MatchedFilter(n, nd, nt)
    f.set_data(Dn)
    f.set_templates(Hn)
    calls = [(n // 64, 0.0, 0, n), (n // 100 + 3, 3.0 * np.sqrt(n), 17, n - 9)]
    for call, (binsize, thr, start, end) in enumerate(calls):
        ref, ref_cnt = f.run(binsize=binsize, threshold=thr, window=(start, end), counts=True)
        idx, val, cnt, grown = _static_run(L, D, H, binsize, thr, start, end)
        np.testing.assert_array_equal(idx, ref["index"])
        scale = np.abs(ref["value"]).max()
        np.testing.assert_allclose(val, ref["value"], rtol=1e-5, atol=1e-6 * scale)
        np.testing.assert_array_equal(cnt, ref_cnt)
        if call == 1:
            assert grown == 0, "device memory fell by %d bytes during the call" % grown


def test_static_refuses_sizes_beyond_its_scratch():
    import torch
    from apogee_b200._lib import lib, MFB_ERR_UNSUPPORTED
    L = lib()
    buf = torch.zeros(16, dtype=torch.complex64, device="cuda:0")
    out = torch.zeros(16, dtype=torch.int64, device="cuda:0")
    p = buf.data_ptr()
    for n, binsize in [(1 << 20, 1 << 12), (1 << 14, 1 << 10), (1 << 16, 8)]:
        rc = L.mfb_run_large_static(0, n, p, 1, p, 1, binsize, 0.0, 0, n, out.data_ptr(), p,
                                    None, None)
        assert rc == MFB_ERR_UNSUPPORTED
        msg = L.mfb_last_error().decode()
        assert ("bytes of scratch" in msg) == (n == 1 << 20), msg
