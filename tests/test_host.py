"""Host-side logic that needs no GPU: layouts, argument checks, device specs."""
import numpy as np
import pytest

import apogee_b200 as mf
from apogee_b200._series import SeriesLayout
from apogee_b200 import device


def test_peak_dtype_is_the_reference_layout():
    assert mf.PEAK_DTYPE == np.dtype([("index", "<i8"), ("value", "<c8")])
    assert mf.PEAK_DTYPE.itemsize == 16


def test_series_layout_groups_and_restores_order():
    st = np.array([0, 10, 20, 30, 40], np.int64)
    lo = np.array([5, 0, 5, 0, 5], np.int64)
    hi = np.array([50, 45, 50, 45, 50], np.int64)
    lay = SeriesLayout(64, st, lo, hi, 16).group()
    assert lay.nbins == 3
    assert lay.order is not None
    # grouped windows are contiguous and cover every block once
    assert sorted(lay.order.tolist()) == list(range(5))
    spans = [(a, b) for (_, _, a, b) in lay.groups]
    assert spans[0][0] == 0 and spans[-1][1] == 5
    assert np.all(lay.starts == st[lay.order])


def test_series_layout_refuses_unequal_bin_counts():
    with pytest.raises(ValueError):
        SeriesLayout(64, np.zeros(2, np.int64), np.array([0, 0]), np.array([64, 10]), 16)
    with pytest.raises(ValueError):
        SeriesLayout(64, np.zeros(1, np.int64), np.array([10]), np.array([10]), 16)


def test_series_layout_keeps_adjacent_groups_in_order():
    st = np.arange(4, dtype=np.int64)
    lo = np.array([0, 0, 3, 3])
    hi = np.array([60, 60, 63, 63])
    lay = SeriesLayout(64, st, lo, hi, 32).group()
    assert lay.order is None
    assert [g[2:] for g in lay.groups] == [(0, 2), (2, 4)]


def test_device_spec_parsing_without_gpu(monkeypatch):
    monkeypatch.setattr(device, "devices", lambda: [device.Device(0, "fake"), device.Device(1, "fake")])
    assert device.parse(None) == "gpu:0"
    assert device.parse("cuda:1").index == 1
    assert device.parse("gpu:1") == device.Device(1)
    with pytest.raises(ValueError):
        device.parse("cpu")
    with pytest.raises(ValueError):
        device.parse("tpu")
    with pytest.raises(ValueError):
        device.parse("gpu:7")
    with pytest.raises(TypeError):
        device.parse(3)
    monkeypatch.setenv("MF_DEVICE", "gpu:1")
    assert device.parse(None).index == 1


def test_no_cpu_fallback_without_device(monkeypatch):
    monkeypatch.setattr(device, "devices", lambda: [])
    with pytest.raises(RuntimeError):
        mf.MatchedFilter(4096, 1, 1)


def test_batch_own_launch_rule():
    """A job leaves the persistent launch when forced, or when its pairs times
    the measured per-pair saving exceed the launch cost."""
    from apogee_b200.batch import DEDICATED_LAUNCH_US, Job, dedicated
    H = np.zeros((100, 4096), np.complex64)
    D = np.zeros((10, 4096), np.complex64)
    job = Job(H, data=D, binsize=256)              # 1000 pairs
    assert not dedicated(job, {})
    assert dedicated(job, {"dedicated": True})
    gain = DEDICATED_LAUNCH_US / 1000.0
    assert dedicated(job, {"pp_us": 0.02 + 2 * gain, "dedicated_pp_us": 0.02})
    assert not dedicated(job, {"pp_us": 0.02 + 0.5 * gain, "dedicated_pp_us": 0.02})


def test_costmodel_candidates_and_pick():
    """Band candidates span n/16 .. n/2 (>= 64, as the kind allows); the
    fastest measured band wins and ties go to the wider band."""
    from apogee_b200 import costmodel
    assert costmodel.candidate_bands(4096, lambda b: True) == [256, 512, 1024, 2048]
    assert costmodel.candidate_bands(4096, lambda b: b == 512) == [512]
    assert costmodel.candidate_bands(512, lambda b: True) == [64, 128, 256]
    assert costmodel.pick({256: 40.0, 512: 31.0, 1024: 55.0}) == 512
    assert costmodel.pick({256: 30.0, 512: 30.0}) == 512
    with pytest.raises(ValueError):
        costmodel.pick({})


def test_coarse_kind_auto_and_tensor_core_bands():
    """coarse="auto" takes the BF16 split tensor-core pass at the bands where
    it is the faster (AUTO_TC_BANDS) and the FP32 pass elsewhere; the explicit
    tensor-core kinds cover TC_BANDS only."""
    import apogee_b200 as mf
    from apogee_b200 import _lib
    assert mf.AUTO_TC_BANDS <= mf.TC_BANDS
    assert mf._coarse_kind("auto", 512) == _lib.COARSE_BF16X3
    assert mf._coarse_kind("auto", 16384) == _lib.COARSE_FP32
    assert mf._coarse_kind("auto", 1024) == _lib.COARSE_FP32
    assert mf._coarse_kind("auto") is None
    assert mf._coarse_kind("fp16x3", 16384) == _lib.COARSE_FP16X3
    import pytest
    with pytest.raises(ValueError):
        mf._coarse_kind("tf32")


def test_large_workload_subsample_is_the_full_banks_draws():
    """A materialised subsample of the large-bank generator has the full
    bank's data, profile and injections (CPU torch)."""
    import numpy as np
    import torch
    from apogee_b200 import synthetic
    n, nt = 1024, 12
    D1, H1, p1, inj1 = synthetic.large_workload(n, 3, nt, seed=4, device="cpu", chunk=5)
    D2, H2, p2, inj2 = synthetic.large_workload(n, 3, nt, seed=4, device="cpu", chunk=5,
                                                materialize=[2, 7, 11])
    assert inj1 == inj2
    torch.testing.assert_close(D1, D2)
    torch.testing.assert_close(p1, p2)
    torch.testing.assert_close(H1[[2, 7, 11]], H2)
    assert np.isclose(float(p1.sum()) * n / n, float((H1.abs().double() ** 2).mean(0).sum()),
                      rtol=1e-6)


def test_repeat_key_accepts_only_immutable_arguments():
    """run() arguments that a later call can be compared with by value (None,
    numbers, tuples of ints) identify a repeat; lists, arrays and NaN do not."""
    import numpy as np
    from apogee_b200 import _repeat_key
    assert _repeat_key(256, 5.5, None, None, None) == (256, 5.5, None, None, None)
    assert _repeat_key(None, 0, (0, 4096), (0, 16), (8, 64)) is not None
    assert _repeat_key(256, 5.5, [0, 4096], None, None) is None
    assert _repeat_key(256, 5.5, np.array([0, 4096]), None, None) is None
    assert _repeat_key(256, float("nan"), None, None, None) is None
    assert _repeat_key(np.int64(256), 5.5, None, None, None) is None
    assert _repeat_key(256, np.float32(5.5), None, None, None) is None
    assert _repeat_key(256, 5.5, (0, 4096.0), None, None) is None
