"""ShardedFilter on the GPU: one NCCL rank with the default engine
(MatchedFilter and HierarchicalFilter on the rank's device) gives the plain
filter's table; the all-gather runs on the device."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    import apogee_b200 as mf
    from apogee_b200.shard import ShardedFilter
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        n, nd, nt = 4096, 3, 9
        rng = np.random.default_rng(1)
        D = (rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))).astype(np.complex64)
        H = (rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))).astype(np.complex64)
        f = ShardedFilter(n, nd, nt)
        f.set_data(D)
        f.set_templates(H)
        a = f.run(binsize=256)
        ref = mf.MatchedFilter(n, nd, nt)
        ref.set_data(D)
        ref.set_templates(H)
        b = ref.run(binsize=256)
        h = ShardedFilter(n, nd, nt, kind="hier", band=512, coarse="fp32")
        h.local.set_coarse_threshold(0.0)
        h.set_data(D)
        h.set_templates(H)
        c = h.run(binsize=256)
        # the device-resident assembly: records stay on the GPU
        rec = f.run_records(binsize=256)
        hrec = h.run_records(binsize=256)
        dev_ok = rec.is_cuda and hrec.is_cuda
        r = rec.cpu().numpy().view(mf.PEAK_DTYPE)[..., 0]
        hr = hrec.cpu().numpy().view(mf.PEAK_DTYPE)[..., 0]
        np.save(os.path.join(out_dir, "ok.npy"), np.array([
            int(np.array_equal(a, b)), int(np.array_equal(c, b)),
            int(dev_ok and np.array_equal(r, b) and np.array_equal(hr, b)), *h.stats]))
    finally:
        dist.destroy_process_group()


def test_one_nccl_rank_matches_plain_filter(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=1, join=True,
                       start_method="spawn")
    flat_ok, hier_ok, rec_ok, pairs, trig = np.load(tmp_path / "ok.npy")
    assert flat_ok == 1 and hier_ok == 1 and rec_ok == 1
    assert pairs == 54 and trig == 54
