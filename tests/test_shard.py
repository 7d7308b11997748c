"""Template sharding across ranks: two gloo ranks on CPU, each filtering its
template slice with an oracle-backed engine, assemble the same table as one
process filtering the whole bank."""
import os
import socket

import numpy as np
import pytest

from apogee_b200.shard import PEAK_DTYPE, template_slice


def test_template_slices_cover_the_bank():
    for nt in (1, 2, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            if nt < world:
                continue
            slices = [template_slice(nt, r, world) for r in range(world)]
            assert slices[0][0] == 0
            for (a, n_a), (b, _) in zip(slices, slices[1:]):
                assert a + n_a == b
            assert sum(c for _, c in slices) == nt
            assert max(c for _, c in slices) - min(c for _, c in slices) <= 1
    with pytest.raises(ValueError):
        template_slice(4, 2, 2)


class OracleEngine:
    """CPU stand-in for the rank-local GPU filter (test-only)."""

    def __init__(self, n, nd, nt):
        self.n, self.nd, self.nt = n, nd, nt
        self.pairs, self.trig = 0, 0

    def set_data(self, D):
        self.D = np.asarray(D)

    def set_templates(self, H):
        assert H.shape[0] == self.nt
        self.H = np.asarray(H)

    def run(self, binsize=None, threshold=0.0, window=None):
        from oracle import oracle
        idx, val, cnt, _ = oracle.flat(self.D, self.H, binsize, threshold, window)
        out = np.empty(idx.shape, PEAK_DTYPE)
        out["index"], out["value"] = idx, val
        self.pairs += self.nd * self.nt
        self.trig += int((idx >= 0).any(-1).sum())
        return out

    def run_records(self, binsize=None, threshold=0.0, window=None):
        import torch
        out = self.run(binsize, threshold, window)
        return torch.from_numpy(out.view(np.int64).reshape(out.shape + (2,)).copy())

    @property
    def stats(self):
        return self.pairs, self.trig


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir):
    import torch.distributed as dist
    from apogee_b200.shard import ShardedFilter
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, nd, nt, bs, thr = case
        rng = np.random.default_rng(5)
        D = (rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))).astype(np.complex64)
        H = (rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))).astype(np.complex64)
        f = ShardedFilter(n, nd, nt, engine=OracleEngine)
        f.set_data(D)
        f.set_templates(H)
        full = f.run(binsize=bs, threshold=thr)
        rec = f.run_records(binsize=bs, threshold=thr)
        assert tuple(rec.shape) == full.shape + (2,)
        np.testing.assert_array_equal(rec.numpy().view(PEAK_DTYPE)[..., 0], full)
        pairs, trig = f.stats
        np.save(os.path.join(out_dir, "r%d.npy" % rank), full)
        np.save(os.path.join(out_dir, "s%d.npy" % rank), np.array([pairs, trig]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [(256, 3, 7, 32, 0.0), (512, 2, 4, 512, 20.0)])
def test_two_gloo_ranks_assemble_the_full_table(tmp_path, case):
    import torch.multiprocessing as mp
    from oracle import oracle
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), case, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    n, nd, nt, bs, thr = case
    rng = np.random.default_rng(5)
    D = (rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))).astype(np.complex64)
    H = (rng.standard_normal((nt, n)) + 1j * rng.standard_normal((nt, n))).astype(np.complex64)
    idx, val, _, _ = oracle.flat(D, H, bs, thr)
    for r in range(world):
        full = np.load(tmp_path / ("r%d.npy" % r))
        assert full.dtype == PEAK_DTYPE and full.shape == idx.shape
        np.testing.assert_array_equal(full["index"], idx)
        np.testing.assert_array_equal(full["value"], val.astype(np.complex64))
        pairs, trig = np.load(tmp_path / ("s%d.npy" % r))
        assert pairs == 2 * nd * nt                 # run and run_records
        assert trig == 2 * int((idx >= 0).any(-1).sum())
