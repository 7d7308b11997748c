"""The benchmark's shared coarse threshold is the one the FP64 recipe in
tests/golden/make_gate.py derived (tests/golden/gate_config1.json)."""
import json
import os

import bench

HERE = os.path.dirname(os.path.abspath(__file__))


def test_bench_gate_is_the_fp64_derived_gate():
    with open(os.path.join(HERE, "golden", "gate_config1.json")) as fh:
        g = json.load(fh)
    assert g["gate"] == bench.CAL_GATE
    assert (g["n"], g["band"], g["snr"], g["fd"]) == (bench.N, bench.BAND, bench.SNR, bench.FD)
    cfg = bench.workload_config()
    assert cfg["gate_value"] == bench.CAL_GATE and cfg["pairs_per_gpu"] == bench.ND * bench.NT
