"""The benchmark's roofline inputs, checked on CPU: the algorithmic bytes
of one MTTKRP (index/value stream once, each factor once, output once) and
the DRAM traffic per MTTKRP that bench.py reads from the committed ncu
summaries for the full-size workloads."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_algorithmic_bytes_of_the_headline_workload():
    dims, nnz, R = bench.WORKLOAD["dims"], bench.WORKLOAD["nnz"], bench.WORKLOAD["rank"]
    # FP64: 16 B per nonzero + 2 input factors + output
    b0 = bench.mttkrp_alg_bytes(dims, nnz, R, 0)
    assert b0 == nnz * 16 + (dims[1] + dims[2]) * R * 8 + dims[0] * R * 8
    # mixed FP32: 12 B per nonzero, 4-byte factors and output
    b = [bench.mttkrp_alg_bytes(dims, nnz, R, m, 8, 4, 4, 4) for m in range(3)]
    assert abs(b[0] / 1e9 - 2.915) < 0.01


def test_algorithmic_bytes_of_the_wide_workload():
    dims, nnz, R = bench.WIDE["dims"], bench.WIDE["nnz"], bench.WIDE["rank"]
    b = [bench.mttkrp_alg_bytes(dims, nnz, R, m) for m in range(4)]
    # every mode reads the same stream and touches each factor once
    assert len(set(b)) == 1 and abs(b[0] / 1e9 - 2.406) < 0.01


def test_traffic_read_from_committed_profiles():
    t = bench.traffic_from_profiles("mixed_f32", bench.WORKLOAD["nnz"])
    assert t is not None and 5e9 < t < 1e10
    w = bench.traffic_from_profiles("fp64", bench.WIDE["nnz"], "mttkrp_wide_zipf_2p20x3x4096_r32.md", bench.WIDE["nnz"])
    assert w is not None and 5e9 < w < 2e10
    # another size has no full-size capture
    assert bench.traffic_from_profiles("mixed_f32", 1000) is None
