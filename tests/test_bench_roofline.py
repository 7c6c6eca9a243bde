"""The benchmark's roofline arithmetic on the CPU: the on-chip bound of the
hot-path scope (2 * W * elem_bytes * max(0, log2 W - 10) bytes per array at the
measured shared-memory copy rate), the distributed-shared-memory reads of
the cluster kernels, and the layer counts behind the ALU model."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.fixture
def bench(monkeypatch):
    import bench as b
    monkeypatch.setattr(b, "onchip_peaks", lambda device, cluster=0: {
        "smem_read_gbs": 30000.0, "smem_copy_gbs": 20000.0,
        **({"dsmem_read_gbs": 5000.0} if cluster > 1 else {})})
    return b


def test_arrays_inside_one_window_cost_no_onchip_bytes(bench):
    r = bench.onchip_roofline(np.full(4096, 1024), 4, 24e-6, 5e-6, 0)
    assert r["bytes"] == 0 and r["frac_max_hbm_onchip"] == pytest.approx(5 / 24)


def test_onchip_bytes_follow_the_stage_count_above_1024(bench):
    # records n = 4096: R = 2, 1024 arrays, 8-byte elements
    r = bench.onchip_roofline(np.full(1024, 4096), 8, 100e-6, 10e-6, 0)
    assert r["bytes"] == 2 * 4096 * 8 * 2 * 1024
    assert r["t_us"] == pytest.approx(r["bytes"] / 20000e9 * 1e6)
    assert r["frac_max_hbm_onchip"] == pytest.approx(max(10e-6, r["t_us"] * 1e-6) / 100e-6)


def test_cluster_counts_dsmem_reads_per_cross_cta_layer(bench):
    # 256 arrays of W = 65536 records over 8-CTA clusters: 6 cross-CTA layers
    r = bench.onchip_roofline(np.full(256, 65536), 8, 1.5e-3, 41e-6, 0, lc=3, arrays=256)
    assert r["bytes"] == 256 * 2 * 65536 * 8 * 6
    assert r["dsmem"]["cross_cta_layers"] == 6
    assert r["dsmem"]["bytes"] == 256 * 6 * 65536 * 8
    assert r["dsmem"]["t_us"] == pytest.approx(r["dsmem"]["bytes"] / 5000e9 * 1e6)


def test_mixed_widths_sum_per_array(bench):
    r = bench.onchip_roofline(np.array([32, 1024, 2048, 8192]), 8, 1e-3, 1e-5, 0)
    assert r["bytes"] == 2 * 8 * (2048 * 1 + 8192 * 3)


def test_layer_counts_of_the_headline_tile(bench):
    # K = 16 registers, 32 lanes, 2 warps: 55 layers of a 1024-key network
    assert bench.layer_counts(4, 5, 1) == [34, 20, 1, 0]
    assert sum(bench.layer_counts(4, 5, 4, 3)) == 16 * 17 // 2
