"""Host-side arithmetic of bench.py (no GPU): the edge counts of the
configurations and the dominant kernel's figure against its own bound."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_edge_counts_of_the_configurations():
    # rows x layers x 32 non-zeros per output x outputs
    assert bench.edges(bench.config_nets("c1")[0]) == 60000 * 120 * 32 * 1024
    assert bench.edges(bench.config_nets("c2")[0]) == pytest.approx(9.437e11, rel=1e-3)
    assert bench.edges(bench.config_nets("c4")[0]) == pytest.approx(1.510e13, rel=1e-3)


def test_own_bound_of_the_row_tile_kernel():
    # 7.86e9 FMAs in 0.5 ms on 148 SMs at 1965 MHz = 27.0 FMA/clk/SM of 64
    fma = 60000 * 4096 * 32.0
    ob = bench.own_bound(["k_layer_cc<__half, 256, 16>"], "fp16", fma, 0.5, 148, 1965.0)
    assert ob["unit"] == "FMA/clk/SM" and ob["peak"] == 64.0
    assert ob["achieved"] == pytest.approx(fma / 0.5e-3 / (148 * 1965e6))
    assert ob["frac"] == pytest.approx(ob["achieved"] / 64.0)
    # FP32 rows: 32 FMAs per wavefront; the feature-split kernel counts like 16-bit rows
    assert bench.own_bound(["k_layer_cc<float, 256, 16>"], "fp32", fma, 0.5, 148, 1965.0)["peak"] == 32.0
    assert bench.own_bound(["k_layer_cs<__half>"], "fp16", fma, 0.5, 148, 1965.0)["peak"] == 64.0


def test_own_bound_only_for_cuda_core_row_tiles():
    assert bench.own_bound(["k_layer_tc<__half>"], "fp16", 1e9, 0.5, 148, 1965.0) is None
    assert bench.own_bound(["k_layer_cc<__half, 256, 16>", "k_layer_plain<float>"], "fp16", 1e9, 0.5, 148,
                           1965.0) is None
    assert bench.own_bound([], "fp16", 1e9, 0.5, 148, 1965.0) is None
    assert bench.own_bound(["k_layer_cc<__half, 256, 16>"], "fp16", 1e9, 0.0, 148, 1965.0) is None
    assert bench.own_bound(["k_layer_cc<__half, 256, 16>"], "fp16", 1e9, 0.5, 148, 0.0) is None


def test_reference_build_runs_in_a_child_process():
    """The reference's host code exits its process on a CUDA error (no device
    here); the arm still gets a result dict back from the child process."""
    r = bench.reference_cuda_build_isolated([(1024, 2, 256)], "xor", (0.08, 0.25), timeout_s=120.0)
    assert isinstance(r, dict) and ("unavailable" in r or "kernel_exec_ms" in r)
    # sizes the arm does not run the reference on come back from the child too
    r = bench.reference_cuda_build_isolated([(16384, 2, 256)], "xor", (0.08, 0.25), timeout_s=120.0)
    assert r == {"unavailable": "measured for single networks of at most 4096 neurons"}
