"""bench.py's host-side pieces without a GPU: the kernel named for each
phase, the roofline arithmetic against the recorded peaks and DRAM traffic,
and the argument surface the benchmark contract uses."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_phase_kernel_names():
    assert bench.phase_kernel("gram", 48, "plain") == "gram_z_kernel"
    assert bench.phase_kernel("gram", 48, "tensor") == "gram_tc_kernel"
    assert bench.phase_kernel("gram", 96, "tensor") == "gram_z_kernel"
    assert bench.phase_kernel("gram", 48, "tensor_bf16") == "gram_tc_kernel"
    assert bench.phase_kernel("recon", 48, "tensor") == "recon_tc_kernel"
    assert bench.phase_kernel("recon", 96, "tensor") == "recon_warp_kernel"
    assert bench.phase_kernel("eigh_mp", 64, "plain") == "eigh_reg_kernel"
    assert bench.phase_kernel("eigh_mp", 96, "plain") == "eigh_cta_kernel"
    assert bench.phase_kernel("recon", 48, "plain") == "recon_warp_kernel"
    assert bench.phase_kernel("recon", 96, "accurate") == "recon_warp_kernel"
    assert bench.phase_kernel("recon", 46, "plain") == "recon_kernel_t24s2"
    assert bench.phase_kernel("recon", 80, "plain") == "recon_kernel"


def test_roofline_arithmetic():
    shape, patch, P = (96, 96, 48, 48), (11, 11, 11), 12600
    peaks = bench.measured_peaks()
    # eigensolver dominant: bytes = 2 T^2 x 4 per patch
    r = bench.roofline({"center": 0.05, "gram": 0.8, "eigh_mp": 1.4, "recon": 1.3}, shape, patch, P, "plain")
    assert r["kernel"] == "eigh_reg_kernel" and r["bound"] == "hbm"
    assert r["achieved"] == pytest.approx(2 * 48 * 48 * 4 * P / 1.4e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / peaks["hbm_gbs"])
    # reconstruction dominant: flops = 2 N T^2 per patch
    r = bench.roofline({"center": 0.05, "gram": 0.8, "eigh_mp": 1.0, "recon": 1.3}, shape, patch, P, "plain")
    assert r["bound"] == "tensor" and r["unit"] == "TFLOP/s"
    assert r["achieved"] == pytest.approx(2 * 1331 * 48 * 48 * P / 1.3e-3 / 1e12)


def test_contract_arguments(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2", "--steps", "3", "--warmup", "4"])
    a = bench.parse()
    assert (a.gpus, a.steps, a.warmup, a.impl, a.parallel) == (2, 3, 4, "ours", "shard")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    assert bench.parse().impl == "reference"


def test_golden_accuracy_of_the_step0_sample():
    """The accuracy block of the bench line: the step-0 sample itself has zero
    error against step 0, its own distance from float64, and no rank
    mismatches with step 0."""
    import numpy as np

    d = np.load(os.path.join(ROOT, "tests", "golden", "config1_lowrank.npz"))
    out = np.zeros(tuple(int(s) for s in d["shape"]), dtype=np.float32)
    out.reshape(-1)[d["sample_idx"]] = d["out_sample"]
    a = bench.golden_accuracy(out, d["ranks"], "config1_lowrank.npz")
    assert a["rel_err_vs_step0"] == 0.0
    assert a["rel_err_vs_fp64"] == pytest.approx(a["step0_vs_fp64"])
    assert 1e-8 < a["rel_err_vs_fp64"] < 1e-6
    assert a["rank_mismatch_vs_step0"] == 0 and a["n_patches"] == 1176


def test_executed_fp32_counts():
    """Executed FP32 work: the column Gram's plane Grams (upper-triangle 4x4
    blocks, one per plane per (x, y) column) and the reconstruction's 4 p T
    flops per covered voxel-patch pair."""
    import numpy as np

    ranks = np.full(12600, 4, dtype=np.int32)
    ph = {"center": 0.05, "gram": 0.68, "eigh_mp": 1.1, "recon": 1.2}
    r = bench.executed_fp32(ph, (96, 96, 48, 48), (11, 11, 11), 3, ranks, 64.0, "plain")
    assert r["executed_gflop_gram"] == pytest.approx(2 * 30 * 30 * 48 * 121 * 16 * 78 / 1e9)
    assert r["executed_gflop_recon"] == pytest.approx(4 * 48 * 1331 * 4 * 12600 / 1e9)
    assert r["recon_frac_of_sgemm"] == pytest.approx(r["executed_tflops_recon"] / 64.0)


def test_rank_mismatch_counts():
    from lowrank_gpu_fastest_b200 import report

    r = report.count_mismatches([1, 2, 3, 4], [1, 2, 3, 5], [1, 0, 3, 5])
    assert r == dict(n=4, vs_step0=1, vs_fp64=2, step0_vs_fp64=1)
    assert "vs fp64" in report.rank_table([dict(case="c", shape=(4, 4, 4, 8), patch=(3, 3, 3), stride=1,
                                                form="plain", **r)])
