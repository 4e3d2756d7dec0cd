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
    assert bench.phase_kernel("eigh_mp", 64, "plain") == "eigh_reg_kernel"
    assert bench.phase_kernel("eigh_mp", 96, "plain") == "eigh_cta_kernel"
    assert bench.phase_kernel("recon", 48, "plain") == "recon_kernel_t24s2"
    assert bench.phase_kernel("recon", 48, "accurate") == "recon_kernel"
    assert bench.phase_kernel("recon", 64, "plain") == "recon_kernel"


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
