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


def test_report_kernel_name_and_launch_table(tmp_path):
    from lowrank_gpu_fastest_b200 import report

    assert report.kernel_name("void lrd::eigh_reg_kernel<48>(const float *, float *, int)") == "eigh_reg_kernel"
    assert report.kernel_name("lrd::(anonymous namespace)::k<lrd::Q<2>, true>(int)") == "k"
    # an ncu launch-list CSV: preamble lines, a header, one row per launch and metric
    rows = [
        "==PROF== Connected to process 1",
        '"ID","Kernel Name","Metric Name","Metric Unit","Metric Value"',
        '"0","void lrd::gram_z_kernel<2>(CUtensorMap, float *)","gpu__time_duration.sum","usecond","600.0"',
        '"1","void lrd::eigh_reg_kernel<48>(const float *)","gpu__time_duration.sum","usecond","1,000.0"',
        '"2","void lrd::eigh_reg_kernel<48>(const float *)","gpu__time_duration.sum","msecond","1.0"',
        '"3","void at::native::elementwise_kernel<128>(int)","gpu__time_duration.sum","nsecond","400000"',
        '"4","void lrd::gram_z_kernel<2>(CUtensorMap, float *)","dram__bytes_read.sum","byte","5"',
    ]
    f = tmp_path / "launches.csv"
    f.write_text("\n".join(rows) + "\n")
    t = report.ncu_launch_table(str(f))
    assert [r["kernel"] for r in t] == ["eigh_reg_kernel", "gram_z_kernel", "elementwise_kernel"]
    assert t[0]["launches"] == 2 and t[0]["total_ms"] == pytest.approx(2.0)
    assert t[1]["launches"] == 1 and t[1]["mean_us"] == pytest.approx(600.0)
    assert sum(r["share"] for r in t) == pytest.approx(1.0)
    assert t[0]["share"] == pytest.approx(2.0 / 3.0)
    t2 = report.ncu_launch_table(str(f), skip="elementwise")
    assert [r["kernel"] for r in t2] == ["eigh_reg_kernel", "gram_z_kernel"]
    assert t2[0]["share"] == pytest.approx(2.0 / 2.6)


def test_report_summary_table():
    from lowrank_gpu_fastest_b200 import report

    line = dict(metric="patches/s", value=4.5e6, unit="patches/s", n_gpus=1, ms_per_step=2.8,
                config=dict(workload="96x96x48x48", form="plain"), e2e=dict(value=3.4e6),
                roofline=dict(kernel="recon_warp_kernel", frac=0.25), clocks=dict(sm_mhz=1965))
    ref = dict(impl="reference", value=7000.0, unit="patches/s", n_gpus=1, ms_per_step=1800.0,
               config=dict(workload="96x96x48x48"))
    md = report.summary([line, ref]).splitlines()
    assert md[0].startswith("| impl | workload | form |")
    assert len(md) == 4
    assert "4,500,000 patches/s" in md[2] and "recon_warp_kernel 0.250" in md[2] and "1965" in md[2]
    assert md[3].startswith("| reference | 96x96x48x48 |")
