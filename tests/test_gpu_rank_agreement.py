"""MP-rank agreement of every form with step 0 run in float32 and in float64,
on every golden case (the ladder counts the same for its FP32 routes against
an FP64 SVD in micro/rank_agreement.py:46-102). The library's ranks must
equal step 0's float32 ranks on every case and form; their disagreement
with the float64 run is then step 0's own, and the table states it."""

import os

import pytest

from conftest import GOLDEN, LARGE_CASES, SMALL_CASES
from lowrank_gpu_fastest_b200 import report

pytestmark = pytest.mark.gpu


def test_rank_agreement_all_cases_and_forms(cuda_ok):
    paths = [os.path.join(GOLDEN, f"{n}.npz") for n in SMALL_CASES + LARGE_CASES]
    rows = report.rank_agreement(paths)
    print("\n" + report.rank_table(rows))
    assert len(rows) == 4 * len(paths)
    for r in rows:
        assert r["vs_step0"] == 0, r
        assert r["vs_fp64"] == r["step0_vs_fp64"], r


def test_harness_subcommand_times_host_calls(cuda_ok, capsys, tmp_path):
    """The ladder-protocol timing (common.py:103-172) of the library's
    host->host denoise: best-of timing, patch count, RMSE against the clean
    phantom below the noisy input's."""
    import json

    out = tmp_path / "h.json"
    assert report.main(["harness", "--shape", "48,48,24,48", "--repeats", "2", "--json", str(out)]) == 0
    res = json.loads(out.read_text())
    assert res["n_patches"] == 1176 and res["seconds"] > 0
    assert res["rmse_denoised"] < res["rmse_noisy"]
