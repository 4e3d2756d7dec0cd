"""Precision forms across signal rank and noise level (the precision
configuration: rank in {2, 4, 8} x sigma in {0.01, 0.05, 0.2}), each output
against the float64 oracle (step 0 on the float64 volume), on the
48x48x24x48 / 11^3 / stride 3 volume (1176 patches).

Bars: accurate and tensor within 2e-7 relative L2 of float64 (the north
star's FP64 bar); plain within 2e-7 of the float32 step-0 loop (its own bar)
and within 4e-7 of float64 (step 0 itself sits 2-3e-7 from float64); ranks
equal to step 0's in every form. Each case prints its measured errors.
"""

import json

import numpy as np
import pytest

from lowrank_gpu_fastest_b200 import api, rel_l2
from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank
from oracle import mppca as orc

pytestmark = pytest.mark.gpu

SHAPE, PATCH, STRIDE = (48, 48, 24, 48), (11, 11, 11), 3


@pytest.mark.parametrize("rank", [2, 4, 8])
@pytest.mark.parametrize("sigma", [0.01, 0.05, 0.2])
def test_precision_forms_vs_fp64(cuda_ok, rank, sigma):
    import torch

    vol = make_phantom_lowrank(SHAPE, rank=rank, sigma=sigma, seed=3)[0]
    ref64, _ = orc.denoise_fp64_parallel(vol, PATCH, STRIDE)
    ref32, ranks32 = orc.denoise(vol, PATCH, STRIDE)
    d = torch.from_numpy(vol).cuda()
    errs = {}
    for form in ("plain", "accurate", "tensor"):
        out, ranks = api.denoise(d, PATCH, STRIDE, form=form, return_ranks=True)
        torch.cuda.synchronize()
        out, ranks = out.cpu().numpy(), ranks.cpu().numpy()
        np.testing.assert_array_equal(ranks, ranks32)
        errs[form] = rel_l2(out.astype(np.float64), ref64)
        if form == "plain":
            errs["plain_vs_step0"] = rel_l2(out, ref32)
    errs["step0_vs_fp64"] = rel_l2(ref32.astype(np.float64), ref64)
    print("precision", json.dumps(dict(rank=rank, sigma=sigma, **{k: float(v) for k, v in errs.items()})))
    assert errs["accurate"] <= 2e-7 and errs["tensor"] <= 2e-7
    assert errs["plain_vs_step0"] <= 2e-7 and errs["plain"] <= 4e-7


HEADLINE = (96, 96, 48, 48)
# 9^3 boxes where the step-0 loop runs over exactly the patches touching them
# (bit for bit the full float32 loop there): plain vs step 0 on the headline
BOXES = [((40, 17, 20), (49, 26, 29)), ((0, 0, 0), (9, 9, 9)), ((87, 60, 39), (96, 69, 48))]


@pytest.mark.parametrize("rank", [2, 4, 8])
@pytest.mark.parametrize("sigma", [0.01, 0.05, 0.2])
def test_precision_forms_vs_fp64_headline(cuda_ok, rank, sigma):
    """The same grid on the 96x96x48x48 / 11^3 / stride 3 headline volume
    (12600 patches): every form against the float64 oracle over the whole
    volume (a spawn pool), ranks against step 0's (all 12600, pool), plain
    against the float32 step-0 loop on three 9^3 boxes."""
    import torch

    vol = make_phantom_lowrank(HEADLINE, rank=rank, sigma=sigma, seed=3)[0]
    ref64, ranks64 = orc.denoise_fp64_parallel(vol, PATCH, STRIDE)
    ranks32 = orc.ranks_parallel(vol, PATCH, STRIDE)
    d = torch.from_numpy(vol).cuda()
    errs = {}
    outs = {}
    for form in ("plain", "accurate", "tensor"):
        out, ranks = api.denoise(d, PATCH, STRIDE, form=form, return_ranks=True)
        torch.cuda.synchronize()
        out, ranks = out.cpu().numpy(), ranks.cpu().numpy()
        # every rank equals step 0's, except where step 0's float32 decision differs
        # from the float64 run's (a margin below step 0's own rounding): there the
        # library's float64 near-tie pass takes the float64 decision
        step0_off = ranks32 != ranks64
        ok = (ranks == ranks32) | (step0_off & (ranks == ranks64))
        assert ok.all(), f"{form}: {(~ok).sum()} ranks differ from step 0 and from the float64 run"
        errs[f"{form}_ranks_at_step0_near_ties"] = int((ranks != ranks32).sum())
        errs[form] = rel_l2(out.astype(np.float64), ref64)
        outs[form] = out
    num = den = 0.0
    for lo, hi in BOXES:
        box, _, _ = orc.denoise_region(vol, PATCH, STRIDE, lo, hi)
        sl = tuple(slice(a, b) for a, b in zip(lo, hi))
        num += float(np.sum((outs["plain"][sl].astype(np.float64) - box) ** 2))
        den += float(np.sum(box.astype(np.float64) ** 2))
    errs["plain_vs_step0_boxes"] = (num / den) ** 0.5
    print("precision_headline", json.dumps(dict(rank=rank, sigma=sigma, **{k: float(v) for k, v in errs.items()})))
    assert errs["accurate"] <= 2e-7 and errs["tensor"] <= 2e-7
    assert errs["plain_vs_step0_boxes"] <= 2e-7 and errs["plain"] <= 4e-7
