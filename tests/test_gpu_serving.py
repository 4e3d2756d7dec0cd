"""Serving loop: continuous batching, HBM admission, same result alone and in the mix."""

import numpy as np
import pytest
import torch

from lowrank_gpu_fastest_b200 import api, make_phantom_lowrank
from lowrank_gpu_fastest_b200.serve import Server, draw_request_shapes, poisson_arrivals

pytestmark = pytest.mark.gpu

SHAPES = [((20, 18, 16, 32), (5, 5, 5), 2), ((17, 15, 13, 48), (11, 11, 11), 3),
          ((14, 13, 12, 64), (7, 7, 7), 2), ((12, 11, 10, 96), (5, 5, 5), 3),
          ((24, 20, 18, 48), (7, 7, 7), 1)]


def _alone(vol, patch, stride):
    out, ranks = api.denoise(torch.from_numpy(vol).cuda(), patch, stride, return_ranks=True)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ranks.cpu().numpy()


def test_results_identical_alone_and_in_mix(cuda_ok):
    reqs = [(make_phantom_lowrank(s, seed=i)[0], p, st) for i, (s, p, st) in enumerate(SHAPES * 3)]
    with Server(n_slots=4) as srv:
        futs = [srv.submit(v, p, st) for v, p, st in reqs]
        res = [f.result(timeout=120) for f in futs]
        stats = srv.stats()
    assert stats["n"] == len(reqs) and stats["p99_ms"] >= stats["p50_ms"] > 0
    for (v, p, st), (out, ranks) in zip(reqs, res):
        a, ar = _alone(v, p, st)
        np.testing.assert_array_equal(out, a)
        np.testing.assert_array_equal(ranks, ar)


def test_admission_waits_for_memory(cuda_ok):
    """A device budget that fits one request at a time still completes all,
    in order, with at most one in flight."""
    v, p, st = make_phantom_lowrank((20, 18, 16, 32), seed=1)[0], (5, 5, 5), 2
    plan = api.get_plan(v.shape, p, st)
    need = 2 * v.nbytes + 4 * plan.n_patches + plan.workspace_bytes + (1 << 20)
    with Server(n_slots=4, hbm_budget_bytes=int(need * 1.5)) as srv:
        futs = [srv.submit(v, p, st) for _ in range(5)]
        res = [f.result(timeout=120) for f in futs]
        stats = srv.stats()
    a, _ = _alone(v, p, st)
    for out, _ in res:
        np.testing.assert_array_equal(out, a)
    assert stats["n"] == 5


def test_invalid_request_fails_only_itself(cuda_ok):
    with Server(n_slots=2) as srv:
        bad = srv.submit(np.zeros((4, 4, 4, 8), np.float32), (5, 5, 5), 2)  # patch larger than volume
        good = srv.submit(make_phantom_lowrank((20, 18, 16, 32), seed=2)[0], (5, 5, 5), 2)
        with pytest.raises(Exception):
            bad.result(timeout=60)
        out, _ = good.result(timeout=60)
    assert np.isfinite(out).all()


