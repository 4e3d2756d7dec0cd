"""Batched uneven form: each volume's result equals its single-volume result."""

import numpy as np
import pytest
import torch

from lowrank_gpu_fastest_b200 import api, make_phantom_lowrank, tune
from oracle import mppca as orc

pytestmark = pytest.mark.gpu

CASES = [  # shape, patch, stride
    ((20, 18, 16, 32), (5, 5, 5), 2),
    ((17, 15, 13, 48), (11, 11, 11), 3),
    ((14, 13, 12, 64), (7, 7, 7), 2),
    ((12, 11, 10, 96), (5, 5, 5), 3),
    ((16, 16, 14, 48), (5, 5, 5), 1),
    ((13, 12, 11, 20), (5, 7, 3), 2),
]


def _vols():
    return [make_phantom_lowrank(s, seed=i, sigma=0.02 + 0.01 * i)[0] for i, (s, _, _) in enumerate(CASES)]


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_equals_single(cuda_ok, use_graph):
    vols = _vols()
    dev = [torch.from_numpy(v).cuda() for v in vols]
    outs, ranks = api.denoise_batch(dev, [c[1] for c in CASES], [c[2] for c in CASES], use_graph=use_graph,
                                    n_streams=3, return_ranks=True)
    # twice: the graph replay path on the second call
    outs2 = api.denoise_batch(dev, [c[1] for c in CASES], [c[2] for c in CASES], use_graph=use_graph, n_streams=3)
    torch.cuda.synchronize()
    for v, (shape, patch, stride), o, r, o2 in zip(dev, CASES, outs, ranks, outs2):
        single, sr = api.denoise(v, patch, stride, return_ranks=True)
        torch.cuda.synchronize()
        assert torch.equal(o, single)
        assert torch.equal(o2, single)
        assert torch.equal(r, sr)


def test_packed_launch_count(cuda_ok):
    """The batch runs in packed launches: far fewer than six per volume."""
    from lowrank_gpu_fastest_b200 import _native

    bp = _native.BatchPlan([dict(shape=s, patch=p, stride=st) for s, p, st in CASES])
    print("launches per batch", bp.launches, "for", len(CASES), "volumes")
    assert bp.launches < 6 * len(CASES)


def test_batch_matches_oracle_ranks(cuda_ok):
    vols = _vols()
    outs, ranks = api.denoise_batch(vols, [c[1] for c in CASES], [c[2] for c in CASES], return_ranks=True)
    for v, (shape, patch, stride), o, r in zip(vols, CASES, outs, ranks):
        ref, rref = orc.denoise(v, patch, stride)
        np.testing.assert_array_equal(r, rref)
        assert np.linalg.norm(o.astype(np.float64) - ref) / np.linalg.norm(ref) <= 2e-7


def test_autotuned_batch_is_bit_identical(cuda_ok, tmp_path, monkeypatch):
    monkeypatch.setenv("LRD_TUNE_CACHE", str(tmp_path / "tune.json"))
    tune.clear_memory_cache()
    vols = [torch.from_numpy(v).cuda() for v in _vols()[:3]]
    cases = CASES[:3]
    a = api.denoise_batch(vols, [c[1] for c in cases], [c[2] for c in cases], autotune=True)
    b = api.denoise_batch(vols, [c[1] for c in cases], [c[2] for c in cases], autotune=False)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    assert (tmp_path / "tune.json").exists()
