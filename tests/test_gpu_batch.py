"""Batched uneven form: each volume's result equals its single-volume result."""

import json

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


def test_autotuned_batch_matches_untuned(cuda_ok, tmp_path, monkeypatch):
    """The tuner's choices (reconstruction brick and split: bit-identical;
    Gram split and eigensolver schedule: other float32 rounding) keep every
    rank and the output within the plain form's tolerance."""
    monkeypatch.setenv("LRD_TUNE_CACHE", str(tmp_path / "tune.json"))
    tune.clear_memory_cache()
    vols = [torch.from_numpy(v).cuda() for v in _vols()[:3]]
    cases = CASES[:3]
    a, ra = api.denoise_batch(vols, [c[1] for c in cases], [c[2] for c in cases], autotune=True, return_ranks=True)
    b, rb = api.denoise_batch(vols, [c[1] for c in cases], [c[2] for c in cases], autotune=False,
                              return_ranks=True)
    for x, y, p, q in zip(a, b, ra, rb):
        assert torch.equal(p, q)
        assert float(torch.linalg.norm((x - y).double()) / torch.linalg.norm(y.double())) <= 2e-7
    assert (tmp_path / "tune.json").exists()
    entries = json.load(open(tmp_path / "tune.json"))
    for e in entries.values():
        assert e["gram_split"] in (0, 1, 2, 4) and e["eigh_block"] in (0, 1, 2)
        assert {"recon", "gram", "eigh_mp"} <= set(e["timed"])


@pytest.mark.parametrize("gram_split,eigh_block", [(1, 0), (4, 0), (0, 1), (0, 2), (4, 2)])
def test_gram_split_and_eigh_block_keep_ranks(cuda_ok, gram_split, eigh_block):
    """Every Gram split and eigensolver schedule gives step 0's ranks and an
    output within the plain form's tolerance of step 0 (golden fixture)."""
    from conftest import golden_input, load_golden
    from lowrank_gpu_fastest_b200 import rel_l2

    g = load_golden("config1_lowrank")
    vol = torch.from_numpy(golden_input(g)).cuda()
    plan = api.get_plan(tuple(vol.shape), (11, 11, 11), 3, gram_split=gram_split, eigh_block=eigh_block)
    ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device="cuda")
    out = torch.empty_like(vol)
    ranks = torch.empty(plan.n_patches, dtype=torch.int32, device="cuda")
    plan.denoise(vol.data_ptr(), out.data_ptr(), ranks.data_ptr(), ws.data_ptr(),
                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ranks.cpu().numpy(), g["ranks"])
    assert rel_l2(out.cpu().numpy().reshape(-1)[g["sample_idx"]], g["out_sample"]) <= 2e-7
