"""Slab sharding through the C ABI on one GPU: every slab's plan runs on the
same device, one after another, and the halo hand-off is a device copy (the
multi-rank NCCL exchange of the same buffers is covered on CPU with gloo).
The owned planes of the slabs, put together, must equal the unsharded output
bit for bit (same patches, same per-voxel x-major accumulation order), and
the slab ranks the unsharded ranks.
"""

import numpy as np
import pytest
import torch

from conftest import golden_input, load_golden
from lowrank_gpu_fastest_b200 import api
from lowrank_gpu_fastest_b200._native import SLAB_HALO_IN, SLAB_HALO_OUT, SLAB_INTERIOR
from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank
from lowrank_gpu_fastest_b200.shard import CudaSlab, slab_partition

pytestmark = pytest.mark.gpu


def sharded_on_one_gpu(vol, patch, stride, form, n):
    shape = vol.shape
    parts = slab_partition(shape, patch, stride, n)
    slabs = [CudaSlab(shape, r, n, patch, stride, form) for r in range(n)]
    for r, s in enumerate(slabs):
        s.load(torch.from_numpy(np.ascontiguousarray(vol[parts[r]["x0"]:parts[r]["x1"]])))
        s.prepare()
        s.recon(SLAB_HALO_OUT)
    for r in range(1, n):
        assert slabs[r].halo_in.shape == slabs[r - 1].halo_out.shape
        slabs[r].halo_in.copy_(slabs[r - 1].halo_out)
    for s in slabs:
        s.recon(SLAB_INTERIOR)
        s.recon(SLAB_HALO_IN)
    torch.cuda.synchronize()
    for s in slabs:
        assert s.status() == 0
    out = torch.cat([s.owned() for s in slabs]).cpu().numpy()
    ranks = torch.cat([s.ranks for s in slabs]).cpu().numpy()
    return out, ranks


def unsharded(vol, patch, stride, form):
    d = torch.from_numpy(vol).cuda()
    out, ranks = api.denoise(d, patch, stride, form=form, return_ranks=True)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ranks.cpu().numpy()


@pytest.mark.parametrize("form", ["plain", "accurate", "tensor", "tensor_bf16"])
@pytest.mark.parametrize("n", [2, 3])
def test_slabs_equal_unsharded(cuda_ok, form, n):
    vol = make_phantom_lowrank((40, 20, 18, 32), seed=5)[0]
    patch, stride = (5, 5, 5), 2
    ref, ref_ranks = unsharded(vol, patch, stride, form)
    out, ranks = sharded_on_one_gpu(vol, patch, stride, form, n)
    np.testing.assert_array_equal(ranks, ref_ranks)
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("n", [2, 4])
def test_slabs_config1_vs_step0(cuda_ok, n):
    g = load_golden("config1_lowrank")
    vol = golden_input(g)
    patch, stride = tuple(int(v) for v in g["patch"]), int(g["stride"])
    ref, _ = unsharded(vol, patch, stride, "plain")
    out, ranks = sharded_on_one_gpu(vol, patch, stride, "plain", n)
    np.testing.assert_array_equal(ranks, g["ranks"])
    np.testing.assert_array_equal(out, ref)


def test_slabs_uncovered_planes(cuda_ok):
    # stride > patch side along x: planes between slabs that no patch touches
    vol = make_phantom_lowrank((26, 10, 10, 16), seed=2)[0]
    patch, stride = (3, 5, 5), 4
    ref, ref_ranks = unsharded(vol, patch, stride, "plain")
    out, ranks = sharded_on_one_gpu(vol, patch, stride, "plain", 3)
    np.testing.assert_array_equal(ranks, ref_ranks)
    np.testing.assert_array_equal(out, ref)
