"""Slab sharding on CPU: the partition (C ABI, host-only) and the multi-rank
orchestration (gloo, world_size 2 and 3) with a slab engine built on the
oracle's step-0 loop, whose all-gathered output must equal the unsharded
oracle bit for bit.

The oracle engine restates the slab semantics the CUDA engine implements:
each slab's patches are accumulated in x-major order in float32 (the ladder's
``out[sl] += w * xd``, step0_numpy_loop.py:32-38), the shared bottom planes
starting from the sums handed up by the slab below.
"""

import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lowrank_gpu_fastest_b200 import _native, build  # noqa: E402
from lowrank_gpu_fastest_b200._native import SLAB_HALO_IN, SLAB_HALO_OUT, SLAB_INTERIOR  # noqa: E402
from oracle import mppca  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def lib():
    build.build()
    return _native.load()


class OracleSlab:
    """Slab engine on the oracle (float32 step-0 arithmetic)."""

    def __init__(self, shape, slab, n_slabs, patch, stride):
        from lowrank_gpu_fastest_b200.shard import slab_partition

        parts = slab_partition(shape, patch, stride, n_slabs)
        me = parts[slab]
        self.patch, self.shape = patch, shape
        self.x0, self.x1 = me["x0"], me["x1"]
        self.nx = self.x1 - self.x0
        self.own_hi = me["own_hi"] - self.x0
        self.hin = (parts[slab - 1]["x1"] - self.x0) if slab > 0 else 0
        cx = mppca.axis_corners(shape[0], patch[0], stride)[me["ci_lo"]:me["ci_hi"]]
        cy = mppca.axis_corners(shape[1], patch[1], stride)
        cz = mppca.axis_corners(shape[2], patch[2], stride)
        self.corners = [(i - self.x0, j, k) for i in cx for j in cy for k in cz]
        ny, nz, nt = shape[1:]
        self.halo_in = torch.zeros((self.hin, ny, nz, nt + 1), dtype=torch.float64)
        self.halo_out = torch.zeros((self.nx - self.own_hi, ny, nz, nt + 1), dtype=torch.float64)
        self.out = np.zeros((self.nx, ny, nz, nt), dtype=np.float32)

    def load(self, planes):
        self.vol = np.asarray(planes, dtype=np.float32)

    def prepare(self):
        px, py, pz = self.patch
        self.pd = []
        rk = []
        for i, j, k in self.corners:
            x = self.vol[i:i + px, j:j + py, k:k + pz].reshape(-1, self.vol.shape[-1])
            xd, p = mppca.mppca_patch(x)
            rk.append(p)
            self.pd.append(((i, j, k), 1.0 / (2.0 + p), xd.reshape(px, py, pz, -1)))
        self.ranks = torch.tensor(rk, dtype=torch.int32)

    def _sums(self, a, b, init=None):
        ny, nz, nt = self.shape[1:]
        acc = np.zeros((b - a, ny, nz, nt), np.float32)
        ws = np.zeros((b - a, ny, nz, 1), np.float32)
        if init is not None:
            h = init.numpy()
            acc[:] = h[..., :nt].astype(np.float32)
            ws[:] = h[..., nt:].astype(np.float32)
        px, py, pz = self.patch
        for (i, j, k), w, xd in self.pd:
            lo, hi = max(i, a), min(i + px, b)
            if lo >= hi:
                continue
            acc[lo - a:hi - a, j:j + py, k:k + pz] += w * xd[lo - i:hi - i]
            ws[lo - a:hi - a, j:j + py, k:k + pz] += w
        return acc, ws

    def recon(self, part):
        if part == SLAB_HALO_OUT:
            a, b = self.own_hi, self.nx
            if a < b:
                acc, ws = self._sums(a, b)
                self.halo_out.copy_(torch.from_numpy(np.concatenate([acc, ws], -1).astype(np.float64)))
            return
        a, b = (self.hin, self.own_hi) if part == SLAB_INTERIOR else (0, self.hin)
        if a < b:
            acc, ws = self._sums(a, b, self.halo_in if part == SLAB_HALO_IN else None)
            self.out[a:b] = acc / np.maximum(ws, 1e-12)

    def owned(self):
        return torch.from_numpy(self.out[: self.own_hi])


def _worker(rank, world, port, vol, patch, stride, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from lowrank_gpu_fastest_b200.shard import denoise_sharded

        eng = OracleSlab(vol.shape, rank, world, patch, stride)
        out, ranks = denoise_sharded(vol, patch, stride, engine=eng)
        q.put((rank, out.numpy(), ranks.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,shape,patch,stride", [
    (2, (17, 9, 8, 12), (5, 5, 5), 2),
    (3, (23, 8, 7, 10), (5, 5, 5), 2),
    (2, (16, 8, 8, 12), (3, 5, 5), 4),  # stride > patch along x: uncovered planes
])
def test_sharded_equals_unsharded_oracle(world, shape, patch, stride):
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    vol = make_phantom_lowrank(shape, seed=3)[0]
    ref, ref_ranks = mppca.denoise(vol, patch, stride)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, vol, patch, stride, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    for _, out, _ in res:
        np.testing.assert_array_equal(out, ref)
    np.testing.assert_array_equal(np.concatenate([r[2] for r in res]), ref_ranks)


def test_partition_covers_and_respects_neighbours():
    from lowrank_gpu_fastest_b200.shard import slab_partition

    shape, patch, stride = (96 * 8, 96, 48, 48), (11, 11, 11), 3
    for n in (1, 2, 3, 8):
        parts = slab_partition(shape, patch, stride, n)
        ncx = len(mppca.axis_corners(shape[0], patch[0], stride))
        assert parts[0]["ci_lo"] == 0 and parts[-1]["ci_hi"] == ncx
        assert parts[0]["own_lo"] == 0 and parts[-1]["own_hi"] == shape[0]
        for a, b in zip(parts, parts[1:]):
            assert a["ci_hi"] == b["ci_lo"] and a["own_hi"] == b["own_lo"]
            assert a["x1"] >= b["x0"]  # the halo planes
        for a, c in zip(parts, parts[2:]):
            assert a["x1"] <= c["x0"]  # no plane touched by three slabs
    # the headline volume cut in 8: about 4 x-corners per slab
    parts = slab_partition((96, 96, 48, 48), patch, stride, 8)
    assert all(p["ci_hi"] - p["ci_lo"] in (3, 4) for p in parts)


def test_partition_rejects_too_many_slabs():
    with pytest.raises(_native.LrdError) as e:
        _native.slab_partition((30, 20, 20, 12), (11, 11, 11), 3, 8)
    assert e.value.code == _native.LRD_ERR_UNSUPPORTED
    with pytest.raises(_native.LrdError) as e:
        _native.slab_partition((30, 20, 20, 12), (11, 11, 11), 3, 100)
    assert e.value.code == _native.LRD_ERR_INVALID
