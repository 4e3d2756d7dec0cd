"""Slab sharding of one volume over GPUs, one process per GPU.

The x-corner list of the volume is cut into ``world`` contiguous slabs
(``lrd_slab_partition``); rank r denoises the patches of slab r on its own GPU
from the x-planes those patches touch, which it copies in from the host (no
input traffic between GPUs). The one exchange is a neighbour halo: the top
planes of slab r are touched by slab r+1's patches too, so rank r sends its
unnormalised sums for them (sum of w * xd per frame, then sum of w, float64)
to rank r+1, which continues them with its own patches. The patches of a
voxel are therefore added in the single-GPU x-major order of the ladder's loop
(step0_numpy_loop.py:32-38) and every rank's owned planes equal the 1-GPU
output bit for bit.

Per rank, on the compute stream:

1. ``prepare``: centre, Gram, eigensolve and MP rank of the slab's patches;
2. ``recon(HALO_OUT)``: the planes handed up; the send starts as soon as they
   are done (``batch_isend_irecv`` on the process group's stream);
3. ``recon(INTERIOR)``: the planes only this slab touches, overlapping the
   exchange;
4. wait for the halo from below, ``recon(HALO_IN)``: the shared bottom planes.

The slab work is behind a small engine interface (``load``, ``prepare``,
``recon``, ``owned``), implemented here by :class:`CudaSlab` on the C ABI; the
orchestration (:func:`run_slab`) does not depend on it.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import _native
from ._native import SLAB_HALO_IN, SLAB_HALO_OUT, SLAB_INTERIOR


def slab_partition(shape, patch=(11, 11, 11), stride=3, n_slabs=1):
    """Per slab ``dict(ci_lo, ci_hi, x0, x1, own_lo, own_hi)`` in global planes:
    the slab reads ``[x0, x1)`` and owns output planes ``[own_lo, own_hi)``."""
    b = _native.slab_partition(shape, patch, stride, n_slabs)
    out = []
    for r, (ci_lo, ci_hi, x0, x1) in enumerate(b):
        own_hi = b[r + 1][2] if r + 1 < len(b) else int(shape[0])
        out.append(dict(ci_lo=ci_lo, ci_hi=ci_hi, x0=x0, x1=x1, own_lo=x0, own_hi=own_hi))
    return out


class CudaSlab:
    """One GPU's slab: its plan, device buffers and halos."""

    def __init__(self, shape, slab, n_slabs, patch=(11, 11, 11), stride=3, form="plain", device=None,
                 brick=None, split=0):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        with torch.cuda.device(self.device):
            self.plan = _native.SlabPlan(shape, slab, n_slabs, patch, stride, form, brick, split)
        p = self.plan
        ny, nz, nt = (int(v) for v in shape[1:])
        dev = self.device
        self.vol = torch.empty((p.nx, ny, nz, nt), dtype=torch.float32, device=dev)
        self.out = torch.empty_like(self.vol)
        self.ranks = torch.empty(p.n_patches, dtype=torch.int32, device=dev)
        self.ws = torch.empty(p.workspace_bytes, dtype=torch.uint8, device=dev)
        plane = ny * nz * (nt + 1)
        self.halo_in = torch.empty((p.hin, ny, nz, nt + 1), dtype=torch.float64, device=dev)
        self.halo_out = torch.empty((p.nx - p.own_hi, ny, nz, nt + 1), dtype=torch.float64, device=dev)
        self.halo_plane_bytes = 8 * plane
        self.x0, self.x1 = p.x0, p.x0 + p.nx
        self.own = (p.x0, p.x0 + p.own_hi)
        self.n_patches = p.n_patches

    def _sid(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def load(self, planes):
        """Copy the slab's input planes ``[x0, x1)`` (host or device tensor)."""
        src = torch.as_tensor(planes)
        if tuple(src.shape) != tuple(self.vol.shape):
            raise ValueError(f"slab input must have shape {tuple(self.vol.shape)}, got {tuple(src.shape)}")
        self.vol.copy_(src, non_blocking=True)

    def prepare(self):
        self.plan.prepare(self.vol.data_ptr(), self.ranks.data_ptr(), self.ws.data_ptr(), self._sid())

    def recon(self, part):
        self.plan.recon(part, self.out.data_ptr(), self.ws.data_ptr(),
                        self.halo_in.data_ptr() if self.halo_in.numel() else None,
                        self.halo_out.data_ptr() if self.halo_out.numel() else None, self._sid())

    def owned(self):
        """Output planes this slab owns (a view of the local output)."""
        return self.out[: self.plan.own_hi]

    def status(self):
        return self.plan.status(self.ws.data_ptr(), self._sid())


def _peer(group, r):
    return r if group is None else dist.get_global_rank(group, r)


def run_slab(engine, rank, world, group=None):
    """Steps 1-4 above for this rank's ``engine`` (input already loaded)."""
    engine.prepare()
    engine.recon(SLAB_HALO_OUT)
    ops = []
    if rank + 1 < world and engine.halo_out.numel():
        ops.append(dist.P2POp(dist.isend, engine.halo_out, _peer(group, rank + 1), group))
    if rank > 0 and engine.halo_in.numel():
        ops.append(dist.P2POp(dist.irecv, engine.halo_in, _peer(group, rank - 1), group))
    reqs = dist.batch_isend_irecv(ops) if ops else []
    engine.recon(SLAB_INTERIOR)
    for q in reqs:
        q.wait()
    engine.recon(SLAB_HALO_IN)


def gather_owned(owned, parts, world, group=None):
    """All-gather the ranks' owned planes into the full output on every rank."""
    sizes = [p["own_hi"] - p["own_lo"] for p in parts]
    mx = max(sizes)
    buf = torch.zeros((mx,) + tuple(owned.shape[1:]), dtype=owned.dtype, device=owned.device)
    buf[: owned.shape[0]].copy_(owned)
    bufs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    return torch.cat([b[:s] for b, s in zip(bufs, sizes)], dim=0)


def denoise_sharded(vol, patch=(11, 11, 11), stride=3, form="plain", group=None, gather=True, engine=None):
    """Denoise ``vol`` (the global (X, Y, Z, T) volume, host array or tensor,
    read only in this rank's planes) across the ranks of ``group``.

    Returns ``(out, ranks)``: with ``gather`` the full output volume on every
    rank (on this rank's device), else this rank's owned planes; ``ranks`` are
    this slab's per-patch MP ranks (corner indices ``[ci_lo, ci_hi)`` of the
    x-axis, x-major like the ladder's corner list)."""
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    shape = tuple(int(s) for s in vol.shape)
    parts = slab_partition(shape, patch, stride, world)
    if engine is None:
        engine = CudaSlab(shape, rank, world, patch, stride, form)
    x0, x1 = parts[rank]["x0"], parts[rank]["x1"]
    v = vol[x0:x1]
    engine.load(np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v)
    run_slab(engine, rank, world, group)
    if hasattr(engine, "status"):
        st = engine.status()
        if st:
            raise _native.LrdError(_native.LRD_ERR_TIMEOUT, f"a device wait gave up (status {st:#x})")
    owned = engine.owned()
    out = gather_owned(owned, parts, world, group) if (gather and world > 1) else owned
    return out, engine.ranks
