"""Drop-in ``denoise`` for the ladder's entry point.

The ladder's surface is ``denoise(vol_np) -> np.ndarray`` (step8_tuned.py:
116-146) with patch, stride and batch from module globals (common.py:28-29,
step8_tuned.py:21). Here they are arguments with the ladder's defaults, so
``functools.partial(denoise, patch=..., stride=...)`` or plain
``denoise(vol)`` can be handed to a ``common.run``-style harness.

* numpy input (or a CPU tensor): host -> host, like the ladder - the volume is
  copied to the device, denoised, and returned as a numpy array backed by
  pinned host memory (step8_tuned.py:144-146 does the same D2H into pinned).
* CUDA tensor input: device-resident; returns a CUDA tensor, enqueued on the
  current stream, no host synchronisation.

All compute runs in the native library (``liblrd.so``, include/lrd.h); torch
provides device memory, streams and pinned buffers.
"""

from __future__ import annotations

import threading

import numpy as np
import torch

from . import _native

_plans: dict = {}
_workspaces: dict = {}
_lock = threading.Lock()


def _plan(shape, patch, stride, form, batch, device, brick=None, split=0, gram_split=0, eigh_block=0):
    key = (tuple(shape), tuple(patch), int(stride), form, int(batch or 0), device,
           tuple(brick) if brick else None, int(split or 0), int(gram_split or 0), int(eigh_block or 0))
    with _lock:
        p = _plans.get(key)
        if p is None:
            with torch.cuda.device(device):
                p = _native.Plan(shape, patch, stride, form, batch or 0, brick, split, gram_split=gram_split,
                                 eigh_block=eigh_block)
            _plans[key] = p
    return p


def _workspace(plan, device, stream):
    key = (id(plan), device, stream)
    with _lock:
        ws = _workspaces.get(key)
        if ws is None or ws.numel() < plan.workspace_bytes:
            ws = torch.empty(max(plan.workspace_bytes, 1), dtype=torch.uint8, device=f"cuda:{device}")
            _workspaces[key] = ws
    return ws


def get_plan(shape, patch=(11, 11, 11), stride=3, form="plain", batch=None, device=None, brick=None,
             split=0, gram_split=0, eigh_block=0):
    """The cached native plan for a problem (creates it on first use). The
    launch-shape arguments (brick, split, gram_split, eigh_block) default to
    the plan's own choices; :func:`lowrank_gpu_fastest_b200.tune.tune` picks
    them by timing."""
    if device is None:
        device = torch.cuda.current_device()
    return _plan(shape, patch, stride, form, batch, device, brick, split, gram_split, eigh_block)


def denoise(vol, patch=(11, 11, 11), stride=3, batch=None, *, form="plain", return_ranks=False,
            out=None):
    """MP-PCA denoise of a 4D ``(x, y, z, t)`` float32 volume.

    Parameters mirror the ladder: ``patch`` (common.py:28), ``stride``
    (common.py:29), ``batch`` = patches per Gram/eigensolver launch
    (step8_tuned.py:21; ``None`` = all). ``form`` is ``"plain"`` (float32,
    step-0 accumulation order), ``"accurate"`` (float64 accumulation, close
    to the float64 run), ``"tensor"`` (the Gram and the reconstruction on the
    tensor cores in split TF32, the mean kept out of the sums as in accurate)
    or ``"tensor_bf16"`` (as tensor, the Gram with three-term BF16 split
    products). With ``return_ranks`` the per-patch MP ranks
    (x-major patch order) are returned too. ``out`` (CUDA input only): a
    preallocated output tensor of the volume's shape.
    """
    if not torch.cuda.is_available():
        raise RuntimeError("denoise needs a CUDA device (the native CUDA library is the only path)")
    is_np = isinstance(vol, np.ndarray)
    if is_np or (torch.is_tensor(vol) and not vol.is_cuda):
        t = torch.from_numpy(np.ascontiguousarray(vol, dtype=np.float32)) if is_np else vol.contiguous().float()
        return _denoise_host(t, patch, stride, batch, form, return_ranks, as_numpy=is_np)
    if not torch.is_tensor(vol):
        raise TypeError(f"vol must be a numpy array or torch tensor, got {type(vol)}")
    if vol.dtype != torch.float32:
        raise TypeError(f"vol must be float32, got {vol.dtype}")
    if vol.dim() != 4:
        raise ValueError(f"vol must be 4D (x, y, z, t), got shape {tuple(vol.shape)}")
    vol = vol.contiguous()
    device = vol.device.index if vol.device.index is not None else torch.cuda.current_device()
    with torch.cuda.device(device):
        plan = _plan(vol.shape, patch, stride, form, batch, device)
        stream = torch.cuda.current_stream(device)
        ws = _workspace(plan, device, stream.cuda_stream)
        if out is None:
            out = torch.empty_like(vol)
        elif out.shape != vol.shape or out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError("out must be a contiguous float32 tensor of the volume's shape")
        ranks = torch.empty(plan.n_patches, dtype=torch.int32, device=vol.device) if return_ranks else None
        plan.denoise(vol.data_ptr(), out.data_ptr(), ranks.data_ptr() if ranks is not None else None,
                     ws.data_ptr(), stream.cuda_stream)
        ws.record_stream(stream)
    return (out, ranks) if return_ranks else out


def denoise_with_noise(vol, patch=(11, 11, 11), stride=3, batch=None, *, form="plain"):
    """``denoise`` plus the per-patch by-products of the MP step: returns a dict
    with ``out`` (the denoised volume), ``ranks`` (per patch, x-major),
    ``sigma2`` (per patch: the MP noise variance estimate, the mean of the
    patch's t - p noise eigenvalues lambda / N) and ``noise`` (per voxel: the
    covering patches' estimates averaged with the denoiser's weights 1/(2+p)).
    numpy in -> numpy out; CUDA tensor in -> CUDA tensors (current stream)."""
    is_np = not (torch.is_tensor(vol) and vol.is_cuda)
    d = torch.from_numpy(np.ascontiguousarray(vol, dtype=np.float32)).cuda() if is_np else vol
    device = d.device.index if d.device.index is not None else torch.cuda.current_device()
    out, ranks = denoise(d, patch, stride, batch, form=form, return_ranks=True)
    with torch.cuda.device(device):
        plan = _plan(d.shape, patch, stride, form, batch, device)
        stream = torch.cuda.current_stream(device)
        ws = _workspace(plan, device, stream.cuda_stream)
        sigma2 = torch.empty(plan.n_patches, dtype=torch.float32, device=d.device)
        noise = torch.empty(d.shape[:3], dtype=torch.float32, device=d.device)
        plan.noise_map(ws.data_ptr(), sigma2.data_ptr(), noise.data_ptr(), stream.cuda_stream)
    res = dict(out=out, ranks=ranks, sigma2=sigma2, noise=noise)
    if is_np:
        res = {k: v.cpu().numpy() for k, v in res.items()}
    return res


def _denoise_host(t, patch, stride, batch, form, return_ranks, as_numpy):
    """Host -> host through ``lrd_denoise_host``: the volume moves in x-slabs
    on the plan's copy streams while earlier slabs compute; the result lands in
    pinned host memory (as step8_tuned.py:144-146 copies into pinned)."""
    if t.dim() != 4:
        raise ValueError(f"vol must be 4D (x, y, z, t), got shape {tuple(t.shape)}")
    device = torch.cuda.current_device()
    plan = _plan(t.shape, patch, stride, form, batch, device)
    stream = torch.cuda.current_stream(device)
    ws = _workspace(plan, device, stream.cuda_stream)
    dev = f"cuda:{device}"
    d_in = torch.empty(t.shape, dtype=torch.float32, device=dev)
    d_out = torch.empty_like(d_in)
    d_ranks = torch.empty(plan.n_patches, dtype=torch.int32, device=dev)
    host = torch.empty(t.shape, dtype=torch.float32, pin_memory=True)
    h_ranks = torch.empty(plan.n_patches, dtype=torch.int32, pin_memory=True) if return_ranks else None
    src = t.contiguous()
    plan.denoise_host(src.data_ptr(), host.data_ptr(), h_ranks.data_ptr() if h_ranks is not None else None,
                      d_in.data_ptr(), d_out.data_ptr(), d_ranks.data_ptr(), ws.data_ptr(), stream.cuda_stream)
    res = host.numpy() if as_numpy else host
    if return_ranks:
        return res, (h_ranks.numpy() if as_numpy else h_ranks)
    return res


_batch_plans: dict = {}


def denoise_batch(vols, patches=(11, 11, 11), strides=3, *, form="plain", use_graph=True, n_streams=4,
                  autotune=False, return_ranks=False):
    """Denoise many 4D volumes of different shapes in one batched call.

    ``vols``: list of float32 CUDA tensors (device-resident; outputs are CUDA
    tensors) or numpy arrays (copied in and out). ``patches`` / ``strides``:
    one value for all volumes or one per volume. The volumes run in packed
    launches - one grid per phase and kernel class across all of them
    (``lrd_batch_*``; ``n_streams`` is kept for compatibility and unused);
    with ``use_graph`` the whole batch is one CUDA-graph launch, captured on
    the first call with these buffers. With
    ``autotune`` each distinct (frames, patch, stride) gets its launch shapes
    (reconstruction brick and split, Gram split, eigensolver schedule) from
    :func:`lowrank_gpu_fastest_b200.tune.tune`.
    """
    if not torch.cuda.is_available():
        raise RuntimeError("denoise_batch needs a CUDA device")
    n = len(vols)
    if n == 0:
        return ([], []) if return_ranks else []
    if isinstance(patches, (list, tuple)) and len(patches) == n and isinstance(patches[0], (list, tuple)):
        plist = [tuple(int(v) for v in p) for p in patches]
    else:
        plist = [tuple(int(v) for v in patches)] * n
    slist = list(strides) if isinstance(strides, (list, tuple)) else [int(strides)] * n
    host = not torch.is_tensor(vols[0]) or not vols[0].is_cuda
    device = torch.cuda.current_device()
    dev_vols = []
    for v in vols:
        if host:
            t = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)) if isinstance(v, np.ndarray) else v
            dev_vols.append(t.to(f"cuda:{device}", non_blocking=False).contiguous())
        else:
            if v.dtype != torch.float32 or v.dim() != 4:
                raise ValueError("every volume must be a 4D float32 tensor")
            dev_vols.append(v.contiguous())
    problems = []
    for v, p, s in zip(dev_vols, plist, slist):
        pr = dict(shape=tuple(v.shape), patch=p, stride=int(s), form=form)
        if autotune:
            from .tune import tune

            pr.update(tune(tuple(v.shape), p, int(s), form, device))
        problems.append(pr)
    key = (device, int(n_streams), tuple((pr["shape"], pr["patch"], pr["stride"], pr["form"],
                                          tuple(pr.get("brick") or ()), pr.get("split", 0), pr.get("gram_split", 0),
                                          pr.get("eigh_block", 0)) for pr in problems))
    with _lock:
        bp = _batch_plans.get(key)
        if bp is None:
            bp = _native.BatchPlan(problems, n_streams)
            _batch_plans[key] = bp
            bp.buffers = None
    if bp.buffers is None or any(o.shape != v.shape for o, v in zip(bp.buffers["outs"], dev_vols)):
        bp.buffers = dict(
            ws=torch.empty(max(bp.workspace_bytes, 1), dtype=torch.uint8, device=f"cuda:{device}"),
            outs=[torch.empty_like(v) for v in dev_vols],
            ranks=[torch.empty(_n_patches(pr), dtype=torch.int32, device=f"cuda:{device}") for pr in problems],
        )
    buf = bp.buffers
    stream = torch.cuda.current_stream(device)
    bp.denoise([v.data_ptr() for v in dev_vols], [o.data_ptr() for o in buf["outs"]],
               [r.data_ptr() for r in buf["ranks"]], buf["ws"].data_ptr(), stream.cuda_stream, use_graph)
    if host:
        outs = [o.cpu().numpy() for o in buf["outs"]]
        ranks = [r.cpu().numpy() for r in buf["ranks"]]
    else:
        outs = [o.clone() for o in buf["outs"]]
        ranks = [r.clone() for r in buf["ranks"]]
    return (outs, ranks) if return_ranks else outs


def _n_patches(pr):
    from .problem import n_patches

    return n_patches(pr["shape"], pr["patch"], pr["stride"])
