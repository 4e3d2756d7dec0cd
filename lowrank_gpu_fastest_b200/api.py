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


def _plan(shape, patch, stride, form, batch, device, brick=None, split=0):
    key = (tuple(shape), tuple(patch), int(stride), form, int(batch or 0), device,
           tuple(brick) if brick else None, int(split or 0))
    with _lock:
        p = _plans.get(key)
        if p is None:
            with torch.cuda.device(device):
                p = _native.Plan(shape, patch, stride, form, batch or 0, brick, split)
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
             split=0):
    """The cached native plan for a problem (creates it on first use)."""
    if device is None:
        device = torch.cuda.current_device()
    return _plan(shape, patch, stride, form, batch, device, brick, split)


def denoise(vol, patch=(11, 11, 11), stride=3, batch=None, *, form="plain", return_ranks=False,
            out=None):
    """MP-PCA denoise of a 4D ``(x, y, z, t)`` float32 volume.

    Parameters mirror the ladder: ``patch`` (common.py:28), ``stride``
    (common.py:29), ``batch`` = patches per Gram/eigensolver launch
    (step8_tuned.py:21; ``None`` = all). ``form`` is ``"plain"`` (float32,
    step-0 accumulation order) or ``"accurate"``. With ``return_ranks`` the
    per-patch MP ranks (x-major patch order) are returned too.
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


def _denoise_host(t, patch, stride, batch, form, return_ranks, as_numpy):
    if t.dim() != 4:
        raise ValueError(f"vol must be 4D (x, y, z, t), got shape {tuple(t.shape)}")
    device = torch.cuda.current_device()
    plan = _plan(t.shape, patch, stride, form, batch, device)
    stream = torch.cuda.current_stream(device)
    ws = _workspace(plan, device, stream.cuda_stream)
    d_in = torch.empty(t.shape, dtype=torch.float32, device=f"cuda:{device}")
    d_out = torch.empty_like(d_in)
    d_in.copy_(t, non_blocking=True)
    ranks = torch.empty(plan.n_patches, dtype=torch.int32, device=d_in.device) if return_ranks else None
    plan.denoise(d_in.data_ptr(), d_out.data_ptr(), ranks.data_ptr() if ranks is not None else None,
                 ws.data_ptr(), stream.cuda_stream)
    host = torch.empty(t.shape, dtype=torch.float32, pin_memory=True)
    host.copy_(d_out)  # synchronous w.r.t. the host: the result is ready on return
    res = host.numpy() if as_numpy else host
    if return_ranks:
        r = ranks.cpu()
        return res, (r.numpy() if as_numpy else r)
    return res
