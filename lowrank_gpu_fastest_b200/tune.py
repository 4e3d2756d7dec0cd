"""Autotuner for the reconstruction launch shape (brick and threads per voxel).

Brick (0, 0, 0) with split 0 is the plan's own choice: the warp kernel (one
warp per 2x2x2 voxel block) for the frame counts it is built for, else the
brick kernel with the cost model's brick.

The reconstruction kernel's speed depends on the brick of voxels a CTA owns
(how many of the patches touching the brick actually cover each voxel, how
many CTAs fit on an SM) and on how many threads share a voxel's frames. The
plan's cost model picks a default; this module times a small candidate set on
the current GPU with a synthetic volume of the problem's shape and keeps the
fastest. Results are cached per (GPU architecture, frames, patch, stride, form)
in a JSON file (``LRD_TUNE_CACHE``, default
``~/.cache/lowrank_gpu_fastest_b200/tune.json``). Every candidate gives
bit-identical output - only the time differs.
"""

from __future__ import annotations

import json
import os
import threading

import numpy as np

_lock = threading.Lock()
_mem: dict = {}


def cache_path() -> str:
    return os.environ.get("LRD_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "lowrank_gpu_fastest_b200", "tune.json"))


def _load():
    p = cache_path()
    if os.path.exists(p):
        try:
            with open(p) as f:
                return json.load(f)
        except (OSError, ValueError):
            return {}
    return {}


def _save(d):
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def key(arch: str, T: int, patch, stride: int, form: str) -> str:
    return f"{arch}|T{T}|p{'x'.join(str(int(v)) for v in patch)}|s{int(stride)}|{form}"


def candidates(T: int, patch, stride: int):
    """Bricks near the stride lattice, two thread layouts, 27..256 threads."""
    s = max(1, int(stride))
    sides = sorted({1, 2, 3, 4, 6, s, 2 * s})
    out = []
    for split in ((2, 4) if T <= 96 else (4,)):
        for bx in sides:
            for by in sides:
                for bz in sides + [8, 12]:
                    th = bx * by * bz * split
                    if 27 <= th <= 256 and bx <= 8 and by <= 8:
                        out.append(((bx, by, bz), split))
    return out


def tune(shape, patch=(11, 11, 11), stride=3, form="plain", device=None, max_candidates=24, reps=3,
         force=False):
    """Best ``(brick, split)`` for the problem on the current GPU (cached).

    Candidates are ranked by a proxy first (thread-slots of the brick, as the
    plan's model) and the ``max_candidates`` best are timed by the library's
    phase events (reconstruction phase, mean of ``reps`` warm calls).
    """
    import torch

    from . import _native
    from .harness import make_phantom_lowrank
    from .problem import axis_corners

    if device is None:
        device = torch.cuda.current_device()
    props = torch.cuda.get_device_properties(device)
    arch = f"sm_{props.major}{props.minor}:{props.multi_processor_count}"
    T = int(shape[3])
    k = key(arch, T, patch, stride, form)
    with _lock:
        if not force:
            if k in _mem:
                return _mem[k]
            disk = _load()
            if k in disk:
                v = disk[k]
                _mem[k] = (tuple(v["brick"]), int(v["split"]))
                return _mem[k]

    def slots(b):
        tot = 1.0
        for a in range(3):
            c = axis_corners(int(shape[a]), int(patch[a]), int(stride))
            nb = -(-int(shape[a]) // b[a])
            s_ = 0
            for i in range(nb):
                lo, hi = i * b[a], min(int(shape[a]), (i + 1) * b[a]) - 1
                s_ += int(((c <= hi) & (c + patch[a] - 1 >= lo)).sum()) * b[a]
            tot *= s_
        return tot

    cands = candidates(T, patch, stride)
    cands.sort(key=lambda c: slots(c[0]) * c[1] / max(1, min(4, c[1])))
    # the plan's own choice first (brick and split 0: the warp-per-2x2x2-block
    # kernel where it is built for T, else the cost model's brick)
    cands = [((0, 0, 0), 0)] + cands[:max_candidates]
    vol, _ = make_phantom_lowrank(tuple(int(v) for v in shape), seed=7)
    best, best_ms, results = None, float("inf"), []
    with torch.cuda.device(device):
        d = torch.from_numpy(vol).cuda()
        out = torch.empty_like(d)
        s = torch.cuda.current_stream().cuda_stream
        ws = None
        for brick, split in cands:
            try:
                plan = _native.Plan(shape, patch, stride, form, 0, brick, split)
            except _native.LrdError:
                continue
            if ws is None or ws.numel() < plan.workspace_bytes:
                ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device=d.device)
            plan.denoise(d.data_ptr(), out.data_ptr(), None, ws.data_ptr(), s)
            plan.set_profiling(True)
            for _ in range(reps):
                plan.denoise(d.data_ptr(), out.data_ptr(), None, ws.data_ptr(), s)
            ph, n = plan.phase_ms()
            plan.set_profiling(False)
            ms = ph["recon"] / max(n, 1)
            results.append((brick, split, ms))
            if ms < best_ms:
                best, best_ms = (tuple(brick), int(split)), ms
    if best is None:
        raise RuntimeError("autotuner: no candidate plan could be created")
    with _lock:
        _mem[k] = best
        disk = _load()
        disk[k] = {"brick": list(best[0]), "split": best[1], "recon_ms": best_ms,
                   "timed": [[list(b), sp, round(ms, 4)] for b, sp, ms in results]}
        _save(disk)
    return best


def clear_memory_cache():
    with _lock:
        _mem.clear()


__all__ = ["tune", "key", "candidates", "cache_path", "clear_memory_cache", "np"]
