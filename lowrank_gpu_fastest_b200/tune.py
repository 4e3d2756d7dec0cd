"""Autotuner for the launch shapes of a problem: the reconstruction's brick
and threads per voxel, the column Gram's voxel-row split, and the
eigensolver's matrix-per-warp or matrix-per-CTA schedule.

Brick (0, 0, 0) with split 0, gram_split 0 and eigh_block 0 are the plan's
own choices: the warp kernel (one warp per 2x2x2 voxel block) for the frame
counts it is built for, else the brick kernel with the cost model's brick;
the Gram split measured best per frame count; one warp per matrix up to
T = 64.

Each phase is tuned on its own phase time (the library's phase events, mean
of ``reps`` warm calls) on a synthetic volume of the problem's shape: first
the reconstruction over a candidate set of bricks and splits, then the Gram
split over 1, 2, 4 (column Gram only), then the eigensolver schedule (T <= 64:
warp or CTA). Results are cached per (GPU architecture, frames, patch,
stride, form) in a JSON file (``LRD_TUNE_CACHE``, default
``~/.cache/lowrank_gpu_fastest_b200/tune.json``). The reconstruction choices
give bit-identical output; the Gram split and the eigensolver schedule
change the float32 rounding of the Gram and the eigenvalues (the ranks stay
the same: near-ties are decided in float64 from the input).
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
    return f"v2|{arch}|T{T}|p{'x'.join(str(int(v)) for v in patch)}|s{int(stride)}|{form}"


def _choice(d) -> dict:
    return dict(brick=tuple(int(v) for v in d["brick"]), split=int(d["split"]),
                gram_split=int(d.get("gram_split", 0)), eigh_block=int(d.get("eigh_block", 0)))


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
    """Best launch shapes for the problem on the current GPU (cached): a dict
    with ``brick``, ``split``, ``gram_split`` and ``eigh_block`` (the keyword
    arguments of :func:`lowrank_gpu_fastest_b200.api.get_plan`).

    Reconstruction candidates are ranked by a proxy first (thread-slots of
    the brick, as the plan's model) and the ``max_candidates`` best are timed.
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
                return dict(_mem[k])
            disk = _load()
            if k in disk:
                _mem[k] = _choice(disk[k])
                return dict(_mem[k])

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
    timed = {"recon": [], "gram": [], "eigh_mp": []}
    with torch.cuda.device(device):
        d = torch.from_numpy(vol).cuda()
        out = torch.empty_like(d)
        s = torch.cuda.current_stream().cuda_stream
        ws = [None]

        def phase_ms(phase, brick, split, gram_split=0, eigh_block=0):
            try:
                plan = _native.Plan(shape, patch, stride, form, 0, brick, split, gram_split=gram_split,
                                    eigh_block=eigh_block)
            except _native.LrdError:
                return None
            if ws[0] is None or ws[0].numel() < plan.workspace_bytes:
                ws[0] = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device=d.device)
            plan.denoise(d.data_ptr(), out.data_ptr(), None, ws[0].data_ptr(), s)
            plan.set_profiling(True)
            for _ in range(reps):
                plan.denoise(d.data_ptr(), out.data_ptr(), None, ws[0].data_ptr(), s)
            ph, n = plan.phase_ms()
            plan.set_profiling(False)
            return ph[phase] / max(n, 1)

        best = None
        best_ms = float("inf")
        for brick, split in cands:  # reconstruction
            ms = phase_ms("recon", brick, split)
            if ms is None:
                continue
            timed["recon"].append([list(brick), split, round(ms, 4)])
            if ms < best_ms:
                best, best_ms = (tuple(brick), int(split)), ms
        if best is None:
            raise RuntimeError("autotuner: no candidate plan could be created")
        choice = dict(brick=best[0], split=best[1], gram_split=0, eigh_block=0)
        best_gram = (None, float("inf"))
        for gs in (1, 2, 4):  # column-Gram voxel-row split
            ms = phase_ms("gram", best[0], best[1], gram_split=gs)
            if ms is not None:
                timed["gram"].append([gs, round(ms, 4)])
                if ms < best_gram[1]:
                    best_gram = (gs, ms)
        if best_gram[0] is not None:
            choice["gram_split"] = best_gram[0]
        best_eigh = (None, float("inf"))
        for eb in ((1, 2) if T <= 64 else (2,)):  # eigensolver: warp or CTA per matrix
            ms = phase_ms("eigh_mp", best[0], best[1], gram_split=choice["gram_split"], eigh_block=eb)
            if ms is not None:
                timed["eigh_mp"].append([eb, round(ms, 4)])
                if ms < best_eigh[1]:
                    best_eigh = (eb, ms)
        if best_eigh[0] is not None:
            choice["eigh_block"] = best_eigh[0]
    with _lock:
        _mem[k] = dict(choice)
        disk = _load()
        disk[k] = {"brick": list(choice["brick"]), "split": choice["split"], "gram_split": choice["gram_split"],
                   "eigh_block": choice["eigh_block"], "recon_ms": best_ms, "timed": timed}
        _save(disk)
    return dict(choice)


def clear_memory_cache():
    with _lock:
        _mem.clear()


__all__ = ["tune", "key", "candidates", "cache_path", "clear_memory_cache", "np"]
