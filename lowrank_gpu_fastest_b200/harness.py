"""Synthetic inputs and the timing/validation harness around ``denoise``.

Two phantom generators:

* :func:`make_phantom` - the ladder's own phantom (common.py:47-77): a rank-5
  smooth spatio-temporal signal on a ~1000 baseline plus N(0, 4^2) noise. Same
  draws from the same ``numpy.random.default_rng(seed)`` stream, so the output
  is bit-identical to the ladder's for equal arguments.
* :func:`make_phantom_lowrank` - the benchmark phantom: a rank-r signal built as
  a sum of r smooth random spatial maps times random temporal curves, scaled
  into [0, 1], plus i.i.d. N(0, sigma^2) noise, float32, fixed seed.

:func:`run` mirrors ``common.run`` (common.py:103-172): one warm call, then the
best of ``repeats`` host->host wall-clock calls, relative L2 against a
reference output, and the same JSON result fields.
"""

from __future__ import annotations

import json
import time

import numpy as np


def _smooth_field(rng, grids):
    freqs = rng.uniform(0.5, 3.0, size=3)
    phases = rng.uniform(0, 2 * np.pi, size=3)
    return np.prod(
        [np.cos(2 * np.pi * f * g + ph) for f, g, ph in zip(freqs, grids, phases)], axis=0
    )


def make_phantom(shape=(96, 96, 48, 48), rank=5, sigma=4.0, seed=0):
    """The ladder's phantom (common.py:47-77). Returns ``(noisy, clean)`` float32.

    The draw order (field frequencies/phases, then course frequencies/phases,
    then the baseline field, then the noise) follows the ladder so the same
    seed yields the same arrays.
    """
    rng = np.random.default_rng(seed)
    *spatial, t = shape
    grids = np.meshgrid(*(np.linspace(0, 1, s) for s in spatial), indexing="ij")
    maps = np.stack([_smooth_field(rng, grids) for _ in range(rank)], axis=-1)
    time_axis = np.linspace(0, 1, t)
    courses = np.stack(
        [np.sin(2 * np.pi * rng.uniform(1, 6) * time_axis + rng.uniform(0, 6)) for _ in range(rank)]
    )
    baseline = 1000.0 * (1.2 + _smooth_field(rng, grids))[..., None]
    clean = baseline + 20.0 * maps @ courses
    noisy = clean + rng.normal(scale=sigma, size=shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def make_phantom_lowrank(shape=(96, 96, 48, 48), rank=4, sigma=0.05, seed=0):
    """Benchmark phantom: rank-``rank`` signal in [0, 1] plus N(0, sigma^2) noise.

    Spatial maps are products of cosines with random frequencies and phases,
    temporal curves are sinusoids with random frequency and phase; the product
    sum is min-max scaled into [0, 1]. Returns ``(noisy, clean)`` float32.
    """
    rng = np.random.default_rng(seed)
    *spatial, t = shape
    grids = np.meshgrid(*(np.linspace(0, 1, s) for s in spatial), indexing="ij")
    maps = np.stack([_smooth_field(rng, grids) for _ in range(rank)], axis=-1)
    time_axis = np.linspace(0, 1, t)
    curves = np.stack(
        [np.sin(2 * np.pi * rng.uniform(1, 6) * time_axis + rng.uniform(0, 6)) for _ in range(rank)]
    )
    sig = maps @ curves
    lo, hi = sig.min(), sig.max()
    clean = (sig - lo) / (hi - lo) if hi > lo else np.zeros_like(sig)
    noisy = clean + rng.normal(scale=sigma, size=shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def rel_l2(x, ref) -> float:
    """``||x - ref|| / ||ref||`` in float64 (common.py:149)."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(x - ref) / den) if den > 0 else float(np.linalg.norm(x - ref))


def rmse(x, ref) -> float:
    return float(np.sqrt(np.mean((np.asarray(x, np.float64) - ref) ** 2)))


def run(name, denoise, noisy, clean=None, ref=None, n_patches=None, repeats=5, max_seconds=60.0,
        sync=None, out_json=None):
    """Benchmark ``denoise(noisy) -> denoised`` host->host and validate it.

    Mirrors common.py:103-172: a warm-up call (absorbs allocation and module
    load), then up to ``repeats`` timed calls within ``max_seconds``, best of.
    ``ref`` is the output the result is compared with (the step-0 oracle's
    output in the ladder); ``sync`` is called after each call (a device
    synchronize when the work is asynchronous).
    """
    sync = sync or (lambda: None)
    t0 = time.perf_counter()
    out = denoise(noisy)
    sync()
    first = time.perf_counter() - t0
    times = []
    budget = time.perf_counter() + max_seconds
    for _ in range(repeats):
        t0 = time.perf_counter()
        denoise(noisy)
        sync()
        times.append(time.perf_counter() - t0)
        if time.perf_counter() > budget:
            break
    best = min(times)
    res = dict(
        name=name,
        seconds=best,
        first_call=first,
        us_per_patch=1e6 * best / n_patches if n_patches else None,
        patches_per_s=n_patches / best if n_patches else None,
        rel_err_vs_ref=rel_l2(out, ref) if ref is not None else 0.0,
        rmse_noisy=rmse(noisy, clean) if clean is not None else None,
        rmse_denoised=rmse(out, clean) if clean is not None else None,
        n_patches=n_patches,
    )
    if out_json:
        with open(out_json, "w") as f:
            json.dump(res, f, indent=1)
    return res, out
