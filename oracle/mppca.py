"""CPU oracle for the patch-wise MP-PCA denoiser - TEST INFRASTRUCTURE ONLY.

This module is the checker: the pytest suite, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` call it to
produce reference outputs and CPU timings. The product path never imports it.

It restates the ladder's step-0 NumPy loop (step0_numpy_loop.py:8-39) with the
problem definition of common.py:37-44:

* per patch, the ``(N, T)`` Casorati matrix ``x`` is centred along time with
  NumPy's float32 mean (step0:11), its thin SVD is taken (step0:12), the null
  direction created by centring is dropped (step0:15-16), ``eigs = s**2 / n``
  (step0:18) and the MP rank is the COUNT of indices passing
  ``(eigs - eigs[-1]) * (t - i) * (n - i) > 4 * rcum * sqrt(t * n)``
  (step0:19-24; NumPy promotes this test to float64 because ``i`` is int64);
* the denoised patch is ``(u_p * s_p) @ vt_p + m`` (step0:25), accumulated with
  weight ``w = 1 / (2 + p)`` into ``out`` and ``wsum`` in patch order, in the
  volume's dtype (step0:36-38), and the result is ``out / max(wsum, 1e-12)``
  (step0:39).

Calling it with a float64 volume gives the FP64 oracle (the same code on
``vol.astype(float64)``). :func:`gram_route_patch` restates step 4's U-free
route (step4_gram_eigh.py:40-67) in float64 as a per-stage checker (Gram,
eigenvalues, rank, projector).

Parity pin: tests/golden holds outputs of the ladder's own step 0 (generated by
tests/golden/make_golden.py, which imports the reference); the oracle is checked
against them in tests/test_oracle.py.
"""

from __future__ import annotations

import itertools
import os

import numpy as np


def axis_corners(size, patch, step):
    """common.py:40-43."""
    return sorted({*range(0, size - patch + 1, step), size - patch})


def patch_corners(vol_shape, patch=(11, 11, 11), step=3):
    """common.py:37-44: product of the per-axis corner lists, x-major."""
    ranges = [axis_corners(s, p, step) for s, p in zip(vol_shape[:3], patch)]
    return np.array(list(itertools.product(*ranges)), dtype=np.int64).reshape(-1, 3)


def mp_rank_from_eigs(eigs, n):
    """MP rank from descending ``eigs = s**2 / n`` with the null direction dropped.

    step0_numpy_loop.py:19-24. ``eigs`` keeps its dtype (float32 in the fp32
    oracle); the product with the int64 ``p_range`` makes the test float64.
    """
    t = eigs.shape[0]
    rcum = np.cumsum(eigs[::-1])[::-1]
    p_range = np.arange(t)
    signal = (eigs - eigs[-1]) * (t - p_range) * (n - p_range) > 4 * rcum * np.sqrt(t * n)
    return int(signal.sum())


def mppca_patch(x):
    """MP-PCA on one ``(N, T)`` Casorati matrix -> ``(denoised, rank)``.

    step0_numpy_loop.py:8-25.
    """
    n, t = x.shape
    m = x.mean(axis=1, keepdims=True)
    u, s, vt = np.linalg.svd(x - m, full_matrices=False)
    t -= 1
    u, s, vt = u[:, :t], s[:t], vt[:t]
    eigs = s**2 / n
    p = mp_rank_from_eigs(eigs, n)
    return (u[:, :p] * s[:p]) @ vt[:p] + m, p


def denoise(vol, patch=(11, 11, 11), step=3, corners=None):
    """Step-0 loop (step0_numpy_loop.py:28-39). Returns ``(out, ranks)``.

    Arithmetic runs in ``vol.dtype`` (float32 for the oracle proper, float64 for
    the FP64 oracle). ``ranks[i]`` is the rank chosen for ``corners[i]``.
    """
    vol = np.asarray(vol)
    out = np.zeros_like(vol)
    wsum = np.zeros(vol.shape[:3] + (1,), dtype=vol.dtype)
    px, py, pz = patch
    if corners is None:
        corners = patch_corners(vol.shape, patch, step)
    ranks = np.empty(len(corners), dtype=np.int32)
    for idx, (i, j, k) in enumerate(corners):
        sl = np.s_[i : i + px, j : j + py, k : k + pz]
        x = vol[sl].reshape(-1, vol.shape[-1])
        xd, p = mppca_patch(x)
        ranks[idx] = p
        w = 1.0 / (2.0 + p)
        out[sl] += w * xd.reshape(px, py, pz, -1)
        wsum[sl] += w
    return out / np.maximum(wsum, 1e-12), ranks


def patch_noise(x):
    """MP rank and noise variance estimate of one ``(N, T)`` patch: the mean
    of the t - p noise eigenvalues ``eigs = s**2 / N`` after step 0's rank
    test (step0_numpy_loop.py:10-24): ``rcum[p] / (t - p)`` in float32, 0 when
    p = t. The reference computes ``rcum`` but returns only the denoised
    patch; the estimate is the package's per-patch output."""
    n, t = x.shape
    m = x.mean(axis=1, keepdims=True)
    s = np.linalg.svd(x - m, compute_uv=False)[: t - 1]
    t -= 1
    eigs = s**2 / n
    p = mp_rank_from_eigs(eigs, n)
    rcum = np.cumsum(eigs[::-1])[::-1]
    sig2 = np.float32(rcum[p] / np.float32(t - p)) if p < t else np.float32(0)
    return p, sig2


def noise_map(vol, patch=(11, 11, 11), step=3):
    """Per-patch ``(ranks, sigma2)`` and the voxel map: the covering patches'
    estimates averaged with weights 1/(2+p) in step 0's patch order and
    float32 rounding (step0_numpy_loop.py:32-39)."""
    vol = np.asarray(vol, dtype=np.float32)
    px, py, pz = patch
    corners = patch_corners(vol.shape, patch, step)
    ranks = np.empty(len(corners), dtype=np.int32)
    sig2 = np.empty(len(corners), dtype=np.float32)
    acc = np.zeros(vol.shape[:3], dtype=np.float32)
    wsum = np.zeros(vol.shape[:3], dtype=np.float32)
    for idx, (i, j, k) in enumerate(corners):
        x = vol[i : i + px, j : j + py, k : k + pz].reshape(-1, vol.shape[-1])
        p, s2 = patch_noise(x)
        ranks[idx], sig2[idx] = p, s2
        w = np.float32(1.0 / (2.0 + p))
        acc[i : i + px, j : j + py, k : k + pz] += w * s2
        wsum[i : i + px, j : j + py, k : k + pz] += w
    return ranks, sig2, acc / np.maximum(wsum, np.float32(1e-12))


def denoise_fp64(vol, patch=(11, 11, 11), step=3):
    """FP64 oracle: the same loop on ``vol.astype(float64)``."""
    return denoise(np.asarray(vol, dtype=np.float64), patch, step)


def ranks_only(vol, patch=(11, 11, 11), step=3, corners=None):
    """Per-patch step-0 ranks without the accumulation (cheaper: no U)."""
    vol = np.asarray(vol)
    px, py, pz = patch
    if corners is None:
        corners = patch_corners(vol.shape, patch, step)
    ranks = np.empty(len(corners), dtype=np.int32)
    for idx, (i, j, k) in enumerate(corners):
        x = vol[i : i + px, j : j + py, k : k + pz].reshape(-1, vol.shape[-1])
        m = x.mean(axis=1, keepdims=True)
        s = np.linalg.svd(x - m, compute_uv=False)[: x.shape[1] - 1]
        ranks[idx] = mp_rank_from_eigs(s**2 / x.shape[0], x.shape[0])
    return ranks


def patch_matrix(vol, corner, patch):
    """The (N, T) Casorati matrix of the patch at ``corner`` (x-major voxels)."""
    i, j, k = (int(c) for c in corner)
    return vol[i:i + patch[0], j:j + patch[1], k:k + patch[2]].reshape(-1, vol.shape[-1])


def mp_tie_scale(x):
    """Distance of one patch's MP decision from a tie, in units of its largest
    eigenvalue: min over indices i of |lhs_i - rhs_i| / (eigs_0 (t - i)(n - i))
    with the float64 test of step0_numpy_loop.py:19-24 (eigs from a float64
    SVD of the centred patch). An eigenvalue error below this fraction of the
    largest eigenvalue cannot flip the count at index i through its own term.
    """
    x = np.asarray(x, dtype=np.float64)
    n, t = x.shape
    s = np.linalg.svd(x - x.mean(axis=1, keepdims=True), compute_uv=False)
    t -= 1
    eigs = s[:t] ** 2 / n
    rcum = np.cumsum(eigs[::-1])[::-1]
    i = np.arange(t)
    lhs = (eigs - eigs[-1]) * (t - i) * (n - i)
    rhs = 4 * rcum * np.sqrt(t * n)
    return float(np.min(np.abs(lhs - rhs) / (eigs[0] * (t - i) * (n - i))))


def gram_route_patch(x):
    """Step 4's U-free route on one patch, float64 (step4_gram_eigh.py:40-67).

    Returns a dict with the centred Gram ``G``, ascending eigenvalues ``lam``,
    eigenvectors ``v`` (columns), rank ``p`` and projector ``P = V_p V_p^T``.
    """
    x = np.asarray(x, dtype=np.float64)
    n, t = x.shape
    m = x.mean(axis=1, keepdims=True)
    xc = x - m
    g = xc.T @ xc
    lam, v = np.linalg.eigh(g)
    eigs = np.clip(lam[1:][::-1], 0, None) / n
    p = mp_rank_from_eigs(eigs, n)
    vp = v[:, ::-1][:, :p]
    return dict(G=g, lam=lam, v=v, p=p, P=vp @ vp.T, m=m[:, 0])


def region_patches(vol_shape, patch, step, lo, hi):
    """Indices (into the x-major corner list) of patches that touch the box
    ``[lo, hi)`` and the sub-box of voxels all of whose covering patches are
    among them (the whole box: every covering patch touches it)."""
    corners = patch_corners(vol_shape, patch, step)
    p = np.asarray(patch)
    touch = np.all((corners <= np.asarray(hi) - 1) & (corners + p - 1 >= np.asarray(lo)), axis=1)
    return np.nonzero(touch)[0], corners


def denoise_region(vol, patch, step, lo, hi):
    """Step-0 output restricted to the box ``[lo, hi)`` of voxels.

    Every patch covering a voxel of the box touches the box, so running the
    step-0 loop over exactly those patches (in the same x-major order) gives
    the box's output bit-for-bit as the full loop would. Returns
    ``(out_box, patch_indices, ranks)``.
    """
    vol = np.asarray(vol)
    idx, corners = region_patches(vol.shape, patch, step, lo, hi)
    out, ranks = denoise(vol, patch, step, corners=corners[idx])
    sl = tuple(slice(a, b) for a, b in zip(lo, hi))
    return out[sl], idx, ranks


def _worker(args):
    vol, patch, step, corners = args
    return ranks_only(vol, patch, step, corners)


def ranks_parallel(vol, patch=(11, 11, 11), step=3, processes=None):
    """Per-patch ranks with a ``spawn`` process pool, one BLAS thread each."""
    import multiprocessing as mp

    corners = patch_corners(vol.shape, patch, step)
    processes = processes or os.cpu_count() or 1
    chunks = np.array_split(corners, processes * 4)
    ctx = mp.get_context("spawn")
    env_old = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in env_old:
        os.environ[k] = "1"
    try:
        with ctx.Pool(processes) as pool:
            parts = pool.map(_worker, [(vol, patch, step, c) for c in chunks if len(c)])
    finally:
        for k, v in env_old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return np.concatenate(parts)


def _sums_worker(args):
    vol, patch, corners = args
    vol = np.asarray(vol)
    out = np.zeros_like(vol)
    wsum = np.zeros(vol.shape[:3] + (1,), dtype=vol.dtype)
    px, py, pz = patch
    ranks = np.empty(len(corners), dtype=np.int32)
    for idx, (i, j, k) in enumerate(corners):
        sl = np.s_[i : i + px, j : j + py, k : k + pz]
        xd, p = mppca_patch(vol[sl].reshape(-1, vol.shape[-1]))
        ranks[idx] = p
        w = 1.0 / (2.0 + p)
        out[sl] += w * xd.reshape(px, py, pz, -1)
        wsum[sl] += w
    return out, wsum, ranks


def denoise_fp64_parallel(vol, patch=(11, 11, 11), step=3, processes=None):
    """The FP64 oracle (step 0 on ``vol.astype(float64)``) over a ``spawn``
    process pool: each worker accumulates a contiguous run of the corner
    list, the partial sums are added in float64 (the order of those few
    additions is the only difference from the serial loop, ~1e-16).
    Returns ``(out, ranks)``."""
    import multiprocessing as mp

    vol = np.asarray(vol, dtype=np.float64)
    corners = patch_corners(vol.shape, patch, step)
    processes = processes or os.cpu_count() or 1
    chunks = [c for c in np.array_split(corners, processes) if len(c)]
    env_old = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in env_old:
        os.environ[k] = "1"
    try:
        with mp.get_context("spawn").Pool(len(chunks)) as pool:
            parts = pool.map(_sums_worker, [(vol, patch, c) for c in chunks])
    finally:
        for k, v in env_old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    out = np.zeros_like(vol)
    wsum = np.zeros(vol.shape[:3] + (1,), dtype=np.float64)
    for o, w, _ in parts:
        out += o
        wsum += w
    return out / np.maximum(wsum, 1e-12), np.concatenate([r for _, _, r in parts])
