"""Problem definition of the patch-wise MP-PCA denoiser: the patch index space.

A volume is a C-ordered float32 array ``(X, Y, Z, T)`` (t contiguous). Patches
are ``(px, py, pz)`` windows slid with one stride on all three spatial axes.
Along each axis the corner positions are the stride grid plus one extra,
border-shifted corner ``s - p`` where the grid does not land on the border
(common.py:37-44: ``sorted({*range(0, s - p + 1, step), s - p})``); the patch
list is the Cartesian product of the three axis lists in x-major order, so the
linear patch index is ``(i * ncy + j) * ncz + k`` for axis indices ``i, j, k``.

Everything here is exact integer work on the host; the device kernels receive
the per-axis tables built by :func:`axis_tables`.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np


def axis_corners(size: int, patch: int, stride: int) -> np.ndarray:
    """Sorted corner positions along one axis (common.py:40-43)."""
    if patch > size:
        raise ValueError(f"patch {patch} larger than axis {size}")
    if stride < 1:
        raise ValueError(f"stride must be >= 1, got {stride}")
    return np.array(sorted({*range(0, size - patch + 1, stride), size - patch}), dtype=np.int64)


def patch_corners(vol_shape, patch=(11, 11, 11), stride=3) -> np.ndarray:
    """Corners of every patch, shape ``(n_patches, 3)`` int64, x-major order.

    Same list, in the same order, as ``common.patch_corners`` (common.py:37-44).
    """
    ranges = [axis_corners(s, p, stride) for s, p in zip(vol_shape[:3], patch)]
    return np.array(list(itertools.product(*ranges)), dtype=np.int64).reshape(-1, 3)


def n_patches(vol_shape, patch=(11, 11, 11), stride=3) -> int:
    return int(np.prod([len(axis_corners(s, p, stride)) for s, p in zip(vol_shape[:3], patch)]))


def patch_bases(vol_shape, patch=(11, 11, 11), stride=3) -> np.ndarray:
    """Row of the first voxel of every patch in the ``(X*Y*Z, T)`` view.

    ``base = cx*Y*Z + cy*Z + cz`` (step8_tuned.py:89-93).
    """
    _, ny, nz = vol_shape[:3]
    c = patch_corners(vol_shape, patch, stride)
    return c[:, 0] * ny * nz + c[:, 1] * nz + c[:, 2]


def cover_range(size: int, patch: int, stride: int) -> np.ndarray:
    """For every voxel position along an axis, the inclusive index range
    ``[lo, hi]`` into :func:`axis_corners` of the corners whose window covers it.

    Corners are sorted, so the covering set ``{c : c <= x <= c + patch - 1}`` is
    a contiguous index range. Shape ``(size, 2)`` int32.
    """
    c = axis_corners(size, patch, stride)
    x = np.arange(size)
    lo = np.searchsorted(c, x - patch + 1, side="left")
    hi = np.searchsorted(c, x, side="right") - 1
    return np.stack([lo, hi], axis=1).astype(np.int32)


@dataclass(frozen=True)
class Problem:
    """One denoise problem: volume shape, patch shape and stride."""

    shape: tuple  # (X, Y, Z, T)
    patch: tuple = (11, 11, 11)
    stride: int = 3

    def __post_init__(self):
        if len(self.shape) != 4:
            raise ValueError(f"volume must be 4D (x, y, z, t), got shape {self.shape}")
        if len(self.patch) != 3:
            raise ValueError(f"patch must have 3 sides, got {self.patch}")
        for s, p in zip(self.shape[:3], self.patch):
            if p < 1 or p > s:
                raise ValueError(f"patch {self.patch} does not fit volume {self.shape}")
        if self.stride < 1:
            raise ValueError(f"stride must be >= 1, got {self.stride}")
        if self.shape[3] < 2:
            raise ValueError("need at least 2 frames")

    @property
    def n_voxels_per_patch(self) -> int:
        return int(np.prod(self.patch))

    @property
    def n_patches(self) -> int:
        return n_patches(self.shape, self.patch, self.stride)

    def corners(self) -> np.ndarray:
        return patch_corners(self.shape, self.patch, self.stride)
