"""B200-native patch-wise MP-PCA denoiser (U-free Gram route).

Public surface:

* :func:`denoise` - drop-in for the ladder's ``denoise`` entry point
  (step8_tuned.py:116-146) with patch / stride / batch as arguments;
* :func:`denoise_batch` - many volumes of uneven shape in one call;
* :func:`denoise_with_noise` - ``denoise`` plus per-patch ranks and noise
  variance estimates and the voxel noise map;
* :mod:`.shard` - one volume over several GPUs (x-slabs, halo hand-off);
* :mod:`.serve` - continuous-batching request server;
* :mod:`.report` - per-kernel breakdown and result tables;
* :mod:`.problem` - the patch index space (common.py:37-44);
* :mod:`.harness` - phantoms and the ``common.run``-style timing harness;
* :mod:`._native` - the ctypes binding of ``liblrd.so`` (include/lrd.h).
"""

from .problem import Problem, patch_corners, patch_bases, n_patches  # noqa: F401
from .harness import make_phantom, make_phantom_lowrank, rel_l2  # noqa: F401


def denoise(*args, **kwargs):
    """See :func:`lowrank_gpu_fastest_b200.api.denoise`."""
    from .api import denoise as _d

    return _d(*args, **kwargs)


def denoise_with_noise(*args, **kwargs):
    """See :func:`lowrank_gpu_fastest_b200.api.denoise_with_noise`."""
    from .api import denoise_with_noise as _d

    return _d(*args, **kwargs)


def denoise_batch(*args, **kwargs):
    """See :func:`lowrank_gpu_fastest_b200.api.denoise_batch`."""
    from .api import denoise_batch as _d

    return _d(*args, **kwargs)


__all__ = ["denoise", "denoise_batch", "denoise_with_noise", "Problem", "patch_corners", "patch_bases", "n_patches", "make_phantom",
           "make_phantom_lowrank", "rel_l2"]
