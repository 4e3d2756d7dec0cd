// Per-voxel noise map from the per-patch MP noise estimates.
//
// Every patch's eigensolve leaves sigma^2 = (sum of its t - p noise
// eigenvalues) / (t - p) in the workspace (mp_rank). A voxel's map value is
// the weighted mean over the patches covering it, with the patch weights
// w = 1/(2 + p) of the denoised output and the same x-major patch order and
// float32 rounding as the output's accumulation (step0_numpy_loop.py:32-39):
// sum w sigma^2 / max(sum w, 1e-12), 0 where no patch covers the voxel.
#pragma once

#include "lrd_common.cuh"

namespace lrd {

// grid: ceil(nvox / blockDim.x) blocks; one thread per voxel.
__global__ void noise_map_kernel(const float* __restrict__ sig2, const float* __restrict__ wgt,
                                 float* __restrict__ out, Geom g, AxisTables tab) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nvox = (long long)g.nx * g.ny * g.nz;
  if (v >= nvox) return;
  const int z = (int)(v % g.nz);
  const int y = (int)((v / g.nz) % g.ny);
  const int x = (int)(v / ((long long)g.ny * g.nz));
  const int ilo = tab.cover[0][2 * x], ihi = tab.cover[0][2 * x + 1];
  const int jlo = tab.cover[1][2 * y], jhi = tab.cover[1][2 * y + 1];
  const int klo = tab.cover[2][2 * z], khi = tab.cover[2][2 * z + 1];
  float acc = 0.f, ws = 0.f;
  for (int i = ilo; i <= ihi; ++i)
    for (int j = jlo; j <= jhi; ++j)
      for (int k = klo; k <= khi; ++k) {
        const long long pid = ((long long)i * g.ncy + j) * g.ncz + k;
        const float w = wgt[pid];
        acc = __fadd_rn(acc, __fmul_rn(w, sig2[pid]));
        ws = __fadd_rn(ws, w);
      }
  out[v] = __fdiv_rn(acc, fmaxf(ws, 1e-12f));
}

}  // namespace lrd
