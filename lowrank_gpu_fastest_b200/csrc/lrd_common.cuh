// Shared device-side types of the MP-PCA denoiser kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lrd {

// Largest frame count the compiled kernels take (register/shared tiles are
// sized from it). The problem family spans T in 32..96.
constexpr int kMaxT = 128;

// Per-axis patch-index tables, device pointers (built by the plan).
//  corners[a][i]          corner position of axis-a index i (sorted, common.py:40-43)
//  cover[a][2*x+{0,1}]    inclusive corner-index range [lo, hi] covering voxel x
//  brick[a][2*b+{0,1}]    inclusive corner-index range touching recon brick b
struct AxisTables {
  const int32_t* corners[3];
  const int32_t* cover[3];
  const int32_t* brick[3];
};

struct Geom {
  int nx, ny, nz, nt;      // volume
  int px, py, pz;          // patch
  int ncx, ncy, ncz;       // corners per axis
  long long npatch;        // ncx*ncy*ncz
  int nvox_patch;          // px*py*pz
  int bx, by, bz;          // recon brick (voxels per axis)
  int nbx, nby, nbz;       // bricks per axis
};

// Patch linear index (x-major, common.py:37-44 itertools.product order) ->
// axis corner indices.
__device__ __forceinline__ void patch_axes(const Geom& g, long long p, int& i, int& j, int& k) {
  k = (int)(p % g.ncz);
  long long r = p / g.ncz;
  j = (int)(r % g.ncy);
  i = (int)(r / g.ncy);
}

__device__ __forceinline__ long long voxel_row(const Geom& g, int x, int y, int z) {
  return ((long long)x * g.ny + y) * g.nz + z;
}

}  // namespace lrd
