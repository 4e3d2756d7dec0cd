// Per-patch Gram matrix G = Xc^T Xc (T x T, K = voxels of the patch).
//
// Role of the ladder's gram_kernel (step8_tuned.py:32-56; math of
// step4_gram_eigh.py:62-64): every accumulated term is already centred (never
// the C X^T X C shortcut, step7_triton_fused.py:20-25). The centred volume
// comes from center_kernel, so the patch's rows are read as-is.
//
// Layout: one CTA per patch. The patch is walked one x-plane at a time
// (py*pz voxel rows of T floats; each of the py runs is pz*T contiguous floats
// in the volume) staged in shared memory. Thread (bi, bj), bi <= bj, owns the
// 4x4 block G[4bi:4bi+4, 4bj:4bj+4] (upper block triangle, the lower half is
// written by symmetry). Each plane's 4x4 partial sums are accumulated in
// float32 and then added into float64 accumulators, so the K = px*py*pz sum
// rounds like a two-level blocked sum (plane of py*pz terms, then px planes).
#pragma once

#include "lrd_common.cuh"

namespace lrd {

// grid: (n patches in this launch); block: nb*(nb+1)/2 threads, nb = ceil(T/4)
// dynamic smem: py*pz*(4*nb) floats.
__global__ void gram_kernel(const float* __restrict__ xc, float* __restrict__ gram, Geom g,
                            AxisTables tab, long long patch0) {
  extern __shared__ float4 smem_gram4[];
  float* plane = reinterpret_cast<float*>(smem_gram4);
  const long long p = patch0 + blockIdx.x;
  int ci, cj, ck;
  patch_axes(g, p, ci, cj, ck);
  const int cx = tab.corners[0][ci], cy = tab.corners[1][cj], cz = tab.corners[2][ck];
  const int T = g.nt;
  const int nb = (T + 3) >> 2;
  const int ld = nb * 4;
  const int tid = threadIdx.x;
  const int ntile = nb * (nb + 1) / 2;

  // tid -> (bi, bj) in row-major order over the upper block triangle
  int bi = 0, bj = 0;
  {
    int rem = tid;
    while (bi < nb && rem >= nb - bi) {
      rem -= nb - bi;
      ++bi;
    }
    bj = bi + rem;
  }
  const bool active = tid < ntile;

  double acc64[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) acc64[u] = 0.0;

  const int rows = g.py * g.pz;
  const int runlen = g.pz * T;  // contiguous floats per (x, y) run
  for (int a = 0; a < g.px; ++a) {
    __syncthreads();
    // stage plane x = cx + a: rows (yy, zz) -> smem row yy*pz + zz, padded to ld
    for (int yy = 0; yy < g.py; ++yy) {
      const float* src = xc + voxel_row(g, cx + a, cy + yy, cz) * T;
      float* dst = plane + (size_t)yy * g.pz * ld;
      if (ld == T) {
        for (int e = tid; e < runlen; e += blockDim.x) dst[e] = src[e];
      } else {
        for (int e = tid; e < g.pz * ld; e += blockDim.x) {
          const int zz = e / ld, t = e - zz * ld;
          dst[e] = t < T ? src[zz * T + t] : 0.f;
        }
      }
    }
    __syncthreads();
    if (active) {
      float acc[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) acc[u] = 0.f;
      const float4* rowp = reinterpret_cast<const float4*>(plane);
      const int ld4 = ld >> 2;
      for (int r = 0; r < rows; ++r) {
        const float4 va = rowp[r * ld4 + bi];
        const float4 vb = rowp[r * ld4 + bj];
        const float a4[4] = {va.x, va.y, va.z, va.w};
        const float b4[4] = {vb.x, vb.y, vb.z, vb.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u * 4 + v] = fmaf(a4[u], b4[v], acc[u * 4 + v]);
      }
#pragma unroll
      for (int u = 0; u < 16; ++u) acc64[u] += (double)acc[u];
    }
  }
  if (!active) return;
  float* G = gram + (size_t)(p - patch0) * T * T;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int r = bi * 4 + u, c = bj * 4 + v;
      if (r < T && c < T) {
        const float val = (float)acc64[u * 4 + v];
        G[(size_t)r * T + c] = val;
        G[(size_t)c * T + r] = val;
      }
    }
  }
}

}  // namespace lrd
