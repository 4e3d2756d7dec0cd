// Temporal mean and centring of every voxel's time course.
//
// The ladder centres each patch's Casorati matrix with NumPy's float32 mean
// (step0_numpy_loop.py:11, ``x.mean(axis=1)``); the mean depends on the voxel
// only, so it is computed once per voxel here (step8_tuned.py:50-52 recompute
// it per patch). The sum follows NumPy's pairwise float32 summation for a
// contiguous row of n <= 128 values (8 interleaved partial sums over the
// largest multiple of 8, combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), the
// tail added in order; n < 8 summed in order from 0), added to the reduction's
// identity 0, then divided by n in float32 - bit-identical to ``x.mean``.
// The centred value is the float32 difference ``x - m`` (step0:12).
#pragma once

#include "lrd_common.cuh"

namespace lrd {

__device__ __forceinline__ float np_pairwise_sum_row(const float* row, int n) {
  float s;
  if (n < 8) {
    s = 0.f;
    for (int i = 0; i < n; ++i) s = __fadd_rn(s, row[i]);
    return s;
  }
  float r0 = row[0], r1 = row[1], r2 = row[2], r3 = row[3];
  float r4 = row[4], r5 = row[5], r6 = row[6], r7 = row[7];
  const int lim = n - (n % 8);
  int i = 8;
  for (; i < lim; i += 8) {
    r0 = __fadd_rn(r0, row[i + 0]);
    r1 = __fadd_rn(r1, row[i + 1]);
    r2 = __fadd_rn(r2, row[i + 2]);
    r3 = __fadd_rn(r3, row[i + 3]);
    r4 = __fadd_rn(r4, row[i + 4]);
    r5 = __fadd_rn(r5, row[i + 5]);
    r6 = __fadd_rn(r6, row[i + 6]);
    r7 = __fadd_rn(r7, row[i + 7]);
  }
  s = __fadd_rn(__fadd_rn(__fadd_rn(r0, r1), __fadd_rn(r2, r3)),
                __fadd_rn(__fadd_rn(r4, r5), __fadd_rn(r6, r7)));
  for (; i < n; ++i) s = __fadd_rn(s, row[i]);
  return __fadd_rn(0.f, s);
}

// One warp stages 32 consecutive voxel rows (32*T floats, contiguous in the
// volume) through shared memory so the global loads and stores are
// coalesced; each lane then reduces one row.
// grid: ceil(nvox / (32 * warps_per_block)) blocks of 32*warps_per_block threads,
// dynamic smem: warps_per_block * (32 * (T + 1) + 32) floats.
// Body of one block (index ``bid``); shared by the single-volume kernel below
// and the packed multi-volume launch (batch.cuh).
__device__ __forceinline__ void center_body(const float* __restrict__ vol, float* __restrict__ xc,
                                            float* __restrict__ mean, long long nvox, int T, long long bid) {
  extern __shared__ float smem_center[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int ld = T + 1;  // odd stride: lane-per-row reads are conflict-free
  float* s = smem_center + (size_t)warp * (32 * ld + 32);
  float* s_mean = s + 32 * ld;
  const long long v0 = (bid * (blockDim.x >> 5) + warp) * 32;
  if (v0 >= nvox) return;  // whole warp leaves; no block-level barrier below
  const int nrows = (int)min(32LL, nvox - v0);
  const int nval = nrows * T;
  // flat element e = r*T + t, stepped by 32 without a division per step
  const int dq = 32 / T, dr = 32 - (32 / T) * T;
  const float* src = vol + v0 * T;
  {
    int r = lane / T, t = lane - (lane / T) * T;
    for (int e = lane; e < nval; e += 32) {
      s[r * ld + t] = src[e];
      t += dr;
      r += dq;
      if (t >= T) { t -= T; ++r; }
    }
  }
  __syncwarp();
  if (lane < nrows) {
    const float m = __fdiv_rn(np_pairwise_sum_row(s + lane * ld, T), (float)T);
    mean[v0 + lane] = m;
    s_mean[lane] = m;
  }
  __syncwarp();
  float* dst = xc + v0 * T;
  {
    int r = lane / T, t = lane - (lane / T) * T;
    for (int e = lane; e < nval; e += 32) {
      dst[e] = __fsub_rn(s[r * ld + t], s_mean[r]);
      t += dr;
      r += dq;
      if (t >= T) { t -= T; ++r; }
    }
  }
}

__global__ void center_kernel(const float* __restrict__ vol, float* __restrict__ xc,
                              float* __restrict__ mean, long long nvox, int T) {
  center_body(vol, xc, mean, nvox, T, blockIdx.x);
}

}  // namespace lrd
