// Reconstruction + weighted overlap accumulation + normalisation, fused.
//
// Role of the ladder's recon_scatter_kernel (step8_tuned.py:59-86) and the
// final division (step8:144-145), with the arithmetic of the step-0 loop
// (step0_numpy_loop.py:25, 36-39):
//
//   xd   = float32((x - m) V_p V_p^T) + m             (per voxel, per patch)
//   out += float32(w) * xd,  wsum += float32(w)       (float32, patch order)
//   out  = out / max(wsum, 1e-12)
//
// Instead of atomically scattering each patch into the volume (order-free,
// non-deterministic), every output voxel is owned by one thread group that
// gathers its covering patches itself, in the ladder's x-major patch order.
// The result is deterministic and rounds like the step-0 loop, which adds the
// patches to each voxel in exactly that order.
//
// Layout: one CTA per brick of bx*by*bz voxels, 4 threads per voxel (thread
// ``s`` of a voxel owns frames t = s, s+4, s+8, ...). The CTA walks every patch
// touching the brick in x-major order; the patch's eigenvector block V_p
// (T x p, compact) is staged in shared memory; each thread computes its
// partial y = (x - m)_slice . V_p, the 4 partials of a voxel are combined with
// two shuffles, then xd = y V_p^T + m for its frames; a voxel the patch does
// not cover skips the accumulation. Coverage is separable: per axis the
// covering corner indices of a voxel form one contiguous range.
//
// Form ACCURATE keeps the temporal mean out of the running sums: it
// accumulates w * (x - m) V_p V_p^T with a compensated (two-sum) float32
// accumulator and the weights in float64, then writes m + acc / wsum.
#pragma once

#include "lrd_common.cuh"

namespace lrd {

constexpr int kReconSplit = 4;  // threads per voxel

__device__ __forceinline__ void two_sum_acc(float& acc, float& comp, float x) {
  const float s = __fadd_rn(acc, x);
  const float bp = __fsub_rn(s, acc);
  const float err = __fadd_rn(__fsub_rn(acc, __fsub_rn(s, bp)), __fsub_rn(x, bp));
  comp = __fadd_rn(comp, err);
  acc = s;
}

// grid: nbx*nby*nbz blocks of bx*by*bz*4 threads (<= 1024).
// dynamic smem: T * (T | 1) floats (V tile, row stride p|1).
template <int TPT, bool ACCURATE>
__global__ void recon_kernel(const float* __restrict__ xc, const float* __restrict__ mean,
                             const float* __restrict__ vecs, const int32_t* __restrict__ ranks,
                             const float* __restrict__ wgt, float* __restrict__ out, Geom g,
                             AxisTables tab) {
  extern __shared__ float sV[];
  __shared__ int s_p;
  __shared__ float s_w;
  const int T = g.nt;
  const int tid = threadIdx.x;
  const int slice = tid & (kReconSplit - 1);
  const int vl = tid / kReconSplit;

  int brick = blockIdx.x;
  const int bzi = brick % g.nbz;
  brick /= g.nbz;
  const int byi = brick % g.nby;
  const int bxi = brick / g.nby;

  const int bvox = g.bx * g.by * g.bz;
  const int lz = vl % g.bz, ly = (vl / g.bz) % g.by, lx = vl / (g.by * g.bz);
  const int x = bxi * g.bx + lx, y = byi * g.by + ly, z = bzi * g.bz + lz;
  const bool valid = vl < bvox && x < g.nx && y < g.ny && z < g.nz;

  int cxlo = 1, cxhi = 0, cylo = 1, cyhi = 0, czlo = 1, czhi = 0;
  long long row = 0;
  if (valid) {
    cxlo = tab.cover[0][2 * x];
    cxhi = tab.cover[0][2 * x + 1];
    cylo = tab.cover[1][2 * y];
    cyhi = tab.cover[1][2 * y + 1];
    czlo = tab.cover[2][2 * z];
    czhi = tab.cover[2][2 * z + 1];
    row = voxel_row(g, x, y, z);
  }
  const int ilo = tab.brick[0][2 * bxi], ihi = tab.brick[0][2 * bxi + 1];
  const int jlo = tab.brick[1][2 * byi], jhi = tab.brick[1][2 * byi + 1];
  const int klo = tab.brick[2][2 * bzi], khi = tab.brick[2][2 * bzi + 1];

  float xr[TPT], acc[TPT], comp[TPT];
  float m = 0.f;
#pragma unroll
  for (int u = 0; u < TPT; ++u) {
    const int t = u * kReconSplit + slice;
    xr[u] = (valid && t < T) ? xc[row * T + t] : 0.f;
    acc[u] = 0.f;
    comp[u] = 0.f;
  }
  if (valid) m = mean[row];
  float wacc = 0.f;
  double wacc64 = 0.0;

  for (int i = ilo; i <= ihi; ++i) {
    for (int j = jlo; j <= jhi; ++j) {
      for (int k = klo; k <= khi; ++k) {
        const long long pid = ((long long)i * g.ncy + j) * g.ncz + k;
        __syncthreads();
        if (tid == 0) {
          s_p = ranks[pid];
          s_w = wgt[pid];
        }
        __syncthreads();
        const int p = s_p;
        const float w = s_w;
        const int ldv = p | 1;
        {
          const float* src = vecs + pid * (long long)T * T;
          const int nv = T * p;
          for (int e = tid; e < nv; e += blockDim.x) {
            const int r = e / p, c = e - r * p;
            sV[r * ldv + c] = src[e];
          }
        }
        __syncthreads();
        const bool cov = valid && i >= cxlo && i <= cxhi && j >= cylo && j <= cyhi && k >= czlo &&
                         k <= czhi;
        float xdp[TPT];
#pragma unroll
        for (int u = 0; u < TPT; ++u) xdp[u] = 0.f;
        for (int kk = 0; kk < p; ++kk) {
          float part = 0.f;
#pragma unroll
          for (int u = 0; u < TPT; ++u) {
            const int t = u * kReconSplit + slice;
            if (t < T) part = fmaf(xr[u], sV[t * ldv + kk], part);
          }
          part += __shfl_xor_sync(0xffffffffu, part, 1);
          part += __shfl_xor_sync(0xffffffffu, part, 2);
#pragma unroll
          for (int u = 0; u < TPT; ++u) {
            const int t = u * kReconSplit + slice;
            if (t < T) xdp[u] = fmaf(part, sV[t * ldv + kk], xdp[u]);
          }
        }
        if (cov) {
          if (ACCURATE) {
#pragma unroll
            for (int u = 0; u < TPT; ++u) two_sum_acc(acc[u], comp[u], __fmul_rn(w, xdp[u]));
            wacc64 += (double)w;
          } else {
#pragma unroll
            for (int u = 0; u < TPT; ++u) {
              const float xd = __fadd_rn(xdp[u], m);
              acc[u] = __fadd_rn(acc[u], __fmul_rn(w, xd));
            }
            wacc = __fadd_rn(wacc, w);
          }
        }
      }
    }
  }
  if (!valid) return;
  if (ACCURATE) {
    // a voxel no patch covers (stride > patch side) gets 0, as 0 / max(0, 1e-12)
    // does in the ladder
    const double inv = wacc64 > 0.0 ? 1.0 / wacc64 : 0.0;
    const double mm = wacc64 > 0.0 ? (double)m : 0.0;
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int t = u * kReconSplit + slice;
      if (t < T) out[row * T + t] = (float)(mm + ((double)acc[u] + (double)comp[u]) * inv);
    }
  } else {
    const float den = fmaxf(wacc, 1e-12f);
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int t = u * kReconSplit + slice;
      if (t < T) out[row * T + t] = __fdiv_rn(acc[u], den);
    }
  }
}

}  // namespace lrd
