// Reconstruction + weighted overlap accumulation + normalisation with one
// warp per 2x2x2 block of voxels and no block-level synchronisation.
//
// Same role and the same per-voxel arithmetic as recon_kernel (recon.cuh):
// the ladder's recon_scatter_kernel (step8_tuned.py:59-86) and final division
// (step8:144-145) with the step-0 loop's rounding (step0_numpy_loop.py:25,
// 36-39):
//
//   y_k  = (x - m) . v_k             four frame chunks, ((c0 + c1) + (c2 + c3))
//   xd   = float32(sum_k y_k v_k) + m
//   out += float32(w) * xd,  wsum += float32(w)   (float32, x-major patch order)
//   out  = out / max(wsum, 1e-12)
//
// so its output is bit-identical to recon_kernel's for every form. What
// changes is the work decomposition, for T = 4Q frames with Q a multiple of
// four (T = 32, 48, 64, 96 here):
//
//  * a warp owns the 8 voxels of a 2x2x2 block, four lanes per voxel, lane s
//    of a voxel owning frame chunk [sQ, sQ + Q) - exactly the chunk tree of
//    the y_k sum, so a voxel's y_k is its four lanes' chunk sums combined by
//    two shuffles;
//  * the warp walks the union of its voxels' covering patches in x-major
//    order on its own (per axis the union of two adjacent cover ranges);
//    nothing is staged through shared memory and no barrier is taken: the
//    eigenvector rows are read with read-only cached loads (every lane of a
//    voxel group reads the same 16 bytes, and the warps of an SM walk
//    overlapping patch lists, so they hit L1) and a lane's three float4 of
//    v_k are reused for the expansion xd += y_k v_k;
//  * everything that depends on T is compile-time (frames per lane, the
//    row stride of the eigenvector block): no frame guards, no runtime
//    division in the walk.
//
// A CTA is kReconWarps warps stacked along z: a brick of 2 x 2 x (2 *
// kReconWarps) voxels in the plan's brick grid, so the host pipeline and
// slab sharding address it exactly like recon_kernel's bricks.
#pragma once

#include "lrd_common.cuh"
#include "recon.cuh"

namespace lrd {

constexpr int kReconWarps = 4;

// Brick of the warp kernel along z (x and y are 2).
__host__ __device__ constexpr int recon_warp_bz() { return 2 * kReconWarps; }

// Frame counts the warp kernel is built for: T = 4Q, Q in {8, 12, 16, 24}.
__host__ __device__ inline bool recon_warp_supported(int T) { return T == 32 || T == 48 || T == 64 || T == 96; }

// Body of one CTA: brick brick0 + bid of the plan's brick grid.
template <int Q, bool ACCURATE>
__device__ __forceinline__ void recon_warp_body(const float* __restrict__ xc, const float* __restrict__ mean,
                                                const float* __restrict__ vecs, const int32_t* __restrict__ ranks,
                                                const float* __restrict__ wgt, float* __restrict__ out,
                                                const Geom& g, const AxisTables& tab, int brick0, const SlabIO& io,
                                                int bid) {
  constexpr int T = 4 * Q;
  constexpr int Q4 = Q / 4;  // float4 per lane
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int s = lane & 3;    // frame chunk of this lane
  const int vl = lane >> 2;  // voxel of the 2x2x2 block: (x, y, z) offsets (vl >> 2, (vl >> 1) & 1, vl & 1)

  int brick = brick0 + bid;
  const int bzi = brick % g.nbz;
  brick /= g.nbz;
  const int byi = brick % g.nby;
  const int bxi = brick / g.nby;
  const int x = bxi * 2 + (vl >> 2), y = byi * 2 + ((vl >> 1) & 1);
  const int z = bzi * g.bz + warp * 2 + (vl & 1);
  const bool valid = x < g.nx && y < g.ny && z < g.nz && x >= io.x_lo && x < io.x_hi;

  // this voxel's covering corner ranges; the warp's walk is their union
  int cxlo = 1 << 30, cxhi = -1, cylo = 1 << 30, cyhi = -1, czlo = 1 << 30, czhi = -1;
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
  int ilo = cxlo, ihi = cxhi, jlo = cylo, jhi = cyhi, klo = czlo, khi = czhi;
#pragma unroll
  for (int o = 4; o < 32; o <<= 1) {  // lanes of one voxel hold the same ranges
    ilo = min(ilo, __shfl_xor_sync(0xffffffffu, ilo, o));
    ihi = max(ihi, __shfl_xor_sync(0xffffffffu, ihi, o));
    jlo = min(jlo, __shfl_xor_sync(0xffffffffu, jlo, o));
    jhi = max(jhi, __shfl_xor_sync(0xffffffffu, jhi, o));
    klo = min(klo, __shfl_xor_sync(0xffffffffu, klo, o));
    khi = max(khi, __shfl_xor_sync(0xffffffffu, khi, o));
  }
  if (!__any_sync(0xffffffffu, valid)) return;  // warp-uniform: no voxel of this block is computed

  // centred frames of this lane's chunk, temporal mean, running sums
  float xr[Q];
  const float4* xp = reinterpret_cast<const float4*>(xc + row * T + s * Q);
#pragma unroll
  for (int u4 = 0; u4 < Q4; ++u4) {
    const float4 v = valid ? xp[u4] : make_float4(0.f, 0.f, 0.f, 0.f);
    xr[4 * u4 + 0] = v.x;
    xr[4 * u4 + 1] = v.y;
    xr[4 * u4 + 2] = v.z;
    xr[4 * u4 + 3] = v.w;
  }
  const float m = valid ? mean[row] : 0.f;
  float acc[ACCURATE ? 1 : Q];
  double acc64[ACCURATE ? Q : 1];
#pragma unroll
  for (int u = 0; u < Q; ++u) {
    if constexpr (ACCURATE)
      acc64[u] = 0.0;
    else
      acc[u] = 0.f;
  }
  float wacc = 0.f;
  double wacc64 = 0.0;
  if (valid && x < io.hin && io.halo_in != nullptr) {  // continue a lower slab's sums
    const double* hp = io.halo_in + row * (T + 1);
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      if constexpr (ACCURATE)
        acc64[u] = hp[s * Q + u];
      else
        acc[u] = (float)hp[s * Q + u];
    }
    wacc64 = hp[T];
    wacc = (float)hp[T];
  }

  constexpr long long TT = (long long)T * T;
  for (int i = ilo; i <= ihi; ++i) {
    const bool cx = i >= cxlo && i <= cxhi;
    for (int j = jlo; j <= jhi; ++j) {
      const bool cxy = cx && j >= cylo && j <= cyhi;
      long long pid = ((long long)i * g.ncy + j) * g.ncz + klo;
      for (int k = klo; k <= khi; ++k, ++pid) {
        const int p = __ldg(ranks + pid);
        const float w = __ldg(wgt + pid);
        const bool cov = valid && cxy && k >= czlo && k <= czhi;
        const float4* vb = reinterpret_cast<const float4*>(vecs + pid * TT) + s * Q4;
        float xdp[Q];
#pragma unroll
        for (int u = 0; u < Q; ++u) xdp[u] = 0.f;
#pragma unroll 2
        for (int kk = 0; kk < p; ++kk) {
          float4 q[Q4];
#pragma unroll
          for (int u4 = 0; u4 < Q4; ++u4) q[u4] = __ldg(vb + kk * (T / 4) + u4);
          float part = 0.f;  // this lane's chunk of y_k, frames in order
#pragma unroll
          for (int u4 = 0; u4 < Q4; ++u4) {
            part = fmaf(xr[4 * u4 + 0], q[u4].x, part);
            part = fmaf(xr[4 * u4 + 1], q[u4].y, part);
            part = fmaf(xr[4 * u4 + 2], q[u4].z, part);
            part = fmaf(xr[4 * u4 + 3], q[u4].w, part);
          }
          part = __fadd_rn(part, __shfl_xor_sync(0xffffffffu, part, 1));
          part = __fadd_rn(part, __shfl_xor_sync(0xffffffffu, part, 2));
#pragma unroll
          for (int u4 = 0; u4 < Q4; ++u4) {
            xdp[4 * u4 + 0] = fmaf(part, q[u4].x, xdp[4 * u4 + 0]);
            xdp[4 * u4 + 1] = fmaf(part, q[u4].y, xdp[4 * u4 + 1]);
            xdp[4 * u4 + 2] = fmaf(part, q[u4].z, xdp[4 * u4 + 2]);
            xdp[4 * u4 + 3] = fmaf(part, q[u4].w, xdp[4 * u4 + 3]);
          }
        }
        if (cov) {
          if constexpr (ACCURATE) {
            const double wd = (double)w;
#pragma unroll
            for (int u = 0; u < Q; ++u) acc64[u] = fma(wd, (double)xdp[u], acc64[u]);
            wacc64 += wd;
          } else {
#pragma unroll
            for (int u = 0; u < Q; ++u) acc[u] = __fadd_rn(acc[u], __fmul_rn(w, __fadd_rn(xdp[u], m)));
            wacc = __fadd_rn(wacc, w);
          }
        }
      }
    }
  }
  if (!valid) return;
  if (x >= io.own_hi) {  // the next slab's halo: unnormalised sums in patch order
    double* hp = io.halo_out + (row - (long long)io.own_hi * g.ny * g.nz) * (T + 1);
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      if constexpr (ACCURATE)
        hp[s * Q + u] = acc64[u];
      else
        hp[s * Q + u] = (double)acc[u];
    }
    if (s == 0) hp[T] = ACCURATE ? wacc64 : (double)wacc;
    return;
  }
  float4* op = reinterpret_cast<float4*>(out + row * T + s * Q);
  if constexpr (ACCURATE) {
    // a voxel no patch covers (stride > patch side) gets 0, as 0 / max(0, 1e-12)
    // does in the ladder
    const double inv = wacc64 > 0.0 ? 1.0 / wacc64 : 0.0;
    const double mm = wacc64 > 0.0 ? (double)m : 0.0;
#pragma unroll
    for (int u4 = 0; u4 < Q4; ++u4)
      op[u4] = make_float4((float)(mm + acc64[4 * u4 + 0] * inv), (float)(mm + acc64[4 * u4 + 1] * inv),
                           (float)(mm + acc64[4 * u4 + 2] * inv), (float)(mm + acc64[4 * u4 + 3] * inv));
  } else {
    const float den = fmaxf(wacc, 1e-12f);
#pragma unroll
    for (int u4 = 0; u4 < Q4; ++u4)
      op[u4] = make_float4(__fdiv_rn(acc[4 * u4 + 0], den), __fdiv_rn(acc[4 * u4 + 1], den),
                           __fdiv_rn(acc[4 * u4 + 2], den), __fdiv_rn(acc[4 * u4 + 3], den));
  }
}

template <int Q, bool ACCURATE>
__global__ void __launch_bounds__(32 * kReconWarps)
    recon_warp_kernel(const float* __restrict__ xc, const float* __restrict__ mean, const float* __restrict__ vecs,
                      const int32_t* __restrict__ ranks, const float* __restrict__ wgt, float* __restrict__ out,
                      Geom g, AxisTables tab, int brick0, SlabIO io) {
  recon_warp_body<Q, ACCURATE>(xc, mean, vecs, ranks, wgt, out, g, tab, brick0, io, (int)blockIdx.x);
}

}  // namespace lrd
