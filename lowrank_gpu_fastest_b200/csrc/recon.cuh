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
// Layout: one CTA per brick of bx*by*bz voxels, SPLIT threads per voxel
// (1, 2 or 4; thread ``s`` of a voxel owns the contiguous frames
// [s*TPT, s*TPT + TPT) ∩ [0, T)).
// The ranks and weights of every patch touching the brick are loaded once;
// the CTA then walks those patches in x-major order with the eigenvector
// block V_p (p x T, k-major, rows padded to a multiple of 4 floats) of the
// next patch streamed into the other half of a shared-memory double buffer by
// cp.async while the current one is used. Each thread computes its partial
// y_k = (x - m)_slice . v_k from float4 reads of v_k, the 4 partials of a voxel
// are combined with two shuffles, then xd = y V_p^T + m for its frames; a
// voxel the patch does not cover skips the accumulation. Coverage is
// separable: per axis the covering corner indices of a voxel form one
// contiguous range.
//
// Form ACCURATE keeps the temporal mean out of the running sums: it
// accumulates the exact float64 products w * [(x - m) V_p V_p^T] and the
// weights in float64, then writes m + acc / wsum.
#pragma once

#include "lrd_common.cuh"

namespace lrd {

constexpr int kReconSplit = 4;  // largest number of threads per voxel

__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async16(float* smem_dst, const float* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__host__ __device__ inline int recon_tp(int T) { return (T + 3) & ~3; }

// Dynamic shared memory bytes: two V buffers of T rows x recon_tp(T) floats,
// then ranks (int) and weights (float) of up to max_touch patches.
__host__ __device__ inline size_t recon_smem_bytes(int T, int max_touch) {
  return sizeof(float) * 2 * (size_t)T * recon_tp(T) + (sizeof(int) + sizeof(float)) * (size_t)max_touch;
}

// Slab sharding of one volume over GPUs (x-slabs of patch corners): which
// voxels a launch computes, and the partial sums handed between neighbours.
// A voxel's patches are accumulated in x-major order, so a lower slab's
// partial (sum and weight of its patches, in order) followed by this slab's
// patches is exactly the single-GPU sequence.
struct SlabIO {
  int x_lo, x_hi;         // voxels with x in [x_lo, x_hi) are computed
  int hin;                // planes [0, hin) start from halo_in (nullable)
  const double* halo_in;  // (hin, ny, nz, T + 1): T sums then the weight sum
  int own_hi;             // planes >= own_hi go to halo_out unnormalised
  double* halo_out;       // (nx - own_hi, ny, nz, T + 1)
};

// grid: bricks [brick0, brick0 + gridDim.x) of the nbx*nby*nbz (x-major)
// bricks; bx*by*bz*SPLIT threads per block (<= 1024).
template <int TPT, int SPLIT, bool ACCURATE>
__device__ __forceinline__ void recon_body(const float* __restrict__ xc, const float* __restrict__ mean,
                                           const float* __restrict__ vecs, const int32_t* __restrict__ ranks,
                                           const float* __restrict__ wgt, float* __restrict__ out, Geom g,
                                           AxisTables tab, int brick0, SlabIO io) {
  extern __shared__ __align__(16) float sm_recon[];
  const int T = g.nt;
  const int TP = recon_tp(T);
  float* vbuf0 = sm_recon;
  float* vbuf1 = sm_recon + (size_t)T * TP;
  int* s_rank = reinterpret_cast<int*>(sm_recon + 2 * (size_t)T * TP);
  const int tid = threadIdx.x;
  const int nthreads = blockDim.x;
  const int slice = tid & (SPLIT - 1);
  const int vl = tid / SPLIT;
  const int t0 = slice * TPT;

  int brick = brick0 + blockIdx.x;
  const int bzi = brick % g.nbz;
  brick /= g.nbz;
  const int byi = brick % g.nby;
  const int bxi = brick / g.nby;

  const int bvox = g.bx * g.by * g.bz;
  const int lz = vl % g.bz, ly = (vl / g.bz) % g.by, lx = vl / (g.by * g.bz);
  const int x = bxi * g.bx + lx, y = byi * g.by + ly, z = bzi * g.bz + lz;
  const bool valid = vl < bvox && x < g.nx && y < g.ny && z < g.nz && x >= io.x_lo && x < io.x_hi;

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
  const int ni = max(0, ihi - ilo + 1), nj = max(0, jhi - jlo + 1), nk = max(0, khi - klo + 1);
  const int np = ni * nj * nk;
  float* s_w = reinterpret_cast<float*>(s_rank + np);

  // ranks and weights of the touching patches, x-major order
  for (int e = tid; e < np; e += nthreads) {
    const int kk = e % nk, r = e / nk;
    const int jj = r % nj, ii = r / nj;
    const long long pid = ((long long)(ilo + ii) * g.ncy + (jlo + jj)) * g.ncz + (klo + kk);
    s_rank[e] = ranks[pid];
    s_w[e] = wgt[pid];
  }
  // zero the row padding of both buffers (never written by the copies)
  if (TP != T)
    for (int e = tid; e < 2 * T * (TP - T); e += nthreads) {
      const int r = e / (TP - T), c = T + e % (TP - T);
      sm_recon[(size_t)r * TP + c] = 0.f;
    }

  float xr[TPT], acc[ACCURATE ? 1 : TPT];
  double acc64[ACCURATE ? TPT : 1];
  float m = 0.f;
#pragma unroll
  for (int u = 0; u < TPT; ++u) {
    const int t = t0 + u;
    xr[u] = (valid && t < T) ? xc[row * T + t] : 0.f;
    if constexpr (ACCURATE)
      acc64[u] = 0.0;
    else
      acc[u] = 0.f;
  }
  if (valid) m = mean[row];
  float wacc = 0.f;
  double wacc64 = 0.0;
  if (valid && x < io.hin && io.halo_in != nullptr) {  // continue a lower slab's sums
    const double* hp = io.halo_in + row * (T + 1);
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int t = t0 + u;
      if (t < T) {
        if constexpr (ACCURATE)
          acc64[u] = hp[t];
        else
          acc[u] = (float)hp[t];
      }
    }
    wacc64 = hp[T];
    wacc = (float)hp[T];
  }
  __syncthreads();

  const bool vec16 = (T & 3) == 0;
  auto issue = [&](int kp, float* buf) {
    const int kk = kp % nk, r = kp / nk;
    const int jj = r % nj, ii = r / nj;
    const long long pid = ((long long)(ilo + ii) * g.ncy + (jlo + jj)) * g.ncz + (klo + kk);
    const int p = s_rank[kp];
    const float* src = vecs + pid * (long long)T * T;
    if (vec16) {
      const int n4 = (T * p) >> 2;  // rows of T floats, T % 4 == 0, TP == T
      for (int e = tid; e < n4; e += nthreads) cp_async16(buf + 4 * e, src + 4 * e);
    } else {
      const int nv = T * p;
      for (int e = tid; e < nv; e += nthreads) {
        const int k = e / T, t = e - k * T;
        cp_async4(buf + (size_t)k * TP + t, src + e);
      }
    }
  };

  if (np > 0) issue(0, vbuf0);
  cp_async_commit();
  int ci = 0, cj = 0, ck = 0;  // axis offsets of patch kp within the brick's ranges
  for (int kp = 0; kp < np; ++kp) {
    if (kp + 1 < np) issue(kp + 1, ((kp + 1) & 1) ? vbuf1 : vbuf0);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const float* vb = (kp & 1) ? vbuf1 : vbuf0;
    const int p = s_rank[kp];
    const float w = s_w[kp];
    const int i = ilo + ci, j = jlo + cj, k = klo + ck;
    const bool cov = valid && i >= cxlo && i <= cxhi && j >= cylo && j <= cyhi && k >= czlo && k <= czhi;
    float xdp[TPT];
#pragma unroll
    for (int u = 0; u < TPT; ++u) xdp[u] = 0.f;
    for (int kk = 0; kk < p; ++kk) {
      // v_k is read twice from shared memory rather than held in TPT registers.
      // y_k = (x - m) . v_k is summed as four fixed frame chunks of TPT*SPLIT/4
      // frames, combined ((c0 + c1) + (c2 + c3)), for every SPLIT, so the
      // result does not depend on the thread layout.
      const float4* vr = reinterpret_cast<const float4*>(vb + (size_t)kk * TP + t0);
      constexpr int CH = 4 / SPLIT;         // chunks per thread
      constexpr int CU4 = TPT / 4 / CH;     // float4 groups per chunk
      float cp[CH];
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        float acc_c = 0.f;
#pragma unroll
        for (int u4 = c * CU4; u4 < (c + 1) * CU4; ++u4) {
          if (t0 + 4 * u4 < TP) {
            const float4 q = vr[u4];
            acc_c = fmaf(xr[4 * u4 + 0], q.x, acc_c);
            acc_c = fmaf(xr[4 * u4 + 1], q.y, acc_c);
            acc_c = fmaf(xr[4 * u4 + 2], q.z, acc_c);
            acc_c = fmaf(xr[4 * u4 + 3], q.w, acc_c);
          }
        }
        cp[c] = acc_c;
      }
      float part;
      if (CH == 4)
        part = __fadd_rn(__fadd_rn(cp[0], cp[CH > 1 ? 1 : 0]), __fadd_rn(cp[CH > 2 ? 2 : 0], cp[CH > 3 ? 3 : 0]));
      else if (CH == 2)
        part = __fadd_rn(cp[0], cp[CH > 1 ? 1 : 0]);
      else
        part = cp[0];
      if (SPLIT >= 2) part = __fadd_rn(part, __shfl_xor_sync(0xffffffffu, part, 1));
      if (SPLIT >= 4) part = __fadd_rn(part, __shfl_xor_sync(0xffffffffu, part, 2));
#pragma unroll
      for (int u4 = 0; u4 < TPT / 4; ++u4) {
        if (t0 + 4 * u4 < TP) {
          const float4 q = vr[u4];
          xdp[4 * u4 + 0] = fmaf(part, q.x, xdp[4 * u4 + 0]);
          xdp[4 * u4 + 1] = fmaf(part, q.y, xdp[4 * u4 + 1]);
          xdp[4 * u4 + 2] = fmaf(part, q.z, xdp[4 * u4 + 2]);
          xdp[4 * u4 + 3] = fmaf(part, q.w, xdp[4 * u4 + 3]);
        }
      }
    }
    if (cov) {
      if constexpr (ACCURATE) {
        const double wd = (double)w;
#pragma unroll
        for (int u = 0; u < TPT; ++u) acc64[u] = fma(wd, (double)xdp[u], acc64[u]);
        wacc64 += wd;
      } else {
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
          const float xd = __fadd_rn(xdp[u], m);
          acc[u] = __fadd_rn(acc[u], __fmul_rn(w, xd));
        }
        wacc = __fadd_rn(wacc, w);
      }
    }
    if (++ck == nk) {
      ck = 0;
      if (++cj == nj) {
        cj = 0;
        ++ci;
      }
    }
    __syncthreads();
  }
  if (!valid) return;
  if (x >= io.own_hi) {  // the next slab's halo: unnormalised sums in patch order
    double* hp = io.halo_out + (row - (long long)io.own_hi * g.ny * g.nz) * (T + 1);
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int t = t0 + u;
      if (t < T) {
        if constexpr (ACCURATE)
          hp[t] = acc64[u];
        else
          hp[t] = (double)acc[u];
      }
    }
    if (slice == 0) hp[T] = ACCURATE ? wacc64 : (double)wacc;
    return;
  }
  if constexpr (ACCURATE) {
    // a voxel no patch covers (stride > patch side) gets 0, as 0 / max(0, 1e-12)
    // does in the ladder
    const double inv = wacc64 > 0.0 ? 1.0 / wacc64 : 0.0;
    const double mm = wacc64 > 0.0 ? (double)m : 0.0;
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int t = t0 + u;
      if (t < T) out[row * T + t] = (float)(mm + acc64[u] * inv);
    }
  } else {
    const float den = fmaxf(wacc, 1e-12f);
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int t = t0 + u;
      if (t < T) out[row * T + t] = __fdiv_rn(acc[u], den);
    }
  }
}

template <int TPT, int SPLIT, bool ACCURATE>
__global__ void recon_kernel(const float* __restrict__ xc, const float* __restrict__ mean,
                             const float* __restrict__ vecs, const int32_t* __restrict__ ranks,
                             const float* __restrict__ wgt, float* __restrict__ out, Geom g, AxisTables tab,
                             int brick0, SlabIO io) {
  recon_body<TPT, SPLIT, ACCURATE>(xc, mean, vecs, ranks, wgt, out, g, tab, brick0, io);
}

// The T <= 48 float32 layout (24 frames x 2 threads per voxel) with its
// registers capped at 112: 136 by default allow 6 CTAs of 64 threads per SM,
// 112 allow 9 (96x96x48x48 headline: 1.30 -> 1.22 ms; 96 registers spill
// inside the patch loop and took 2.46 ms).
__global__ void __maxnreg__(112) recon_kernel_t24s2(const float* __restrict__ xc, const float* __restrict__ mean,
                                                    const float* __restrict__ vecs,
                                                    const int32_t* __restrict__ ranks,
                                                    const float* __restrict__ wgt, float* __restrict__ out, Geom g,
                                                    AxisTables tab, int brick0, SlabIO io) {
  recon_body<24, 2, false>(xc, mean, vecs, ranks, wgt, out, g, tab, brick0, io);
}

}  // namespace lrd
