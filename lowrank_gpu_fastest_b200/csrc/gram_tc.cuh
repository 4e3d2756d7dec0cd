// Per-patch Gram matrices on the 5th-generation tensor cores (tcgen05).
//
// Same decomposition as gram_z_kernel (one CTA per (x, y) patch column, TMA
// streams the column's z-planes, each plane Gram H(z) is formed once and added
// into the windows it belongs to), but H(z) = X^T X (X = the plane's px*py
// centred voxel rows, T frames) is computed by tcgen05.mma in kind::tf32 with
// the float32 data split as x = hi + lo (hi = tf32(x), lo = tf32(x - hi)) and
//     H = hi^T hi + hi^T lo + lo^T hi        (3xTF32, FP32 accumulation in TMEM)
// which recovers ~22 bits of each product.
//
// MMA shape: M = 64 (rows = frames t; rows >= T are never read back), N = T
// (rounded up to 8), K = 8 voxels per instruction over the plane's voxels
// padded to a multiple of 8. A (M x K) and B (stored as its K-major transpose,
// N x K) are the same shared-memory tile X^T in the canonical K-major,
// no-swizzle layout: 8-row x 16-byte core matrices, LBO = 128 B between core
// matrices along K, SBO = (K/4) * 128 B between 8-row groups.
//
// Each plane's H is accumulated in tensor memory over its own 3 x K/8 MMAs
// only (accumulating whole windows there - ~500 MMA steps - measured a 10x
// larger Gram error: the tensor-core FP32 accumulation does not round to
// nearest), read back with tcgen05.ld (M = 64: rows 16w..16w+15 in lanes
// 32w..32w+15 of warp w's sub-partition) and added in float32 into the
// windows' rows in shared memory; a completed window is written out.
//
// Waits (TMA and MMA completion) are bounded by %globaltimer deadlines; the
// TMEM allocation is released on every path.
#pragma once

#include "gram_z.cuh"

namespace lrd {

constexpr int kStatusMmaTimeout = 2;

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// Shared-memory matrix descriptor: SWIZZLE_NONE, K-major canonical layout.
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t smem_addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: kind::tf32, D = F32, A = B = TF32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory layout (bytes): hi tile (ceil(T/8) row groups of SBO bytes),
// lo tile (same), one plane slot, windows [ring][T cols][T rows] float32,
// mbarriers, TMEM address, abort flag. An A descriptor spans 8 row groups
// from its tile's start (M = 64); rows past T read whatever follows (they
// only feed accumulator rows >= T, never read), so the allocation just has to
// cover lo + 8 groups.
__host__ __device__ inline int gramtc_kpad(int rows) { return (rows + 7) & ~7; }
__host__ __device__ inline size_t gramtc_sbo(int rows) { return (size_t)(gramtc_kpad(rows) / 4) * 128; }
__host__ __device__ inline size_t gramtc_tile_bytes(int rows, int T) { return (size_t)((T + 7) / 8) * gramtc_sbo(rows); }
__host__ __device__ inline size_t gramtc_off_plane(int rows, int T) { return 2 * gramtc_tile_bytes(rows, T); }
__host__ __device__ inline size_t gramtc_smem_bytes(int rows, int T, int ring) {
  const size_t end = gramtc_off_plane(rows, T) +
                     sizeof(float) * (gramz_plane_floats(rows, T) + (size_t)ring * T * T) + 64;
  const size_t span = gramtc_tile_bytes(rows, T) + 8 * gramtc_sbo(rows);
  return end > span ? end : span;
}
__host__ __device__ inline int gramtc_npad(int T) { return (T + 7) & ~7; }
__host__ __device__ inline int gramtc_tmem_cols(int T) { return gramtc_npad(T) <= 32 ? 32 : 64; }

// grid: (columns in this launch); block: 128 threads (4 warps). T <= 64,
// px*py <= 128. ``gram`` points at the Gram block of patch col0 * ncz.
__global__ void __launch_bounds__(128)
    gram_tc_kernel(const __grid_constant__ CUtensorMap xmap, float* __restrict__ gram, Geom g, AxisTables tab,
                   long long col0, int ring, int* status) {
  extern __shared__ __align__(1024) unsigned char smt[];
  const int T = g.nt;
  const int rows = g.px * g.py;
  const int kpad = gramtc_kpad(rows);
  const uint32_t sbo = (uint32_t)gramtc_sbo(rows);  // bytes between 8-row groups
  const size_t tile = gramtc_tile_bytes(rows, T);
  unsigned char* hi = smt;
  unsigned char* lo = smt + tile;
  float* plane = reinterpret_cast<float*>(smt + gramtc_off_plane(rows, T));
  float* win = plane + gramz_plane_floats(rows, T);  // [ring][T cols][T rows]
  uint64_t* bars = reinterpret_cast<uint64_t*>(win + (size_t)ring * T * T);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);  // set when a wait gave up
  const uint32_t bart = (uint32_t)__cvta_generic_to_shared(&bars[0]);
  const uint32_t barm = (uint32_t)__cvta_generic_to_shared(&bars[1]);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;

  const long long col = col0 + blockIdx.x;
  const int ci = (int)(col / g.ncy), cj = (int)(col % g.ncy);
  const int cx = tab.corners[0][ci], cy = tab.corners[1][cj];
  const uint32_t plane_bytes = (uint32_t)(rows * T * sizeof(float));
  const int Npad = gramtc_npad(T);
  const uint32_t idesc = umma_idesc_tf32(64, Npad);
  const uint32_t ncols = (uint32_t)gramtc_tmem_cols(T);
  const int nv4 = (rows + 3) >> 2;

  // zero the operand tiles once (rows >= T and voxels >= rows stay zero) and the windows
  for (size_t e = tid; e < 2 * tile / 16; e += blockDim.x) reinterpret_cast<uint4*>(smt)[e] = make_uint4(0, 0, 0, 0);
  for (int e = tid; e < ring * T * T; e += blockDim.x) win[e] = 0.f;
  if (tid == 0) {
    *abort_flag = 0;
    mbar_init(bart, 1);
    mbar_init(barm, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t hi_addr = (uint32_t)__cvta_generic_to_shared(hi);
  const uint32_t lo_addr = (uint32_t)__cvta_generic_to_shared(lo);
  const uint32_t plane_addr = (uint32_t)__cvta_generic_to_shared(plane);

  if (tid == 0 && g.nz > 0) {
    mbar_expect_tx(bart, plane_bytes);
    tma_load_4d(plane_addr, &xmap, bart, 0, 0, cy, cx);
  }
  float* G0 = gram + (size_t)((col - col0) * g.ncz) * T * T;
  uint32_t mma_phase = 0;
  // the row of H (and of the windows) this thread owns: t = 16*warp + lane, lanes 0..15
  const int trow = warp * 16 + lane;
  const bool owner = lane < 16 && trow < T;
  for (int z = 0; z < g.nz; ++z) {
    if (*abort_flag) break;  // uniform: read after the barrier closing the previous plane
    if (!mbar_wait_bounded(bart, (uint32_t)(z & 1), status)) *abort_flag = 1;
    const int klo = tab.cover[2][2 * z], khi = tab.cover[2][2 * z + 1];
    const bool active = klo <= khi;  // uniform
    if (active) {
      // split into the hi / lo K-major tiles; item (t, 4 voxels) -> one 16-byte
      // core-matrix row at (t/8)*SBO + v4*128 + (t%8)*16
      for (int e = tid; e < T * nv4; e += blockDim.x) {
        const int v4 = e / T, t = e - v4 * T;
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int v = 4 * v4 + i;
          const float x = v < rows ? plane[v * T + t] : 0.f;
          h[i] = tf32_rna(x);
          l[i] = tf32_rna(x - __uint_as_float(h[i]));
        }
        const uint32_t off = (uint32_t)(t >> 3) * sbo + (uint32_t)v4 * 128 + (uint32_t)(t & 7) * 16;
        *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();  // tiles written, plane slot free
    if (tid == 0) {
      if (z + 1 < g.nz) {  // next plane streams in while this one's MMAs run
        mbar_expect_tx(bart, plane_bytes);
        tma_load_4d(plane_addr, &xmap, bart, 0, z + 1, cy, cx);
      }
      if (active) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        uint32_t acc = 0;
        for (int ks = 0; ks < kpad / 8; ++ks) {
          const uint32_t koff = (uint32_t)ks * 256;  // 8 tf32 = two core matrices along K
          const uint64_t dh = umma_desc_kmajor(hi_addr + koff, 128, sbo);
          const uint64_t dl = umma_desc_kmajor(lo_addr + koff, 128, sbo);
          umma_tf32(tmem, dh, dh, idesc, acc);
          umma_tf32(tmem, dh, dl, idesc, 1);
          umma_tf32(tmem, dl, dh, idesc, 1);
          acc = 1;
        }
        umma_commit(barm);
      }
    }
    if (active) {
      if (!mbar_wait_bounded(barm, mma_phase, status, kStatusMmaTimeout)) *abort_flag = 1;
      mma_phase ^= 1;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      if (warp * 16 < T) {
        for (int c0 = 0; c0 < Npad; c0 += 16) {
          float h[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, h);
          if (owner) {
            for (int k = klo; k <= khi; ++k) {
              float* w = win + (size_t)(k % ring) * T * T + trow;  // column c at w[c * T]
              const bool last = z == tab.corners[2][k] + g.pz - 1;
              float* G = G0 + (size_t)k * T * T + (size_t)trow * T;
#pragma unroll
              for (int c = 0; c < 16; ++c) {
                if (c0 + c < T) {
                  const float val = w[(size_t)(c0 + c) * T] + h[c];
                  if (last) {
                    G[c0 + c] = val;
                    w[(size_t)(c0 + c) * T] = 0.f;
                  } else {
                    w[(size_t)(c0 + c) * T] = val;
                  }
                }
              }
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    __syncthreads();  // TMEM and tiles rewritten next plane
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

}  // namespace lrd
