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
// MMA shape: M = 128 (rows = frames t; rows >= T are never read back), N = T
// (rounded up to 16), K = 8 voxels per instruction over the plane's voxels
// padded to a multiple of 8. A (M x K) and B (stored as its K-major transpose,
// N x K) are the same shared-memory tile X^T in the canonical K-major,
// no-swizzle layout: 8-row x 16-byte core matrices, LBO = 128 B between core
// matrices along K, SBO = (K/4) * 128 B between 8-row groups. The
// accumulator D (row i in TMEM lane i, column j in TMEM column j) is read back
// by the four warps (warp w owns lanes 32w..32w+31) with tcgen05.ld, and
// thread t (< T) adds row t of H into its windows' rows in shared memory.
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
// lo tile (same), two plane slots, windows, mbarriers, TMEM address. An A
// descriptor spans 16 row groups from its tile's start (M = 128); the rows
// past T read whatever follows (they only feed accumulator rows >= T, which
// are never read), so the allocation just has to cover lo + 16 groups.
__host__ __device__ inline int gramtc_kpad(int rows) { return (rows + 7) & ~7; }
__host__ __device__ inline size_t gramtc_sbo(int rows) { return (size_t)(gramtc_kpad(rows) / 4) * 128; }
__host__ __device__ inline size_t gramtc_tile_bytes(int rows, int T) { return (size_t)((T + 7) / 8) * gramtc_sbo(rows); }
__host__ __device__ inline size_t gramtc_off_planes(int rows, int T) { return 2 * gramtc_tile_bytes(rows, T); }
__host__ __device__ inline size_t gramtc_smem_bytes(int rows, int T, int ring) {
  const size_t end = gramtc_off_planes(rows, T) +
                     sizeof(float) * (2 * gramz_plane_floats(rows, T) + (size_t)ring * T * T) + 64;
  const size_t span = gramtc_tile_bytes(rows, T) + 16 * gramtc_sbo(rows);
  return end > span ? end : span;
}
// (+ 64 bytes at the end hold the three mbarriers, the TMEM address and the abort flag)

// grid: (columns in this launch); block: 128 threads (4 warps). T <= 64 and
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
  float* plane0 = reinterpret_cast<float*>(smt + gramtc_off_planes(rows, T));
  float* plane1 = plane0 + gramz_plane_floats(rows, T);
  float* win = plane1 + gramz_plane_floats(rows, T);  // [ring][T cols][T rows]
  uint64_t* bars = reinterpret_cast<uint64_t*>(win + (size_t)ring * T * T);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);  // set when a wait gave up
  const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&bars[0]);
  const uint32_t bar1 = (uint32_t)__cvta_generic_to_shared(&bars[1]);
  const uint32_t barm = (uint32_t)__cvta_generic_to_shared(&bars[2]);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;

  const long long col = col0 + blockIdx.x;
  const int ci = (int)(col / g.ncy), cj = (int)(col % g.ncy);
  const int cx = tab.corners[0][ci], cy = tab.corners[1][cj];
  const uint32_t plane_bytes = (uint32_t)(rows * T * sizeof(float));
  const int Npad = (T + 15) & ~15;
  const uint32_t idesc = umma_idesc_tf32(128, Npad);
  const uint32_t ncols = Npad <= 32 ? 32 : (Npad <= 64 ? 64 : 128);

  // zero the operand tiles once (rows >= T and voxels >= rows stay zero) and the windows
  for (size_t e = tid; e < 2 * tile / 16; e += blockDim.x) reinterpret_cast<uint4*>(smt)[e] = make_uint4(0, 0, 0, 0);
  for (int e = tid; e < ring * T * T; e += blockDim.x) win[e] = 0.f;
  if (tid == 0) {
    *abort_flag = 0;
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
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

  if (tid == 0 && g.nz > 0) {
    mbar_expect_tx(bar0, plane_bytes);
    tma_load_4d((uint32_t)__cvta_generic_to_shared(plane0), &xmap, bar0, 0, 0, cy, cx);
  }
  float* G0 = gram + (size_t)((col - col0) * g.ncz) * T * T;
  uint32_t mma_phase = 0;
  for (int z = 0; z < g.nz; ++z) {
    if (*abort_flag) break;  // uniform: read after the barrier closing the previous plane
    const int slot = z & 1;
    if (tid == 0 && z + 1 < g.nz) {
      const uint32_t nb_ = slot ? bar0 : bar1;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_expect_tx(nb_, plane_bytes);
      tma_load_4d((uint32_t)__cvta_generic_to_shared(slot ? plane0 : plane1), &xmap, nb_, 0, z + 1, cy, cx);
    }
    if (!mbar_wait_bounded(slot ? bar1 : bar0, (uint32_t)((z >> 1) & 1), status)) *abort_flag = 1;
    const int klo = tab.cover[2][2 * z], khi = tab.cover[2][2 * z + 1];
    if (klo <= khi) {  // uniform
      // split the plane into the hi / lo K-major tiles: element (t, v) at
      // (t/8)*SBO + (v/4)*128 + (t%8)*16 + (v%4)*4
      const float* pl = slot ? plane1 : plane0;
      for (int e = tid; e < rows * T; e += blockDim.x) {
        const int v = e / T, t = e - v * T;
        const float x = pl[e];
        const uint32_t h = tf32_rna(x);
        const uint32_t l = tf32_rna(x - __uint_as_float(h));
        const uint32_t off = (uint32_t)(t >> 3) * sbo + (uint32_t)(v >> 2) * 128 + (uint32_t)(t & 7) * 16 +
                             (uint32_t)(v & 3) * 4;
        *reinterpret_cast<uint32_t*>(hi + off) = h;
        *reinterpret_cast<uint32_t*>(lo + off) = l;
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();
      if (tid == 0) {
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
      if (!mbar_wait_bounded(barm, mma_phase, status, kStatusMmaTimeout)) *abort_flag = 1;
      mma_phase ^= 1;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      // row t = 32*warp + lane of H; all lanes of a warp take part in tcgen05.ld
      const int t = warp * 32 + lane;
      if (warp * 32 < T) {
        for (int c0 = 0; c0 < Npad; c0 += 16) {
          float h[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, h);
          if (t < T) {
            for (int k = klo; k <= khi; ++k) {
              float* w = win + (size_t)(k % ring) * T * T;
              const bool last = z == tab.corners[2][k] + g.pz - 1;
              float* G = G0 + (size_t)k * T * T;
#pragma unroll
              for (int c = 0; c < 16; ++c) {
                if (c0 + c < T) {
                  const float val = w[(size_t)(c0 + c) * T + t] + h[c];
                  if (last) {
                    G[(size_t)t * T + c0 + c] = val;
                    w[(size_t)(c0 + c) * T + t] = 0.f;
                  } else {
                    w[(size_t)(c0 + c) * T + t] = val;
                  }
                }
              }
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    __syncthreads();  // plane slot reuse, tiles and TMEM rewritten next plane
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

}  // namespace lrd
