// Per-patch Gram matrices with the z-planes of a patch column shared.
//
// All patches with the same (x, y) corners form a column along z. Their Gram
// matrices G(cz) = sum_{z = cz}^{cz + pz - 1} H(z) are sums of the same
// per-plane Grams H(z) = sum over the px*py voxels of plane z of xc xc^T.
// gram_kernel recomputes every H(z) for each of the ~pz/stride windows that
// contain z; this kernel computes each H(z) once and adds it into every active
// window, which cuts the FFMA work by that factor (3.2x at 11^3 / stride 3).
//
// Layout: one CTA per (x-corner, y-corner) column; ``ks`` adjacent threads
// (lanes of one warp) share the 4x4 block G[4bi:4bi+4, 4bj:4bj+4], bi <= bj,
// each summing every ks-th voxel row of a plane, combined by shuffles (a
// K-split: ks times the warps per column for latency hiding). The block size
// is rounded up to whole warps; the extra threads only join the shuffles and
// barriers. The column's planes are
// streamed into a two-slot shared-memory ring by TMA (one 4D box (T, 1, py, px)
// of the centred volume per plane, completion on an mbarrier); the window
// accumulators of the active windows live in shared memory (a ring of
// ``ring`` slots, slot = window index mod ring). A plane's partial Gram is
// summed in float32 over its px*py voxels (FFMA), then added to the windows in
// float32; a window is written out (and its slot cleared) after its last plane.
// The K = px*py*pz sum therefore rounds as a two-level blocked sum, plane then
// window (the per-patch kernel rounds as x-plane then float64 window).
//
// Every mbarrier wait is bounded by a %globaltimer deadline. On expiry the
// kernel records LRD_STATUS_TMA_TIMEOUT in the status word (the result is
// then invalid and the host reports it), issues no further copy, and the
// issuing thread waits - with the same bound - for the copies it still has in
// flight into the CTA's shared memory before the CTA exits.
#pragma once

#include <cuda.h>

#include "lrd_common.cuh"

namespace lrd {

constexpr int kStatusTmaTimeout = 1;
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the phase with parity ``parity`` to complete; after
// ``limit_ns`` ``code`` is or-ed into the status word and the wait gives up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, int* status,
                                                  int code = kStatusTmaTimeout,
                                                  unsigned long long limit_ns = kWaitNs) {
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (globaltimer_ns() - t0 > limit_ns) {
      atomicOr(status, code);
      return false;
    }
  }
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

// After a wait gave up: wait (bounded) for the copies still in flight into the
// CTA's shared memory - the one whose wait gave up (``a``) and the one issued
// after it (``b``) - before the CTA exits.
__device__ __noinline__ void drain_copies(bool wait_a, uint32_t bar_a, uint32_t par_a, bool wait_b,
                                          uint32_t bar_b, uint32_t par_b, int* status) {
  if (wait_a) mbar_wait_bounded(bar_a, par_a, status);
  if (wait_b) mbar_wait_bounded(bar_b, par_b, status);
}

__host__ __device__ inline size_t gramz_plane_floats(int rows, int T) {
  return ((size_t)rows * T + 31) & ~size_t(31);  // 128-byte multiple
}

// Dynamic shared memory: two plane slots, ring * 16 * nblk float window
// accumulators (nblk = 4x4 blocks of the upper triangle), two mbarriers.
__host__ __device__ inline size_t gramz_smem_bytes(int rows, int T, int ring, int nblk) {
  return sizeof(float) * (2 * gramz_plane_floats(rows, T) + (size_t)ring * 16 * nblk) + 16;
}

// Threads of a column CTA for T frames and K-split ks: nb*(nb+1)/2 blocks
// (nb = T/4) times ks, rounded up to whole warps.
__host__ __device__ inline int gramz_threads(int T, int ks) {
  const int nb = T >> 2;
  return ((nb * (nb + 1) / 2 * ks) + 31) & ~31;
}

// grid: nfull + (columns - nfull) * nsplit CTAs; block: gramz_threads(T, KS)
// (T % 4 == 0, KS in {1, 2, 4}). CTA b < nfull computes every window of column
// col0 + b; the columns after the first nfull are each cut into nsplit units
// of consecutive windows (a unit reads only the planes of its windows), so a
// launch whose last wave would hold a few whole columns spreads that tail
// over many SMs. A window's planes are added in the same order either way: the
// result does not depend on the cut. ``col0`` = first column (x-major index
// ci * ncy + cj); ``gram`` points at the Gram block of the launch's first
// patch (patch index col0 * ncz).
// Body of one CTA (index ``bid``); ``xmap`` points at the tensor map (a kernel
// parameter, or a 64-byte aligned copy in global memory for the packed
// multi-volume launch).
template <int KS>
__device__ __forceinline__ void gram_z_body(const CUtensorMap* xmap, float* __restrict__ gram, const Geom& g,
                                            const AxisTables& tab, long long col0, int ring, int nfull, int nsplit,
                                            int* status, int bid) {
  constexpr int ks = KS;
  extern __shared__ __align__(128) float smz[];
  const int T = g.nt;
  const int rows = g.px * g.py;
  const size_t pf = gramz_plane_floats(rows, T);
  float* plane0 = smz;
  float* plane1 = smz + pf;
  const int nb = T >> 2;
  const int nblk = nb * (nb + 1) / 2;
  float* win = smz + 2 * pf;  // [ring][16][nblk]
  const int nthreads = blockDim.x;
  uint64_t* bars = reinterpret_cast<uint64_t*>(win + (size_t)ring * 16 * nblk);
  const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&bars[0]);
  const uint32_t bar1 = (uint32_t)__cvta_generic_to_shared(&bars[1]);

  // this CTA's column and windows [wlo, whi]
  const bool cut = bid >= nfull;
  const int u = cut ? bid - nfull : 0, nparts = cut ? nsplit : 1, part = u % nparts;
  const long long col = col0 + (cut ? nfull + u / nparts : bid);
  const int wlo = part * g.ncz / nparts, whi = (part + 1) * g.ncz / nparts - 1;
  const int zlo = tab.corners[2][wlo], zhi = tab.corners[2][whi] + g.pz - 1;  // its planes
  const int ci = (int)(col / g.ncy), cj = (int)(col % g.ncy);
  const int cx = tab.corners[0][ci], cy = tab.corners[1][cj];
  const int tid = threadIdx.x;
  const int blk = tid / ks, kq = tid - (tid / ks) * ks;
  const bool owner = blk < nblk;
  int bi = 0, bj = 0;
  if (owner) {
    int rem = blk;
    while (bi < nb && rem >= nb - bi) {
      rem -= nb - bi;
      ++bi;
    }
    bj = bi + rem;
  }
  constexpr int ucount = 16 / ks;  // window entries this thread updates: [kq * ucount, kq * ucount + ucount)
  const uint32_t plane_bytes = (uint32_t)(rows * T * sizeof(float));

  for (int e = tid; e < ring * 16 * nblk; e += nthreads) win[e] = 0.f;
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0 && zlo <= zhi) {
    mbar_expect_tx(bar0, plane_bytes);
    tma_load_4d((uint32_t)__cvta_generic_to_shared(plane0), xmap, bar0, 0, zlo, cy, cx);
  }
  float* G0 = gram + (size_t)((col - col0) * g.ncz) * T * T;
  int gave_up = 0;  // uniform: a wait of some thread gave up at plane stop_z
  int stop_z = zhi;
  bool own_wait_ok = true;
  for (int z = zlo; z <= zhi && !gave_up; ++z) {
    const int it = z - zlo, slot = it & 1;
    // Each slot's barrier has at most one phase pending: plane z + 1 goes into
    // the slot whose previous plane (z - 1) every thread waited for in full.
    const bool issued_next = z + 1 <= zhi;
    if (tid == 0 && issued_next) {
      const uint32_t nb_ = slot ? bar0 : bar1;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_expect_tx(nb_, plane_bytes);
      tma_load_4d((uint32_t)__cvta_generic_to_shared(slot ? plane0 : plane1), xmap, nb_, 0, z + 1, cy, cx);
    }
    const bool ok = mbar_wait_bounded(slot ? bar1 : bar0, (uint32_t)((it >> 1) & 1), status);
    const int klo = max(tab.cover[2][2 * z], wlo), khi = min(tab.cover[2][2 * z + 1], whi);
    if (klo <= khi) {
      const float* pl = slot ? plane1 : plane0;
      float acc[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) acc[u] = 0.f;
      const float4* rp = reinterpret_cast<const float4*>(pl);
      const int ld4 = T >> 2;
#pragma unroll 4
      for (int r = kq; r < rows; r += ks) {
        const float4 va = rp[r * ld4 + bi];
        const float4 vb = rp[r * ld4 + bj];
        const float a4[4] = {va.x, va.y, va.z, va.w};
        const float b4[4] = {vb.x, vb.y, vb.z, vb.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u * 4 + v] = fmaf(a4[u], b4[v], acc[u * 4 + v]);
      }
      // combine the ks partial sums (every lane of the group ends with the total)
      if (ks >= 2) {
#pragma unroll
        for (int u = 0; u < 16; ++u) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], 1);
      }
      if (ks >= 4) {
#pragma unroll
        for (int u = 0; u < 16; ++u) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], 2);
      }
      if (owner) {
        // this thread's entries of the 4x4 block, e = kq * ucount + q
        float mine[ucount];
#pragma unroll
        for (int q = 0; q < ucount; ++q) {
          float v = acc[q];
#pragma unroll
          for (int c = 1; c < ks; ++c)
            if (kq == c) v = acc[c * ucount + q];
          mine[q] = v;
        }
        // Windows are consecutive and their corners increase, so only the
        // lowest window holding plane z (klo) can end at z.
        const bool klo_ends = z == tab.corners[2][klo] + g.pz - 1;
        int slot = klo % ring;
        for (int k = klo; k <= khi; ++k) {
          float* w = win + (size_t)slot * 16 * nblk + blk + (size_t)kq * ucount * nblk;
          if (k != klo || !klo_ends) {
#pragma unroll
            for (int q = 0; q < ucount; ++q) w[q * nblk] += mine[q];
          } else {
            float* G = G0 + (size_t)k * T * T;
#pragma unroll
            for (int q = 0; q < ucount; ++q) {
              const int e = kq * ucount + q;
              const float val = w[q * nblk] + mine[q];
              w[q * nblk] = 0.f;
              const int r = bi * 4 + (e >> 2), c = bj * 4 + (e & 3);
              G[(size_t)r * T + c] = val;
              G[(size_t)c * T + r] = val;
            }
          }
          if (++slot == ring) slot = 0;
        }
      }
    }
    // this slot is refilled by the TMA issued at the start of the next iteration
    gave_up = __syncthreads_or(!ok);
    stop_z = z;
    own_wait_ok = ok;
  }
  if (gave_up && tid == 0) {
    // a wait gave up: nothing more was issued; wait (bounded) for the copies
    // still in flight - plane stop_z if this thread's own wait gave up, and
    // plane stop_z + 1 - so that none lands after the CTA's shared memory is freed
    const int it = stop_z - zlo, slot = it & 1;
    drain_copies(!own_wait_ok, slot ? bar1 : bar0, (uint32_t)((it >> 1) & 1), stop_z + 1 <= zhi,
                 slot ? bar0 : bar1, (uint32_t)(((it + 1) >> 1) & 1), status);
  }
}

template <int KS>
__global__ void __maxnreg__(64) gram_z_kernel(const __grid_constant__ CUtensorMap xmap, float* __restrict__ gram, Geom g,
                              AxisTables tab, long long col0, int ring, int nfull, int nsplit,
                              int* status) {
  gram_z_body<KS>(&xmap, gram, g, tab, col0, ring, nfull, nsplit, status, (int)blockIdx.x);
}

// Self-test of the bounded wait: one thread waits on a freshly initialised
// mbarrier that nothing arrives at, gives up after ``limit_ns`` and records
// ``code`` in ``status``; no copy or MMA is in flight, so the kernel simply
// returns. grid 1, block 32.
__global__ void wait_timeout_selftest_kernel(int* status, unsigned long long limit_ns, int code) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bar);
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    mbar_wait_bounded(b, 0, status, code, limit_ns);
  }
}

}  // namespace lrd
