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
// Waits (TMA and MMA completion) are bounded by %globaltimer deadlines. When
// one gives up, the CTA issues no further copy or MMA, the issuing thread
// waits (with the same bound) for the copies and MMAs it still has in flight,
// and only then is the TMEM allocation released and the CTA retired; the
// status word records the timeout.
//
// A second operand kind, kind::f16 with BF16 operands (the BF16 form): x is
// split into three BF16 terms, x = b0 + b1 + b2 (b0 = bf16(x), b1 = bf16(x -
// b0), b2 = bf16(x - b0 - b1): 24 bits of the float32 value), and
//     H = b0.b0 + b0.b1 + b1.b0 + b0.b2 + b1.b1 + b2.b0
// (every product of combined order <= 2; the dropped terms are below 2^-24
// of the leading one), K = 16 voxels per instruction, FP32 accumulation in
// TMEM as above.
#pragma once

#include <cuda_bf16.h>

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

// Instruction descriptor: kind::f16, D = F32, A = B = BF16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ uint32_t bf16_bits(float x) { return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_value(uint32_t b) { return __uint_as_float(b << 16); }

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

// Two-stage pipeline per column CTA (256 threads): while the tensor cores
// run plane z's MMAs (operand tiles and TMEM accumulator of stage (z - zlo) & 1,
// zlo = the CTA's first plane),
// the CTA reads back plane z-1's Gram from the other accumulator and adds it
// into the windows; planes arrive by TMA two ahead (two plane slots).
//
// Shared-memory layout (bytes): two stages of {hi tile, lo tile}
// (ceil(T/8) row groups of SBO bytes each), two plane slots, the plane Gram
// H (T x (T+1) floats, read back from TMEM), the windows (ring x T(T+1)/2
// floats: upper triangle, r <= c), the upper-triangle index table
// (T(T+1)/2 x uint32, r | c << 16), mbarriers (2 TMA + 2 MMA), TMEM address,
// abort flag. An A descriptor spans 8 row groups from its tile's start
// (M = 64); rows past T read whatever follows (the lo tile, or the plane
// slots after the last tile) and only feed accumulator rows >= T, which are
// never read back.
// Operand layout per kind: a core matrix row holds 16 bytes = 4 TF32 or 8
// BF16 values along K; an instruction's K (8 TF32, 16 BF16) spans two core
// matrices; a stage holds 2 (hi, lo) or 3 (b0, b1, b2) split tiles.
__host__ __device__ inline int gramtc_kvals(bool bf16) { return bf16 ? 8 : 4; }
__host__ __device__ inline int gramtc_parts(bool bf16) { return bf16 ? 3 : 2; }
__host__ __device__ inline int gramtc_kpad(int rows, bool bf16 = false) {
  const int k = 2 * gramtc_kvals(bf16);
  return (rows + k - 1) / k * k;
}
__host__ __device__ inline size_t gramtc_sbo(int rows, bool bf16 = false) {
  return (size_t)(gramtc_kpad(rows, bf16) / gramtc_kvals(bf16)) * 128;
}
__host__ __device__ inline size_t gramtc_tile_bytes(int rows, int T, bool bf16 = false) {
  return (size_t)((T + 7) / 8) * gramtc_sbo(rows, bf16);
}
__host__ __device__ inline size_t gramtc_off_plane(int rows, int T, bool bf16 = false) {
  return 2 * (size_t)gramtc_parts(bf16) * gramtc_tile_bytes(rows, T, bf16);
}
__host__ __device__ inline int gramtc_ntri(int T) { return T * (T + 1) / 2; }
__host__ __device__ inline size_t gramtc_smem_bytes(int rows, int T, int ring, bool bf16 = false) {
  const size_t planes = 2 * sizeof(float) * gramz_plane_floats(rows, T);
  const size_t end = gramtc_off_plane(rows, T, bf16) + planes + sizeof(float) * (size_t)T * (T + 1) +
                     sizeof(float) * (size_t)ring * gramtc_ntri(T) + sizeof(uint32_t) * gramtc_ntri(T) + 64;
  // an A operand spans 8 row groups from the last tile's start
  const size_t span = (2 * (size_t)gramtc_parts(bf16) - 1) * gramtc_tile_bytes(rows, T, bf16) +
                      8 * gramtc_sbo(rows, bf16);
  return end > span ? end : span;
}
__host__ __device__ inline int gramtc_npad(int T) { return (T + 7) & ~7; }
constexpr int kGramTcThreads = 256;
constexpr int kIssuer = 128;  // TMA + MMA issuing thread (warp 4: no TMEM readback)
constexpr uint32_t kGramTcCols = 128;  // two accumulators of up to 64 columns

// grid: nfull + (columns - nfull) * nsplit CTAs (columns cut into window
// ranges as in gram_z_kernel); block: kGramTcThreads. T <= 64, T % 4 == 0,
// px*py <= 128. ``gram`` points at the Gram block of patch col0 * ncz.
template <bool BF16>
__global__ void __launch_bounds__(kGramTcThreads)
    gram_tc_kernel(const __grid_constant__ CUtensorMap xmap, float* __restrict__ gram, Geom g, AxisTables tab,
                   long long col0, int ring, int nfull, int nsplit, int* status) {
  extern __shared__ __align__(1024) unsigned char smt[];
  constexpr int NP = BF16 ? 3 : 2;  // split tiles per stage
  const int T = g.nt;
  const int rows = g.px * g.py;
  const int kpad = gramtc_kpad(rows, BF16);
  const uint32_t sbo = (uint32_t)gramtc_sbo(rows, BF16);  // bytes between 8-row groups
  const size_t tile = gramtc_tile_bytes(rows, T, BF16);
  const size_t pf = gramz_plane_floats(rows, T);
  const int ntri = gramtc_ntri(T);
  const int TH = T + 1;  // H row stride (odd: conflict-free column writes)
  float* planes = reinterpret_cast<float*>(smt + gramtc_off_plane(rows, T, BF16));  // two slots of pf floats
  float* H = planes + 2 * pf;
  float* win = H + (size_t)T * TH;  // [ring][ntri]
  uint32_t* tri = reinterpret_cast<uint32_t*>(win + (size_t)ring * ntri);
  uint64_t* bars = reinterpret_cast<uint64_t*>(tri + ntri + ((ntri & 1) ? 1 : 0));  // 8-byte aligned
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 4);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);  // set when a wait gave up
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int nth = blockDim.x;

  // this CTA's column, windows [wlo, whi] and planes [zlo, zhi]
  const int bid = (int)blockIdx.x;
  const bool cut = bid >= nfull;
  const int u = cut ? bid - nfull : 0, nparts = cut ? nsplit : 1, part = u % nparts;
  const long long col = col0 + (cut ? nfull + u / nparts : bid);
  const int wlo = part * g.ncz / nparts, whi = (part + 1) * g.ncz / nparts - 1;
  const int zlo = tab.corners[2][wlo], zhi = tab.corners[2][whi] + g.pz - 1;
  const int ci = (int)(col / g.ncy), cj = (int)(col % g.ncy);
  const int cx = tab.corners[0][ci], cy = tab.corners[1][cj];
  const uint32_t plane_bytes = (uint32_t)(rows * T * sizeof(float));
  const int Npad = gramtc_npad(T);
  const uint32_t idesc = BF16 ? umma_idesc_bf16(64, Npad) : umma_idesc_tf32(64, Npad);
  constexpr int KV = BF16 ? 8 : 4;  // voxels per 16-byte core-matrix row
  const int nv4 = (rows + KV - 1) / KV;

  // zero both stages' operand tiles (rows >= T and voxels >= rows stay zero) and the windows;
  // the upper-triangle table
  for (size_t e = tid; e < 2 * NP * tile / 16; e += nth) reinterpret_cast<uint4*>(smt)[e] = make_uint4(0, 0, 0, 0);
  for (int e = tid; e < ring * ntri; e += nth) win[e] = 0.f;
  for (int r = warp; r < T; r += nth / 32) {
    const int base = r * T - r * (r - 1) / 2;  // index of (r, r)
    for (int c = r + lane; c < T; c += 32) tri[base + (c - r)] = (uint32_t)r | ((uint32_t)c << 16);
  }
  if (tid == 0) {
    *abort_flag = 0;
    for (int i = 0; i < 4; ++i) mbar_init((uint32_t)__cvta_generic_to_shared(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(kGramTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t smt_addr = (uint32_t)__cvta_generic_to_shared(smt);
  const uint32_t planes_addr = (uint32_t)__cvta_generic_to_shared(planes);
  auto bar_tma = [&](int s) { return (uint32_t)__cvta_generic_to_shared(&bars[s]); };
  auto bar_mma = [&](int s) { return (uint32_t)__cvta_generic_to_shared(&bars[2 + s]); };

  // Work the issuing thread has in flight: per plane slot / accumulator, whether
  // a phase of its barrier is pending and that phase's parity. Each barrier has
  // at most one phase pending: a slot (accumulator) is refilled only after every
  // thread's wait for its previous plane succeeded (nothing is issued once a
  // wait has given up).
  bool tma_pend[2] = {false, false}, mma_pend[2] = {false, false};
  uint32_t tma_par[2] = {0, 0}, mma_par[2] = {0, 0};
  if (tid == kIssuer) {
    for (int i = 0; i < 2 && zlo + i <= zhi; ++i) {
      mbar_expect_tx(bar_tma(i), plane_bytes);
      tma_load_4d(planes_addr + (uint32_t)(i * pf * sizeof(float)), &xmap, bar_tma(i), 0, zlo + i, cy, cx);
      tma_pend[i] = true;
    }
  }
  float* G0 = gram + (size_t)((col - col0) * g.ncz) * T * T;

  // Reads back plane zr's Gram (accumulator (zr - zlo) & 1) into H and adds it
  // into the windows it belongs to; writes out the windows it completes.
  auto drain = [&](int zr) {
    const int s = (zr - zlo) & 1;
    if (!mbar_wait_bounded(bar_mma(s), (uint32_t)(((zr - zlo) >> 1) & 1), status, kStatusMmaTimeout))
      *abort_flag = 1;
    else if (tid == kIssuer)
      mma_pend[s] = false;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp < 4 && warp * 16 < T) {  // M = 64: rows 16w..16w+15 in lanes 0..15 of sub-partition w
      const int trow = warp * 16 + lane;
      for (int c0 = 0; c0 < Npad; c0 += 16) {
        float h[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(s * 64 + c0), h);
        if (lane < 16 && trow < T) {
#pragma unroll
          for (int c = 0; c < 16; ++c)
            if (c0 + c < T) H[trow * TH + c0 + c] = h[c];
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();  // H complete; the accumulator is free for plane zr + 2
    const int klo = max(tab.cover[2][2 * zr], wlo), khi = min(tab.cover[2][2 * zr + 1], whi);
    bool done_any = false;
    const int slot0 = klo % ring;  // window k's slot is (slot0 + k - klo) mod ring
    for (int e = tid; e < ntri; e += nth) {
      const uint32_t rc = tri[e];
      const float h = H[(rc & 0xffff) * TH + (rc >> 16)];
      int slot = slot0;
      for (int k = klo; k <= khi; ++k) {
        win[(size_t)slot * ntri + e] += h;
        if (++slot == ring) slot = 0;
      }
    }
    for (int k = klo; k <= khi; ++k) done_any |= zr == tab.corners[2][k] + g.pz - 1;
    if (done_any) {  // uniform
      __syncthreads();
      for (int k = klo; k <= khi; ++k) {
        if (zr != tab.corners[2][k] + g.pz - 1) continue;
        const float* w = win + (size_t)(k % ring) * ntri;
        float* G = G0 + (size_t)k * T * T;
        for (int r = warp; r < T; r += nth / 32)
          for (int c = lane; c < T; c += 32) {
            const int a = min(r, c), b2 = max(r, c);
            G[r * T + c] = w[a * T - a * (a - 1) / 2 + (b2 - a)];
          }
      }
      __syncthreads();
      for (int k = klo; k <= khi; ++k) {
        if (zr != tab.corners[2][k] + g.pz - 1) continue;
        float* w = win + (size_t)(k % ring) * ntri;
        for (int e = tid; e < ntri; e += nth) w[e] = 0.f;
      }
    }
    __syncthreads();  // H and the windows are rewritten by the next drain
  };

  for (int z = zlo; z <= zhi; ++z) {
    if (*abort_flag) break;  // uniform: read after the barrier closing the previous step
    const int it = z - zlo, s = it & 1;
    if (!mbar_wait_bounded(bar_tma(s), (uint32_t)((it >> 1) & 1), status))
      *abort_flag = 1;
    else if (tid == kIssuer)
      tma_pend[s] = false;
    // split plane z into stage s's K-major tiles; item (t, KV voxels) -> one
    // 16-byte core-matrix row at (t/8)*SBO + v4*128 + (t%8)*16 in each tile.
    // Stage s was last read by plane z-2's MMAs, drained in step z-1.
    const float* pl = planes + (size_t)s * pf;
    unsigned char* hi = smt + (size_t)s * NP * tile;
    unsigned char* lo = hi + tile;
    // item e = v4 * T + t, stepped by nth without a division per step
    const int dq = nth / T, dr = nth - (nth / T) * T;
    int v4 = tid / T, t = tid - (tid / T) * T;
    for (int e = tid; e < T * nv4; e += nth, v4 += dq, t += dr) {
      if (t >= T) {
        t -= T;
        ++v4;
      }
      const uint32_t off = (uint32_t)(t >> 3) * sbo + (uint32_t)v4 * 128 + (uint32_t)(t & 7) * 16;
      if constexpr (BF16) {
        uint32_t b[3][4];  // three terms, 8 BF16 values each, packed in pairs
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          uint32_t lohalf[3], hihalf[3];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int v = KV * v4 + 2 * i + h;
            const float x = v < rows ? pl[v * T + t] : 0.f;
            const uint32_t b0 = bf16_bits(x);
            const float r1 = x - bf16_value(b0);
            const uint32_t b1 = bf16_bits(r1);
            const uint32_t b2 = bf16_bits(r1 - bf16_value(b1));
            (h ? hihalf : lohalf)[0] = b0;
            (h ? hihalf : lohalf)[1] = b1;
            (h ? hihalf : lohalf)[2] = b2;
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) b[q][i] = lohalf[q] | (hihalf[q] << 16);
        }
#pragma unroll
        for (int q = 0; q < 3; ++q)
          *reinterpret_cast<uint4*>(hi + q * tile + off) = make_uint4(b[q][0], b[q][1], b[q][2], b[q][3]);
      } else {
        uint32_t hh[4], ll[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int v = 4 * v4 + i;
          const float x = v < rows ? pl[v * T + t] : 0.f;
          hh[i] = tf32_rna(x);
          ll[i] = tf32_rna(x - __uint_as_float(hh[i]));
        }
        *reinterpret_cast<uint4*>(hi + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
        *reinterpret_cast<uint4*>(lo + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();  // tiles written, plane slot s free
    if (tid == kIssuer && !*abort_flag) {  // a thread of a warp that does not read TMEM back
      if (z + 2 <= zhi) {
        mbar_expect_tx(bar_tma(s), plane_bytes);
        tma_load_4d(planes_addr + (uint32_t)(s * pf * sizeof(float)), &xmap, bar_tma(s), 0, z + 2, cy, cx);
        tma_pend[s] = true;
        tma_par[s] = (uint32_t)(((it + 2) >> 1) & 1);
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t hi_addr = smt_addr + (uint32_t)(s * NP * tile), lo_addr = hi_addr + (uint32_t)tile;
      const uint32_t acc_addr = tmem + (uint32_t)(s * 64);
      // the descriptors' start-address field is address >> 4: one K step (8 TF32
      // or 16 BF16 = two 128-byte core matrices) adds 16 to it
      uint64_t dh = umma_desc_kmajor(hi_addr, 128, sbo), dl = umma_desc_kmajor(lo_addr, 128, sbo);
      uint32_t acc = 0;
      if constexpr (BF16) {
        uint64_t d2 = umma_desc_kmajor(lo_addr + (uint32_t)tile, 128, sbo);
        for (int ks = 0; ks < kpad / 16; ++ks) {
          umma_bf16(acc_addr, dh, dh, idesc, acc);
          umma_bf16(acc_addr, dh, dl, idesc, 1);
          umma_bf16(acc_addr, dl, dh, idesc, 1);
          umma_bf16(acc_addr, dh, d2, idesc, 1);
          umma_bf16(acc_addr, dl, dl, idesc, 1);
          umma_bf16(acc_addr, d2, dh, idesc, 1);
          acc = 1;
          dh += 16;
          dl += 16;
          d2 += 16;
        }
      } else {
        for (int ks = 0; ks < kpad / 8; ++ks) {
          umma_tf32(acc_addr, dh, dh, idesc, acc);
          umma_tf32(acc_addr, dh, dl, idesc, 1);
          umma_tf32(acc_addr, dl, dh, idesc, 1);
          acc = 1;
          dh += 16;
          dl += 16;
        }
      }
      umma_commit(bar_mma(s));
      mma_pend[s] = true;
      mma_par[s] = (uint32_t)((it >> 1) & 1);
    }
    if (z > zlo) drain(z - 1);  // overlaps plane z's MMAs
    else __syncthreads();
  }
  if (!*abort_flag && zlo <= zhi) drain(zhi);
  __syncthreads();
  if (*abort_flag && tid == kIssuer) {
    // a wait gave up: let the copies and MMAs still in flight land (bounded)
    // before the tensor memory and the shared memory they write are released
    for (int i = 0; i < 2; ++i) {
      if (tma_pend[i]) mbar_wait_bounded(bar_tma(i), tma_par[i], status);
      if (mma_pend[i]) mbar_wait_bounded(bar_mma(i), mma_par[i], status, kStatusMmaTimeout);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kGramTcCols) : "memory");
}

}  // namespace lrd
