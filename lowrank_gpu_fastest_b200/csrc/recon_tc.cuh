// Reconstruction of the tensor forms on the tcgen05 tensor cores: both
// contractions of the ladder's recon_scatter_kernel (step8_tuned.py:59-86,
// y = (x - m) V_p, xd = y V_p^T) as two chained split-TF32 GEMMs per brick,
// with the weighted overlap accumulation folded into the second one.
//
// For a brick of 128 voxels (4 x 4 x 8) and the patches that touch it, let
// V be the concatenation of their top-p eigenvector rows (one column per
// (patch, k)) and X the brick's centred time courses (128 x T). Then
//
//   Y  = X V^T                       (GEMM 1: 128 x ncol, K = T)
//   Y~ = Y o S,  S[v, c] = w_q if voxel v lies in patch q of column c, else 0
//   A  = Y~ V                        (GEMM 2: 128 x T,    K = ncol)
//   out[v] = m[v] + A[v] / sum_{q covers v} w_q
//
// which is sum_q w_q (x - m) V_q V_q^T / sum_q w_q + m per voxel
// (step8:137-145): the overlap accumulation is GEMM 2's K sum.
//
// Precision. Every product is a 3xTF32 split (hi = rna_tf32(a), lo =
// rna_tf32(a - hi); hi.hi + hi.lo + lo.hi): float32-grade products. The
// tensor cores' FP32 accumulation in tensor memory rounds every MMA's sum
// towards zero, a bias of about half an ulp of the accumulator per MMA (the
// tcgen05 Gram measures 1.2e-6 of the largest entry after 48 MMAs per plane,
// against 1.2e-7 for FFMA), so no sum here runs through a long MMA chain:
//  * GEMM 1 keeps hi.hi (T/8 MMAs) and the two cross products (2T/8 MMAs,
//    2^-11 smaller) in two accumulators, added in FP32 on the CUDA cores;
//  * GEMM 2 gives each K step (8 columns) its own accumulator (three MMAs,
//    the first one overwriting), and the CUDA cores add the K steps' sums
//    into a per-voxel FP32 accumulator in registers (round to nearest).
// The weight sums are float64 (exact: a few hundred float32 values 1/(2+p)).
//
// Columns are taken in groups of one x corner index (every touching patch
// (i, j, k) of the brick with the same i, j-major then k, then the patch's
// eigenvectors in order), each group cut into chunks of kRtcChunk columns
// (the last one zero-padded). A chunk never mixes two x corners, so a voxel's
// sum is the same sequence of additions whichever x-slab computes which of
// its patches: a slab that hands its partial sums on (SlabIO halo, an exact
// float64 copy) and the next slab that continues from them give
// bit-identical results to one unsharded call.
//
// Per brick, once: the X tiles split into shared memory; the touching
// patches' indices, ranks, weights and cover masks into a shared table, and
// each x-corner group's rank prefix sums (so a chunk's column table is a
// binary search in shared memory); each voxel's weight sum.
// Per chunk (128 threads, thread v = voxel v = TMEM lane v):
//   1. the chunk's eigenvector rows (fetched into registers during the
//      previous chunk), split hi / lo into shared memory twice: as GEMM 1's
//      B (rows = columns, K = frames) and, through a raw copy, transposed as
//      GEMM 2's B (rows = frames, K = columns), both K-major (an MN-major B
//      operand of kind::tf32 read back zeros here);
//   2. GEMM 1 into TMEM columns [0, C) (hi.hi) and [C, 2C) (cross terms);
//      meanwhile the next chunk's column table is built and its rows are
//      fetched;
//   3. each thread reads its row of Y, scales it by S, splits it and writes
//      Y~ hi / lo over the same columns (GEMM 2's A operand, in TMEM);
//   4. GEMM 2, K step s into columns [2C + s Tn, 2C + (s + 1) Tn);
//   5. each thread adds the K steps' sums into its accumulator.
// Two CTAs share an SM (T <= 48: 256 TMEM columns and about 85 KB of shared
// memory each at the headline).
//
// Waits on MMA completion are bounded by %globaltimer deadlines as in the
// tensor-core Gram: a wait that gives up records kStatusMmaTimeout, the CTA
// issues nothing more, the issuing thread waits (bounded) for the commit still
// in flight, and the TMEM allocation is released before the CTA retires.
#pragma once

#include "gram_tc.cuh"
#include "recon.cuh"

namespace lrd {

constexpr int kRtcBX = 4, kRtcBY = 4, kRtcBZ = 8;  // brick (x, y, z): 128 voxels = the MMA's M
constexpr int kRtcThreads = 128;
constexpr int kRtcChunk = 32;                      // columns per chunk: 4 K steps of GEMM 2

// Frame counts the kernel handles: T % 4 == 0 (16-byte rows), T <= 64.
__host__ __device__ inline bool recon_tc_supported(int T) { return T % 4 == 0 && T >= 8 && T <= 64; }
__host__ __device__ inline int recon_tc_tk(int T) { return (T + 7) & ~7; }    // GEMM 1 K (TF32 K step 8)
__host__ __device__ inline int recon_tc_tn(int T) { return (T + 15) & ~15; }  // GEMM 2 N (M = 128: N % 16)

// TMEM columns of a CTA (a power of two >= 32): Y hi.hi / Y~ hi [0, C),
// cross / Y~ lo [C, 2C), K-step sums [2C, 2C + (C / 8) Tn).
__host__ __device__ constexpr uint32_t recon_tc_tmem_cols(int Tn) {
  return (2 * kRtcChunk + kRtcChunk / 8 * Tn) <= 128 ? 128u : ((2 * kRtcChunk + kRtcChunk / 8 * Tn) <= 256 ? 256u : 512u);
}

// Shared-memory layout (bytes): X hi, X lo (128 x Tk each, K-major core
// matrices), V hi, V lo (C rows x Tn), V^T hi, V^T lo (Tn rows x C), raw
// rows for the transpose (C x (Tn + 4) floats), two column tables (C x {row
// offset (8), mask (4), weight (4)} each), mbarrier, TMEM address, abort
// flag, the brick's touching patches (npb of them: index (8), cover mask,
// weight, rank (4 each)) and each x-corner group's rank prefix sums (npb +
// groups ints).
__host__ __device__ inline size_t recon_tc_xbytes(int T) { return (size_t)128 * recon_tc_tk(T) * 4; }
__host__ __device__ inline size_t recon_tc_vbytes(int T) { return (size_t)kRtcChunk * recon_tc_tn(T) * 4; }
// a brick whose patch box holds more patches than this (small strides with
// large patches) takes the warp kernel instead
constexpr int kRtcMaxBoxPatches = 1024;
__host__ __device__ inline size_t recon_tc_smem_bytes(int T, int npb, int ngroups) {
  return 2 * recon_tc_xbytes(T) + 4 * recon_tc_vbytes(T) + (size_t)kRtcChunk * (recon_tc_tn(T) + 4) * 4 +
         (size_t)kRtcChunk * 32 + 24 + 20 * (size_t)npb + 4 * ((size_t)npb + ngroups);
}

// Instruction descriptor: kind::tf32, D = F32, M = 128, A and B K-major.
__host__ __device__ constexpr uint32_t rtc_idesc(int N) { return umma_idesc_tf32(128, N); }

// MMA with A from tensor memory (GEMM 2).
__device__ __forceinline__ void umma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                             uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

// 16 columns of this warp's lanes, without the wait (tcgen05.wait::ld follows).
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};\n" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}

// Bits of the brick-local positions [0, n) along one axis that a patch with
// corner c and side p covers, the brick starting at b0.
__device__ __forceinline__ uint32_t rtc_axis_mask(int c, int p, int b0, int n) {
  const int lo = max(c - b0, 0), hi = min(c + p - 1 - b0, n - 1);
  return hi < lo ? 0u : ((2u << hi) - (1u << lo));
}

__device__ __forceinline__ void rtc_split4(const float4 v, uint4& h, uint4& l) {
  h.x = tf32_rna(v.x);
  h.y = tf32_rna(v.y);
  h.z = tf32_rna(v.z);
  h.w = tf32_rna(v.w);
  l.x = tf32_rna(v.x - __uint_as_float(h.x));
  l.y = tf32_rna(v.y - __uint_as_float(h.y));
  l.z = tf32_rna(v.z - __uint_as_float(h.z));
  l.w = tf32_rna(v.w - __uint_as_float(h.w));
}

// GEMM 1 of a chunk (one thread): Y hi.hi into columns [0, C), hi.lo + lo.hi
// into [C, 2C); K = tk. Out of line, so that its descriptors are not held in
// registers across the chunk loop.
__device__ __noinline__ void rtc_issue_gemm1(uint32_t tmem, uint32_t xhi_a, uint32_t xbytes, uint32_t sbox,
                                            uint32_t vhi_a, uint32_t vbytes, uint32_t sbov, int tk, uint32_t idesc) {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  for (int ks = 0; ks < tk / 8; ++ks) {
    const uint32_t o = (uint32_t)ks * 256;
    const uint64_t ah = umma_desc_kmajor(xhi_a + o, 128, sbox), al = umma_desc_kmajor(xhi_a + xbytes + o, 128, sbox);
    const uint64_t bh = umma_desc_kmajor(vhi_a + o, 128, sbov), bl = umma_desc_kmajor(vhi_a + vbytes + o, 128, sbov);
    umma_tf32(tmem, ah, bh, idesc, ks > 0 ? 1u : 0u);
    umma_tf32(tmem + kRtcChunk, ah, bl, idesc, ks > 0 ? 1u : 0u);
    umma_tf32(tmem + kRtcChunk, al, bh, idesc, 1u);
  }
}

// GEMM 2 of a chunk (one thread): K step s (8 columns of Y~, A from TMEM
// columns [8s, 8s + 8) hi and [C + 8s, ...) lo) into its own accumulator
// [2C + s tn, 2C + (s + 1) tn); B = V^T (rows = frames, K = columns).
__device__ __noinline__ void rtc_issue_gemm2(uint32_t tmem, uint32_t thi_a, uint32_t vbytes, uint32_t sbot, int tn,
                                            uint32_t idesc) {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  for (int ks = 0; ks < kRtcChunk / 8; ++ks) {
    const uint32_t o = (uint32_t)ks * 256;
    const uint64_t bh = umma_desc_kmajor(thi_a + o, 128, sbot), bl = umma_desc_kmajor(thi_a + vbytes + o, 128, sbot);
    const uint32_t d = tmem + (uint32_t)(2 * kRtcChunk + ks * tn);
    const uint32_t ah = tmem + (uint32_t)(ks * 8), al = tmem + (uint32_t)(kRtcChunk + ks * 8);
    umma_tf32_ts(d, ah, bh, idesc, 0u);
    umma_tf32_ts(d, ah, bl, idesc, 1u);
    umma_tf32_ts(d, al, bh, idesc, 1u);
  }
}

// One CTA: brick brick0 + bid of the plan's 4 x 4 x 8 brick grid (x-major).
// Thread v owns voxel (x0 + v / 32, y0 + (v / 8) % 4, z0 + v % 8), MMA row v.
// TN = recon_tc_tn(T): the per-voxel accumulator lives in registers.
template <int TN>
__device__ __forceinline__ void recon_tc_body(const float* __restrict__ xc, const float* __restrict__ mean,
                                              const float* __restrict__ vecs, const int32_t* __restrict__ ranks,
                                              const float* __restrict__ wgt, float* __restrict__ out, const Geom& g,
                                              const AxisTables& tab, int brick0, const SlabIO& io, int* status,
                                              int bid) {
  static_assert(TN % 16 == 0 && TN >= 16 && TN <= 64, "GEMM 2 N: 16, 32, 48 or 64");
  constexpr int C = kRtcChunk;
  constexpr int KS2 = C / 8;  // GEMM 2 K steps per chunk
  static_assert(KS2 == 4, "the K-step sums are added as (s0 + s1) + (s2 + s3)");
  constexpr int NG = TN / 4;                       // frame groups of an eigenvector row
  constexpr int ITEMS = C * NG / kRtcThreads;      // row float4s per thread per chunk
  constexpr int TITEMS = TN * (C / 4) / kRtcThreads;  // transposed units per thread per chunk
  static_assert(ITEMS * kRtcThreads == C * NG && TITEMS * kRtcThreads == TN * (C / 4), "whole items per thread");
  constexpr int RS = TN + 4;                       // raw row stride (floats)
  constexpr uint32_t kCols = recon_tc_tmem_cols(TN);
  extern __shared__ __align__(1024) unsigned char smr[];
  const int T = g.nt;
  const int Tk = recon_tc_tk(T);
  const size_t xb = recon_tc_xbytes(T), vb = recon_tc_vbytes(T);
  unsigned char* Xhi = smr;
  unsigned char* Vhi = smr + 2 * xb;                               // V hi, lo (rows = columns)
  unsigned char* Thi = Vhi + 2 * vb;                               // V^T hi, lo (rows = frames)
  float* raw = reinterpret_cast<float*>(Thi + 2 * vb);             // C x RS raw rows (transpose)
  long long* c_row = reinterpret_cast<long long*>(raw + C * RS);   // [2][C] eigenvector row offset, -1 = padding
  uint32_t* c_mask = reinterpret_cast<uint32_t*>(c_row + 2 * C);   // [2][C] cover bits: x | y << 4 | z << 8
  float* c_w = reinterpret_cast<float*>(c_mask + 2 * C);           // [2][C] patch weight
  uint64_t* bar = reinterpret_cast<uint64_t*>(c_w + 2 * C);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  int brick = brick0 + bid;
  const int bzi = brick % g.nbz;
  brick /= g.nbz;
  const int byi = brick % g.nby;
  const int bxi = brick / g.nby;
  const int x0 = bxi * kRtcBX, y0 = byi * kRtcBY, z0 = bzi * kRtcBZ;
  const int lx = tid >> 5, ly = (tid >> 3) & 3, lz = tid & 7;
  const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
  const bool valid = x < g.nx && y < g.ny && z < g.nz && x >= io.x_lo && x < io.x_hi;
  // a voxel outside the volume or the slab matches no column's cover bits
  const uint32_t vbits = valid ? ((1u << lx) | (1u << (4 + ly)) | (1u << (8 + lz))) : (1u << 16);
  const long long row = valid ? voxel_row(g, x, y, z) : 0;
  const int ilo = tab.brick[0][2 * bxi], ihi = tab.brick[0][2 * bxi + 1];
  const int jlo = tab.brick[1][2 * byi], jhi = tab.brick[1][2 * byi + 1];
  const int klo = tab.brick[2][2 * bzi], khi = tab.brick[2][2 * bzi + 1];
  const int ni = max(ihi - ilo + 1, 0), nk = max(khi - klo + 1, 0), nq = max(jhi - jlo + 1, 0) * nk;
  const int npb = ni * nq;  // the brick's touching patches: x-corner group a, then (j, k) j-major
  long long* pb_pid = reinterpret_cast<long long*>(tmem_slot + 4);
  uint32_t* pb_mask = reinterpret_cast<uint32_t*>(pb_pid + npb);
  float* pb_w = reinterpret_cast<float*>(pb_mask + npb);
  int* pb_rank = reinterpret_cast<int*>(pb_w + npb);
  int* goff = pb_rank + npb;  // group a's rank prefix sums at a (nq + 1)

  const uint32_t bar_addr = (uint32_t)__cvta_generic_to_shared(bar);
  if (tid == 0) {
    *abort_flag = 0;
    mbar_init(bar_addr, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }

  // X hi / lo: row tid, frame group fg -> (tid / 8) * SBO + fg * 128 + (tid % 8) * 16
  const uint32_t sbox = (uint32_t)Tk * 32, sbov = (uint32_t)TN * 32, sbot = (uint32_t)C * 32;
  {
    float4 xv[TN / 4];
#pragma unroll
    for (int fg = 0; fg < TN / 4; ++fg)
      xv[fg] = (valid && 4 * fg < T) ? __ldg(reinterpret_cast<const float4*>(xc + row * T) + fg)
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int fg = 0; fg < TN / 4; ++fg) {
      if (4 * fg >= Tk) break;
      uint4 h, l;
      rtc_split4(xv[fg], h, l);
      const uint32_t off = (uint32_t)(tid >> 3) * sbox + (uint32_t)fg * 128 + (uint32_t)(tid & 7) * 16;
      *reinterpret_cast<uint4*>(Xhi + off) = h;
      *reinterpret_cast<uint4*>(Xhi + xb + off) = l;
    }
  }
  // the brick's patches: index, rank, weight, cover mask
  for (int idx = tid; idx < npb; idx += kRtcThreads) {
    const int a = idx / nq, q = idx - a * nq;
    const int cj = jlo + q / nk, ck = klo + q % nk;
    const long long pid = ((long long)(ilo + a) * g.ncy + cj) * g.ncz + ck;
    pb_pid[idx] = pid;
    pb_rank[idx] = __ldg(ranks + pid);
    pb_w[idx] = __ldg(wgt + pid);
    pb_mask[idx] = rtc_axis_mask(tab.corners[0][ilo + a], g.px, x0, kRtcBX) |
                   (rtc_axis_mask(tab.corners[1][cj], g.py, y0, kRtcBY) << 4) |
                   (rtc_axis_mask(tab.corners[2][ck], g.pz, z0, kRtcBZ) << 8);
  }
  // the reconstruction sums (FP32, round to nearest) and the weight sum
  // (float64: exact), continuing a lower slab's partial sums
  float acc[TN];
#pragma unroll
  for (int f = 0; f < TN; ++f) acc[f] = 0.f;
  double wsum = 0.0;
  if (valid && x < io.hin && io.halo_in != nullptr) {
    const double* hp = io.halo_in + row * (T + 1);
#pragma unroll
    for (int f = 0; f < TN; ++f)
      if (f < T) acc[f] = (float)hp[f];
    wsum = hp[T];
  }
  __syncthreads();  // patch table written
  if (valid) {  // weights of the covering patches, all inside the brick's box
    const int cxlo = tab.cover[0][2 * x], cxhi = tab.cover[0][2 * x + 1];
    const int cylo = tab.cover[1][2 * y], cyhi = tab.cover[1][2 * y + 1];
    const int czlo = tab.cover[2][2 * z], czhi = tab.cover[2][2 * z + 1];
    for (int i = cxlo; i <= cxhi; ++i)
      for (int j = cylo; j <= cyhi; ++j) {
        const float* wr = pb_w + (i - ilo) * nq + (j - jlo) * nk - klo;
        for (int k = czlo; k <= czhi; ++k) wsum += (double)wr[k];
      }
  }
  if (warp == 0) {  // each x-corner group's rank prefix sums
    for (int a = 0; a < ni; ++a) {
      int* qo = goff + a * (nq + 1);
      int carry = 0;
      for (int q0 = 0; q0 < nq; q0 += 32) {
        const int q = q0 + lane;
        int sc = q < nq ? pb_rank[a * nq + q] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, sc, o);
          if (lane >= o) sc += t;
        }
        if (q < nq) qo[q + 1] = carry + sc;
        carry += __shfl_sync(0xffffffffu, sc, 31);
      }
      if (lane == 0) qo[0] = 0;
    }
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's lane quarter
  const uint32_t xhi_a = (uint32_t)__cvta_generic_to_shared(Xhi);
  const uint32_t vhi_a = (uint32_t)__cvta_generic_to_shared(Vhi);
  const uint32_t thi_a = (uint32_t)__cvta_generic_to_shared(Thi);
  constexpr uint32_t idesc1 = rtc_idesc(C), idesc2 = rtc_idesc(TN);
  uint32_t phase = 0;  // parity of the barrier's next phase
  bool pend = false;   // thread 0: a commit in flight
  uint32_t pend_phase = 0;

  // Commits the MMAs issued so far (thread 0) and waits for them (every
  // thread, bounded); a wait that gives up sets the abort flag.
  auto commit = [&]() {
    if (tid == 0) {
      umma_commit(bar_addr);
      pend = true;
      pend_phase = phase;
    }
  };
  auto wait = [&]() {
    if (!mbar_wait_bounded(bar_addr, phase, status, kStatusMmaTimeout))
      *abort_flag = 1;
    else if (tid == 0)
      pend = false;
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  };
  // chunk iterator: x-corner group a, first column c0 (a == ni: done)
  auto ncol_of = [&](int a) { return goff[a * (nq + 1) + nq]; };
  auto advance = [&](int& a, int& c0) {
    c0 += C;
    while (a < ni && c0 >= ncol_of(a)) {
      ++a;
      c0 = 0;
    }
  };
  // column table of chunk (a, c0) into table buffer tb (threads < C)
  auto table = [&](int a, int c0, int tb) {
    if (tid < C) {
      const int* qo = goff + a * (nq + 1);
      const int ncol = qo[nq];
      const int col = c0 + tid;
      long long ro = -1;
      uint32_t m = 0;
      float w = 0.f;
      if (col < ncol) {
        int lo = 0, hi = nq - 1;  // largest q with qo[q] <= col: the patch holding the column
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (qo[mid] <= col)
            lo = mid;
          else
            hi = mid - 1;
        }
        const int idx = a * nq + lo;
        ro = pb_pid[idx] * T * T + (long long)(col - qo[lo]) * T;
        m = pb_mask[idx];
        w = pb_w[idx];
      }
      c_row[tb * C + tid] = ro;
      c_mask[tb * C + tid] = m;
      c_w[tb * C + tid] = w;
    }
  };
  // the chunk's eigenvector rows into registers: item e = tid + 128 i ->
  // column e % C, frame group e / C
  float4 vr[ITEMS];
  auto fetch = [&](int tb) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int e = tid + kRtcThreads * i, pos = e % C, fg = e / C;
      const long long ro = c_row[tb * C + pos];
      vr[i] = (ro >= 0 && 4 * fg < T) ? __ldg(reinterpret_cast<const float4*>(vecs + ro) + fg)
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };

  int ca = 0, cc0 = 0;  // current chunk
  while (ca < ni && ncol_of(ca) == 0) ++ca;
  int tb = 0;
  if (ca < ni) {
    table(ca, cc0, 0);
    __syncthreads();
    fetch(0);
  }
  while (ca < ni) {
    // 1. V (rows = columns) hi / lo from the fetched rows, and a raw copy
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int e = tid + kRtcThreads * i, pos = e % C, fg = e / C;
      uint4 h, l;
      rtc_split4(vr[i], h, l);
      const uint32_t off = (uint32_t)(pos >> 3) * sbov + (uint32_t)fg * 128 + (uint32_t)(pos & 7) * 16;
      *reinterpret_cast<uint4*>(Vhi + off) = h;
      *reinterpret_cast<uint4*>(Vhi + vb + off) = l;
      *reinterpret_cast<float4*>(raw + pos * RS + 4 * fg) = vr[i];
    }
    __syncthreads();
    // V^T (rows = frames): frame f, column group cg -> (f / 8) * SBO + cg * 128 + (f % 8) * 16
#pragma unroll
    for (int i = 0; i < TITEMS; ++i) {
      const int e = tid + kRtcThreads * i, f = e % TN, cg = e / TN;
      uint4 h, l;
      rtc_split4(make_float4(raw[(4 * cg) * RS + f], raw[(4 * cg + 1) * RS + f], raw[(4 * cg + 2) * RS + f],
                             raw[(4 * cg + 3) * RS + f]),
                 h, l);
      const uint32_t off = (uint32_t)(f >> 3) * sbot + (uint32_t)cg * 128 + (uint32_t)(f & 7) * 16;
      *reinterpret_cast<uint4*>(Thi + off) = h;
      *reinterpret_cast<uint4*>(Thi + vb + off) = l;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    // 2. GEMM 1: hi.hi into [0, C), hi.lo + lo.hi into [C, 2C)
    if (tid == 0) rtc_issue_gemm1(tmem, xhi_a, (uint32_t)xb, sbox, vhi_a, (uint32_t)vb, sbov, Tk, idesc1);
    commit();
    // while it runs: the next chunk's table and its rows in flight
    int na = ca, nc0 = cc0;
    advance(na, nc0);
    if (na < ni) table(na, nc0, tb ^ 1);
    __syncthreads();
    if (na < ni) fetch(tb ^ 1);
    wait();
    // 3. Y~ = S o Y, split: hi over [0, C), lo over [C, 2C)
    const uint32_t* sm = c_mask + tb * C;
    const float* sw = c_w + tb * C;
#pragma unroll 1
    for (int j = 0; j < C; j += 16) {
      uint32_t dh[16], dx[16];
      tmem_ld16_nowait(tl + (uint32_t)j, dh);
      tmem_ld16_nowait(tl + (uint32_t)(C + j), dx);
      tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float sc = ((sm[j + i] & vbits) == vbits) ? sw[j + i] : 0.f;
        const float yv = __fmul_rn(__fadd_rn(__uint_as_float(dh[i]), __uint_as_float(dx[i])), sc);
        dh[i] = tf32_rna(yv);
        dx[i] = tf32_rna(__fsub_rn(yv, __uint_as_float(dh[i])));
      }
      tmem_st16(tl + (uint32_t)j, dh);
      tmem_st16(tl + (uint32_t)(C + j), dx);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (*abort_flag) break;  // uniform
    // 4. GEMM 2: K step s -> its own accumulator [2C + s TN, 2C + (s + 1) TN)
    if (tid == 0) rtc_issue_gemm2(tmem, thi_a, (uint32_t)vb, sbot, TN, idesc2);
    commit();
    wait();
    // 5. the K steps' sums into the accumulator ((s0 + s1) + (s2 + s3), then added)
#pragma unroll
    for (int f0 = 0; f0 < TN; f0 += 8) {
      uint32_t r[KS2][8];
#pragma unroll
      for (int ks = 0; ks < KS2; ++ks) tmem_ld8_nowait(tl + (uint32_t)(2 * C + ks * TN + f0), r[ks]);
      tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float a01 = __fadd_rn(__uint_as_float(r[0][i]), __uint_as_float(r[1][i]));
        const float a23 = __fadd_rn(__uint_as_float(r[2][i]), __uint_as_float(r[3][i]));
        acc[f0 + i] = __fadd_rn(acc[f0 + i], __fadd_rn(a01, a23));
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();  // V, V^T, the raw rows and the TMEM columns are free for the next chunk
    if (*abort_flag) break;
    ca = na;
    cc0 = nc0;
    tb ^= 1;
  }
  __syncthreads();
  if (!*abort_flag && valid) {
    if (x >= io.own_hi) {  // the next slab's halo: unnormalised sums in patch order
      double* hp = io.halo_out + (row - (long long)io.own_hi * g.ny * g.nz) * (T + 1);
#pragma unroll
      for (int f = 0; f < TN; ++f)
        if (f < T) hp[f] = (double)acc[f];
      hp[T] = wsum;
    } else {
      // out = m + A / wsum; a voxel no patch covers gets 0, as 0 / max(0, 1e-12)
      const double inv = wsum > 0.0 ? 1.0 / wsum : 0.0;
      const double mm = wsum > 0.0 ? (double)mean[row] : 0.0;
      float4* op = reinterpret_cast<float4*>(out + row * T);
#pragma unroll
      for (int f = 0; f < TN; f += 4)
        if (f < T)
          op[f / 4] = make_float4((float)(mm + (double)acc[f] * inv), (float)(mm + (double)acc[f + 1] * inv),
                                  (float)(mm + (double)acc[f + 2] * inv), (float)(mm + (double)acc[f + 3] * inv));
    }
  }
  if (*abort_flag && tid == 0 && pend)  // let the MMAs in flight finish before the TMEM is released
    mbar_wait_bounded(bar_addr, pend_phase, status, kStatusMmaTimeout);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
}

template <int TN>
__global__ void __launch_bounds__(kRtcThreads, 2)
    recon_tc_kernel(const float* __restrict__ xc, const float* __restrict__ mean, const float* __restrict__ vecs,
                    const int32_t* __restrict__ ranks, const float* __restrict__ wgt, float* __restrict__ out, Geom g,
                    AxisTables tab, int brick0, SlabIO io, int* status) {
  recon_tc_body<TN>(xc, mean, vecs, ranks, wgt, out, g, tab, brick0, io, status, (int)blockIdx.x);
}

}  // namespace lrd
