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
//    into a per-voxel float64 accumulator in registers.
// The weight sums are float64 (exact: a few hundred float32 values 1/(2+p)).
//
// Columns are taken in groups of one x corner index (every touching patch
// (i, j, k) of the brick with the same i, j-major then k, then the patch's
// eigenvectors in order), each group cut into chunks of kRtcChunk columns
// (the last one zero-padded). A chunk never mixes two x corners, so a voxel's
// float64 sum is the same sequence of additions whichever x-slab computes
// which of its patches: a slab that hands its partial sums on (SlabIO halo)
// and the next slab that continues from them give bit-identical results to
// one unsharded call.
//
// Per chunk (128 threads, thread v = voxel v = TMEM lane v):
//   1. column table (eigenvector row, cover mask, weight) and the chunk's
//      eigenvector rows, split hi / lo into shared memory twice: as GEMM 1's
//      B (rows = columns, K = frames) and transposed as GEMM 2's B (rows =
//      frames, K = columns), both K-major (an MN-major B operand of kind::tf32
//      read back zeros here);
//   2. GEMM 1 into TMEM columns [0, C) (hi.hi) and [C, 2C) (cross terms);
//   3. each thread reads its row of Y, scales it by S, splits it and writes
//      Y~ hi / lo over the same columns (GEMM 2's A operand, in TMEM);
//   4. GEMM 2, K step s into columns [2C + s Tn, 2C + (s + 1) Tn);
//   5. each thread adds the K steps' sums into its float64 accumulator.
// The X tiles are split into shared memory once per brick; two CTAs share an
// SM (T <= 48: 256 TMEM columns and about 74 KB of shared memory each).
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
// matrices), V hi, V lo (C rows x Tn), V^T hi, V^T lo (Tn rows x C), the
// chunk's column table (C x {row offset (8), mask (4), weight (4)}),
// mbarrier, TMEM address, abort flag, the group's rank prefix sums (qcap + 1
// ints).
__host__ __device__ inline size_t recon_tc_xbytes(int T) { return (size_t)128 * recon_tc_tk(T) * 4; }
__host__ __device__ inline size_t recon_tc_vbytes(int T) { return (size_t)kRtcChunk * recon_tc_tn(T) * 4; }
__host__ __device__ inline size_t recon_tc_smem_bytes(int T, int qcap) {
  return 2 * recon_tc_xbytes(T) + 4 * recon_tc_vbytes(T) + (size_t)kRtcChunk * 16 + 16 + (size_t)4 * (qcap + 1);
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
// TN = recon_tc_tn(T): the per-voxel float64 accumulator lives in registers.
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
  constexpr uint32_t kCols = recon_tc_tmem_cols(TN);
  extern __shared__ __align__(1024) unsigned char smr[];
  const int T = g.nt;
  const int Tk = recon_tc_tk(T);
  const size_t xb = recon_tc_xbytes(T), vb = recon_tc_vbytes(T);
  unsigned char* Xhi = smr;
  unsigned char* Vhi = smr + 2 * xb;
  unsigned char* Thi = Vhi + 2 * vb;                               // V^T hi, lo
  long long* c_row = reinterpret_cast<long long*>(Thi + 2 * vb);  // eigenvector row offset, -1 = padding
  uint32_t* c_mask = reinterpret_cast<uint32_t*>(c_row + C);      // cover bits: x (4) | y (4) << 4 | z (8) << 8
  float* c_w = reinterpret_cast<float*>(c_mask + C);              // patch weight
  uint64_t* bar = reinterpret_cast<uint64_t*>(c_w + C);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  int* qoff = abort_flag + 1;  // group rank prefix sums, nq + 1
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
  const int nk = khi - klo + 1, nq = (jhi - jlo + 1) * nk;

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
  for (int fg = 0; fg < Tk / 4; ++fg) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid && 4 * fg < T) v = __ldg(reinterpret_cast<const float4*>(xc + row * T) + fg);
    uint4 h, l;
    rtc_split4(v, h, l);
    const uint32_t off = (uint32_t)(tid >> 3) * sbox + (uint32_t)fg * 128 + (uint32_t)(tid & 7) * 16;
    *reinterpret_cast<uint4*>(Xhi + off) = h;
    *reinterpret_cast<uint4*>(Xhi + xb + off) = l;
  }
  // float64 sums: weights over the covering patches (exact) and the
  // reconstruction, continuing a lower slab's partial sums
  double acc[TN];
#pragma unroll
  for (int f = 0; f < TN; ++f) acc[f] = 0.0;
  double wsum = 0.0;
  if (valid && x < io.hin && io.halo_in != nullptr) {
    const double* hp = io.halo_in + row * (T + 1);
#pragma unroll
    for (int f = 0; f < TN; ++f)
      if (f < T) acc[f] = hp[f];
    wsum = hp[T];
  }
  if (valid) {
    const int cxlo = tab.cover[0][2 * x], cxhi = tab.cover[0][2 * x + 1];
    const int cylo = tab.cover[1][2 * y], cyhi = tab.cover[1][2 * y + 1];
    const int czlo = tab.cover[2][2 * z], czhi = tab.cover[2][2 * z + 1];
    for (int i = cxlo; i <= cxhi; ++i)
      for (int j = cylo; j <= cyhi; ++j) {
        const long long p0 = ((long long)i * g.ncy + j) * g.ncz;
        for (int k = czlo; k <= czhi; ++k) wsum += (double)__ldg(wgt + p0 + k);
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
  constexpr int NG = TN / 4;  // frame groups of a V row

  // Issues the MMAs of one step (thread 0), commits them to the barrier and
  // waits (every thread, bounded); a wait that gives up sets the abort flag.
  auto commit_wait = [&]() {
    if (tid == 0) {
      umma_commit(bar_addr);
      pend = true;
      pend_phase = phase;
    }
    if (!mbar_wait_bounded(bar_addr, phase, status, kStatusMmaTimeout))
      *abort_flag = 1;
    else if (tid == 0)
      pend = false;
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  };

  for (int ci = ilo; ci <= ihi; ++ci) {
    // the group's rank prefix sums (j-major, k inner)
    __syncthreads();  // the previous group's table is no longer read
    if (warp == 0) {
      int carry = 0;
      for (int q0 = 0; q0 < nq; q0 += 32) {
        const int q = q0 + lane;
        int r = 0;
        if (q < nq) r = __ldg(ranks + ((long long)ci * g.ncy + jlo + q / nk) * g.ncz + klo + q % nk);
        int sc = r;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, sc, o);
          if (lane >= o) sc += t;
        }
        if (q < nq) qoff[q + 1] = carry + sc;
        carry += __shfl_sync(0xffffffffu, sc, 31);
      }
      if (lane == 0) qoff[0] = 0;
    }
    __syncthreads();
    if (*abort_flag) break;  // uniform: set before the barrier above
    const int ncol = qoff[nq];
    const uint32_t xmask = rtc_axis_mask(tab.corners[0][ci], g.px, x0, kRtcBX);
    for (int c0 = 0; c0 < ncol; c0 += C) {
      // 1. the chunk's column table, then its eigenvector rows split into V hi / lo
      if (tid < C) {
        const int c = c0 + tid;
        long long ro = -1;
        uint32_t m = 0;
        float w = 0.f;
        if (c < ncol) {
          int lo = 0, hi = nq - 1;  // largest q with qoff[q] <= c: the patch holding column c
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (qoff[mid] <= c)
              lo = mid;
            else
              hi = mid - 1;
          }
          const int cj = jlo + lo / nk, ck = klo + lo % nk;
          const long long pid = ((long long)ci * g.ncy + cj) * g.ncz + ck;
          ro = pid * T * T + (long long)(c - qoff[lo]) * T;
          m = xmask | (rtc_axis_mask(tab.corners[1][cj], g.py, y0, kRtcBY) << 4) |
              (rtc_axis_mask(tab.corners[2][ck], g.pz, z0, kRtcBZ) << 8);
          w = __ldg(wgt + pid);
        }
        c_row[tid] = ro;
        c_mask[tid] = m;
        c_w[tid] = w;
      }
      __syncthreads();
      // column pos, frame group fg -> (pos / 8) * SBO + fg * 128 + (pos % 8) * 16
      for (int e = tid; e < C * NG; e += kRtcThreads) {
        const int pos = e % C, fg = e / C;
        const long long ro = c_row[pos];
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ro >= 0 && 4 * fg < T) v = __ldg(reinterpret_cast<const float4*>(vecs + ro) + fg);
        uint4 h, l;
        rtc_split4(v, h, l);
        const uint32_t off = (uint32_t)(pos >> 3) * sbov + (uint32_t)fg * 128 + (uint32_t)(pos & 7) * 16;
        *reinterpret_cast<uint4*>(Vhi + off) = h;
        *reinterpret_cast<uint4*>(Vhi + vb + off) = l;
      }
      // V^T: frame f, column group cg -> (f / 8) * SBO + cg * 128 + (f % 8) * 16
      for (int e = tid; e < TN * (C / 4); e += kRtcThreads) {
        const int f = e % TN, cg = e / TN;
        float vv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const long long ro = c_row[4 * cg + i];
          vv[i] = (ro >= 0 && f < T) ? __ldg(vecs + ro + f) : 0.f;
        }
        uint4 h, l;
        rtc_split4(make_float4(vv[0], vv[1], vv[2], vv[3]), h, l);
        const uint32_t off = (uint32_t)(f >> 3) * sbot + (uint32_t)cg * 128 + (uint32_t)(f & 7) * 16;
        *reinterpret_cast<uint4*>(Thi + off) = h;
        *reinterpret_cast<uint4*>(Thi + vb + off) = l;
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncthreads();
      // 2. GEMM 1: hi.hi into [0, C), hi.lo + lo.hi into [C, 2C)
      if (tid == 0) rtc_issue_gemm1(tmem, xhi_a, (uint32_t)xb, sbox, vhi_a, (uint32_t)vb, sbov, Tk, idesc1);
      commit_wait();
      // 3. Y~ = S o Y, split: hi over [0, C), lo over [C, 2C)
#pragma unroll 1
      for (int j = 0; j < C; j += 16) {
        uint32_t dh[16], dx[16];
        tmem_ld16_nowait(tl + (uint32_t)j, dh);
        tmem_ld16_nowait(tl + (uint32_t)(C + j), dx);
        tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const float sc = ((c_mask[j + i] & vbits) == vbits) ? c_w[j + i] : 0.f;
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
      commit_wait();
      // 5. the K steps' sums into the float64 accumulator ((s0 + s1) + (s2 + s3) in FP32)
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
          acc[f0 + i] += (double)__fadd_rn(a01, a23);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncthreads();  // V, the column table and the TMEM columns are free for the next chunk
      if (*abort_flag) break;
    }
    if (*abort_flag) break;  // uniform: read after the chunk loop's last barrier
  }
  __syncthreads();
  if (!*abort_flag && valid) {
    if (x >= io.own_hi) {  // the next slab's halo: unnormalised sums in patch order
      double* hp = io.halo_out + (row - (long long)io.own_hi * g.ny * g.nz) * (T + 1);
#pragma unroll
      for (int f = 0; f < TN; ++f)
        if (f < T) hp[f] = acc[f];
      hp[T] = wsum;
    } else {
      // out = m + A / wsum; a voxel no patch covers gets 0, as 0 / max(0, 1e-12)
      const double inv = wsum > 0.0 ? 1.0 / wsum : 0.0;
      const double mm = wsum > 0.0 ? (double)mean[row] : 0.0;
      float4* op = reinterpret_cast<float4*>(out + row * T);
#pragma unroll
      for (int f = 0; f < TN; f += 4)
        if (f < T)
          op[f / 4] = make_float4((float)(mm + acc[f] * inv), (float)(mm + acc[f + 1] * inv),
                                  (float)(mm + acc[f + 2] * inv), (float)(mm + acc[f + 3] * inv));
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
