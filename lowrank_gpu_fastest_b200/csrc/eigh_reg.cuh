// Register-resident float32 eigensolver for T <= TMAX (TMAX in {32, 48, 64}).
//
// One warp per matrix: Householder tridiagonalisation, bisection on Sturm
// counts, MP rank (mp_rank, eigh.cuh), inverse iteration, back-transform,
// Gram-Schmidt (the steps of eigh_mp_block, eigh.cuh), with the data placed
// for a warp:
//
//  * lane l holds rows l and l + 32 of the working matrix in registers
//    (a[NR][TMAX], every column index compile-time), so the reflector's
//    matrix-vector product and the rank-2 update touch no shared memory for
//    the matrix itself; at step k the owner of row k broadcasts it through
//    shared memory, which (by symmetry) is column k;
//  * the reflector vectors are kept in shared memory (HV, one row per step,
//    zero above the sub-diagonal and 1 on it) and double as the broadcast
//    buffer of the matrix-vector product; row k is stored packed, from its
//    first live 4-column group (4 * ((k + 1) >> 2)) on, which halves HV;
//  * inverse iteration keeps its vector and the LU factors in shared memory
//    and the pivot swaps as bits of a register (one lane per eigenvector);
//  * the back-transform and the Gram-Schmidt pass work on row-distributed
//    vectors with warp reductions, 8 vectors at a time.
//
// The near-tie test (mp_rank's margin) queues patches for the float64 pass.
#pragma once

#include "eigh.cuh"

namespace lrd {

#ifdef LRD_PHASE_CLOCKS
__device__ long long* g_phase_clocks;  // 8 stamps per block, set by a probe build
#define LRD_STAMP(i) \
  do { __syncwarp(); if ((threadIdx.x & 31) == 0) g_phase_clocks[(long long)blockIdx.x * 8 + (i)] = clock64(); } while (0)
#else
#define LRD_STAMP(i) \
  do { } while (0)
#endif

template <int TMAX>
__host__ __device__ constexpr int eigh_reg_nr() {
  return (TMAX + 31) / 32;
}

// Shared-memory floats per warp: packed HV, d, e, e2, tau, lam (5 TMAX), LU /
// MP scratch (3 TMAX kInvGroup; during the tridiagonalisation the row-k
// broadcast and the w vector), vector transpose buffer (TMAX x kLdy).
template <int TMAX>
__host__ __device__ constexpr size_t eigh_reg_smem_floats() {
  return eigh_hv_floats<TMAX>() + 5 * TMAX + (size_t)3 * TMAX * kInvGroup + (size_t)TMAX * kLdy;
}

template <int V>
struct IntTag {
  static constexpr int value = V;
};

// Sums of G = 4 or 8 values over the warp, every lane getting all G sums:
// halving exchanges (each lane keeps half of its values and adds its
// partner's copies of them: G/2 + G/4 + ... shuffles) until a lane holds one
// value summed over 8 (G = 8) or 16 (G = 4) lanes, two or one more xor steps
// finish it over the warp, then G broadcasts - G + 8 shuffles for G = 8
// against 5 G for a butterfly per value.
template <int G>
__device__ __forceinline__ void warp_allsum(float (&v)[G]) {
  static_assert(G == 4 || G == 8, "4 or 8 values");
  const int lane = threadIdx.x & 31;
  const bool b4 = (lane >> 4) & 1, b3 = (lane >> 3) & 1, b2 = (lane >> 2) & 1;
  float w;
  if constexpr (G == 8) {
    float w4[4], w2[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float keep = b4 ? v[i + 4] : v[i], send = b4 ? v[i] : v[i + 4];
      w4[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float keep = b3 ? w4[i + 2] : w4[i], send = b3 ? w4[i] : w4[i + 2];
      w2[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const float keep = b2 ? w2[1] : w2[0], send = b2 ? w2[0] : w2[1];
    w = keep + __shfl_xor_sync(0xffffffffu, send, 4);  // value 4 b4 + 2 b3 + b2
  } else {
    float w2[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float keep = b4 ? v[i + 2] : v[i], send = b4 ? v[i] : v[i + 2];
      w2[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    const float keep = b3 ? w2[1] : w2[0], send = b3 ? w2[0] : w2[1];
    w = keep + __shfl_xor_sync(0xffffffffu, send, 8);  // value 2 b4 + b3
    w += __shfl_xor_sync(0xffffffffu, w, 4);
  }
  w += __shfl_xor_sync(0xffffffffu, w, 2);
  w += __shfl_xor_sync(0xffffffffu, w, 1);
#pragma unroll
  for (int q = 0; q < G; ++q)  // value q sits in lane (q's bits spread to lane bits 4, 3, 2 / 4, 3)
    v[q] = __shfl_sync(0xffffffffu, w, G == 8 ? (((q & 4) << 2) | ((q & 2) << 2) | ((q & 1) << 2))
                                              : (((q & 2) << 3) | ((q & 1) << 3)));
}

// Sturm counts (eigenvalues below x0 and x1) of the tridiagonal held in
// registers: dr[i] = d_i, e2r[i] = e_i^2. Entries i >= n are padded with
// d_i = +big, e_i = 0, which adds positive pivots only, so the counts equal
// the n x n ones. The pivots follow q_i = (d_i - x) - e_{i-1}^2 / q_{i-1}, a
// pivot smaller than pivmin in magnitude replaced by -pivmin; the count is
// the number of negative pivots (their sign bits: no pivot is a zero).
template <int TMAX>
__device__ __forceinline__ void sturm2_reg(const float (&dr)[TMAX], const float (&e2r)[TMAX], float x0, float x1,
                                           float pivmin, int& c0, int& c1) {
  float q0 = dr[0] - x0, q1 = dr[0] - x1;
  if (fabsf(q0) < pivmin) q0 = -pivmin;
  if (fabsf(q1) < pivmin) q1 = -pivmin;
  int a0 = (int)(__float_as_uint(q0) >> 31), a1 = (int)(__float_as_uint(q1) >> 31);
#pragma unroll
  for (int i = 1; i < TMAX; ++i) {
    q0 = (dr[i] - x0) - __fdividef(e2r[i - 1], q0);
    q1 = (dr[i] - x1) - __fdividef(e2r[i - 1], q1);
    if (fabsf(q0) < pivmin) q0 = -pivmin;
    if (fabsf(q1) < pivmin) q1 = -pivmin;
    a0 += (int)(__float_as_uint(q0) >> 31);
    a1 += (int)(__float_as_uint(q1) >> 31);
  }
  c0 = a0;
  c1 = a1;
}

// All eigenvalues of the tridiagonal (d, e, e2 in shared memory) ascending
// into lam; tnorm = Gerschgorin bound. Bisection (an interval [lo, hi] with
// count(lo) <= j < count(hi), stopped at max(eps tnorm, 2 eps |lambda|): the
// absolute part is LAPACK's default tolerance (eps times the norm of the
// tridiagonal), below the float32 reduction's own error in the eigenvalues)
// with the tridiagonal in registers and one multisection pass first: the 64
// chains evaluate counts at 64 evenly spaced interior points of the
// Gerschgorin interval, and every chain starts from the two neighbouring
// points that bracket its eigenvalue (six bisection steps for the price of
// one). For TMAX <= 32 each lane owns one eigenvalue and its two chains
// trisect it.
template <int TMAX>
__device__ __forceinline__ void bisect_reg(const float* d, const float* e, const float* e2, float* lam, int n,
                                           float& tnorm_out) {
  const int lane = threadIdx.x & 31;
  const float eps = Num<float>::eps();
  float glo = FLT_MAX, ghi = -FLT_MAX;
  for (int i = lane; i < n; i += 32) {
    const float r = (i > 0 ? fabsf(e[i - 1]) : 0.f) + (i < n - 1 ? fabsf(e[i]) : 0.f);
    glo = fminf(glo, d[i] - r);
    ghi = fmaxf(ghi, d[i] + r);
  }
  glo = warp_min(glo);
  ghi = warp_max(ghi);
  const float tnorm = fmaxf(fmaxf(fabsf(glo), fabsf(ghi)), FLT_MIN);
  glo -= 4.f * eps * tnorm * n;
  ghi += 4.f * eps * tnorm * n;
  const float pivmin = FLT_MIN * 4.f;
  const float abstol = eps * tnorm;
  const float big = 4.f * fmaxf(fabsf(glo), fabsf(ghi)) + 1.f;
  float dr[TMAX], e2r[TMAX];
#pragma unroll
  for (int i = 0; i < TMAX; ++i) {
    dr[i] = i < n ? d[i] : big;
    e2r[i] = i < n - 1 ? e2[i] : 0.f;
  }
  // multisection: counts at y_m = glo + (m + 1) h, m = lane and lane + 32
  const float h = (ghi - glo) * (1.f / 65.f);
  int cm0, cm1;
  sturm2_reg<TMAX>(dr, e2r, fmaf((float)(lane + 1), h, glo), fmaf((float)(lane + 33), h, glo), pivmin, cm0, cm1);
  const int j0 = lane, j1 = lane + 32;
  float lo0 = glo, hi0 = ghi, lo1 = glo, hi1 = ghi;
#pragma unroll 4
  for (int m = 0; m < 32; ++m) {
    const int ca = __shfl_sync(0xffffffffu, cm0, m), cb = __shfl_sync(0xffffffffu, cm1, m);
    const float ya = fmaf((float)(m + 1), h, glo), yb = fmaf((float)(m + 33), h, glo);
    if (ca <= j0) lo0 = fmaxf(lo0, ya); else hi0 = fminf(hi0, ya);
    if (cb <= j0) lo0 = fmaxf(lo0, yb); else hi0 = fminf(hi0, yb);
    if (ca <= j1) lo1 = fmaxf(lo1, ya); else hi1 = fminf(hi1, ya);
    if (cb <= j1) lo1 = fmaxf(lo1, yb); else hi1 = fminf(hi1, yb);
  }
  if (!(lo0 < hi0)) { lo0 = glo; hi0 = ghi; }  // counts not monotone: full interval
  if (!(lo1 < hi1)) { lo1 = glo; hi1 = ghi; }
  const bool has0 = j0 < n, has1 = j1 < n;
  if constexpr (TMAX <= 32) {
    // One eigenvalue per lane: the second chain evaluates a second point, so
    // a step cuts the interval in three (12 instead of 18 steps from the
    // multisection's interval to the tolerance).
    bool run = has0;
    for (int it = 0; it < 200 && run; ++it) {
      const float tol = fmaxf(abstol, 2.f * eps * fmaxf(fabsf(lo0), fabsf(hi0)));
      const float w3 = (hi0 - lo0) * (1.f / 3.f);
      const float ma = lo0 + w3, mb = hi0 - w3;
      run = hi0 - lo0 > tol && ma > lo0 && ma < mb && mb < hi0;
      if (!run) break;
      int ca, cb;
      sturm2_reg<TMAX>(dr, e2r, ma, mb, pivmin, ca, cb);
      if (ca > j0) {
        hi0 = ma;
      } else if (cb > j0) {
        lo0 = ma;
        hi0 = mb;
      } else {
        lo0 = mb;
      }
    }
    if (has0) lam[j0] = 0.5f * (lo0 + hi0);
    __syncwarp();
    tnorm_out = tnorm;
    return;
  }
  bool run0 = has0, run1 = has1;
  for (int it = 0; it < 200 && (run0 || run1); ++it) {
    if (run0) {
      const float tol = fmaxf(abstol, 2.f * eps * fmaxf(fabsf(lo0), fabsf(hi0)));
      const float mid = 0.5f * (lo0 + hi0);
      run0 = hi0 - lo0 > tol && mid > lo0 && mid < hi0;
    }
    if (run1) {
      const float tol = fmaxf(abstol, 2.f * eps * fmaxf(fabsf(lo1), fabsf(hi1)));
      const float mid = 0.5f * (lo1 + hi1);
      run1 = hi1 - lo1 > tol && mid > lo1 && mid < hi1;
    }
    if (!run0 && !run1) break;
    const float m0 = 0.5f * (lo0 + hi0), m1 = 0.5f * (lo1 + hi1);
    int c0, c1;
    sturm2_reg<TMAX>(dr, e2r, m0, m1, pivmin, c0, c1);
    if (run0) {
      if (c0 > j0) hi0 = m0; else lo0 = m0;
    }
    if (run1) {
      if (c1 > j1) hi1 = m1; else lo1 = m1;
    }
  }
  if (has0) lam[j0] = 0.5f * (lo0 + hi0);
  if (has1) lam[j1] = 0.5f * (lo1 + hi1);
  __syncwarp();
  tnorm_out = tnorm;
}

// For TMAX in (32, 48] the rows 32..TMAX-1 are held as half-rows: lane l
// holds row l whole and, of row 32 + (l & 15), the columns 4J + 2h and
// 4J + 2h + 1 of every 4-column group J (h = l >> 4), so 1.5 rows of
// registers per lane instead of 2 (72 instead of 96 at TMAX 48: more warps
// per SM). Every FMA chain of the two-row layout stays in one lane in the
// same order - the matvec's column-residue accumulators s0, s1 (h = 0) and
// s2, s3 (h = 1), each element's rank-2 update - and the half-row sum is
// (s0 + s1) + (s2 + s3) after one exchange, so the reduction is
// bit-identical to the two-row layout's.
template <int TMAX>
__host__ __device__ constexpr bool eigh_reg_half() {
  return TMAX > 32 && TMAX <= 48 && TMAX % 4 == 0;
}

// Load (exact power-of-two scaling) and Householder tridiagonalisation in the
// half-row layout: d, e, tau and the packed reflector rows HV as the two-row
// code writes them; returns the unscaling factor and the end of the packed
// rows. xk and ws are the row-broadcast and w vectors (TMAX floats each).
template <int TMAX>
__device__ __forceinline__ void tridiag_half(const float* G, int n, float* HV, float* d, float* e, float* tau,
                                             float* xk, float* ws, float& unscale_out, int& hbase_out) {
  constexpr int NG = TMAX / 4;  // 4-column groups
  const int lane = threadIdx.x & 31;
  const int h = lane >> 4;
  const int r1 = 32 + (lane & 15);
  const bool v0 = lane < n, v1 = r1 < n;
  float a0[TMAX], a1[TMAX / 2];
  float dmax = 0.f;
#pragma unroll
  for (int j = 0; j < TMAX; ++j) a0[j] = (v0 && j < n) ? G[(long long)lane * n + j] : 0.f;
#pragma unroll
  for (int J = 0; J < NG; ++J)
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int c = 4 * J + 2 * h + t;
      a1[2 * J + t] = (v1 && c < n) ? G[(long long)r1 * n + c] : 0.f;
    }
  if (v0) dmax = fmaxf(dmax, fabsf(G[(long long)lane * n + lane]));
  if (v1) dmax = fmaxf(dmax, fabsf(G[(long long)r1 * n + r1]));
  dmax = warp_max(dmax);
  int ex = 0;
  if (dmax > 0.f && isfinite(dmax)) frexpf(dmax, &ex);
  const float scale = ldexpf(1.f, -ex);
  unscale_out = ldexpf(1.f, ex);
#pragma unroll
  for (int j = 0; j < TMAX; ++j) a0[j] *= scale;
#pragma unroll
  for (int j = 0; j < TMAX / 2; ++j) a1[j] *= scale;

  LRD_STAMP(1);
  int hbase = 0;  // packed offset of row k of HV
  for (int k = 0; k < n; ++k) {
    // row k (= column k) into xk: a whole row from its lane, a half-row from
    // its two lanes
    if (k < 32) {
      if (lane == k) {
#pragma unroll
        for (int J = 0; J < NG; ++J)
          reinterpret_cast<float4*>(xk)[J] = make_float4(a0[4 * J], a0[4 * J + 1], a0[4 * J + 2], a0[4 * J + 3]);
      }
    } else if ((lane & 15) == k - 32) {
#pragma unroll
      for (int J = 0; J < NG; ++J)
        *reinterpret_cast<float2*>(xk + 4 * J + 2 * h) = make_float2(a1[2 * J], a1[2 * J + 1]);
    }
    __syncwarp();
    if (k >= n - 2) {
      if (lane == 0) {
        d[k] = xk[k];
        e[k] = (k == n - 2) ? xk[k + 1] : 0.f;
        tau[k] = 0.f;
      }
      __syncwarp();
      continue;
    }
    const float xr0 = v0 ? xk[lane] : 0.f;
    const float xr1 = v1 ? xk[r1] : 0.f;
    float part = 0.f;
    if (lane >= k + 2 && lane < n) part = fmaf(xr0, xr0, part);
    if (h == 0 && r1 >= k + 2 && r1 < n) part = fmaf(xr1, xr1, part);
    const float xnorm2 = warp_sum(part);
    const float alpha = xk[k + 1];
    float taui = 0.f, beta = alpha, sc = 0.f;
    if (xnorm2 > 0.f) {
      beta = -copysignf(sqrtf(fmaf(alpha, alpha, xnorm2)), alpha);
      taui = (beta - alpha) / beta;
      sc = 1.f / (alpha - beta);
    }
    if (lane == 0) {
      d[k] = xk[k];
      e[k] = beta;
      tau[k] = taui;
    }
    const int j4lo = (k + 1) >> 2;
    float* hv = HV + hbase - 4 * j4lo;
    hbase += TMAX - 4 * j4lo;
    const float vr0 = (lane == k + 1) ? 1.f : ((lane >= k + 2 && lane < n) ? xr0 * sc : 0.f);
    const float vr1 = (r1 == k + 1) ? 1.f : ((r1 >= k + 2 && r1 < n) ? xr1 * sc : 0.f);
    if (lane >= 4 * j4lo && lane < TMAX) hv[lane] = vr0;
    if (h == 0 && r1 >= 4 * j4lo && r1 < TMAX) hv[r1] = vr1;
    __syncwarp();
    if (taui != 0.f) {
      // p = taui * A22 v (live column groups from j4lo, as in the two-row code)
      const float4* hv4 = reinterpret_cast<const float4*>(hv);
      float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, t0 = 0.f, t1 = 0.f;
#define LRD_MVH(J)                                        \
  case J:                                                 \
    if constexpr (J < NG) {                               \
      const float4 v4 = hv4[J];                           \
      s0 = fmaf(a0[4 * J + 0], v4.x, s0);                 \
      s1 = fmaf(a0[4 * J + 1], v4.y, s1);                 \
      s2 = fmaf(a0[4 * J + 2], v4.z, s2);                 \
      s3 = fmaf(a0[4 * J + 3], v4.w, s3);                 \
      t0 = fmaf(a1[2 * J + 0], h ? v4.z : v4.x, t0);      \
      t1 = fmaf(a1[2 * J + 1], h ? v4.w : v4.y, t1);      \
    }
      switch (j4lo) {
        LRD_MVH(0) LRD_MVH(1) LRD_MVH(2) LRD_MVH(3) LRD_MVH(4) LRD_MVH(5)
        LRD_MVH(6) LRD_MVH(7) LRD_MVH(8) LRD_MVH(9) LRD_MVH(10) LRD_MVH(11)
        default: break;
      }
#undef LRD_MVH
      const float pr0 = (lane >= k + 1 && lane < n) ? taui * ((s0 + s1) + (s2 + s3)) : 0.f;
      const float pair = t0 + t1;  // s0 + s1 (h = 0) or s2 + s3 (h = 1) of the half-row
      const float other = __shfl_xor_sync(0xffffffffu, pair, 16);
      const float pr1 = (r1 >= k + 1 && r1 < n) ? taui * (h ? other + pair : pair + other) : 0.f;
      float part2 = 0.f;
      part2 = fmaf(pr0, vr0, part2);
      part2 = fmaf(h ? 0.f : pr1, h ? 0.f : vr1, part2);  // the half-row counted once
      const float kc = -0.5f * taui * warp_sum(part2);
      const float wr0 = fmaf(kc, vr0, pr0);
      const float wr1 = fmaf(kc, vr1, pr1);
      if (lane < TMAX) ws[lane] = wr0;
      if (h == 0 && r1 < TMAX) ws[r1] = wr1;
      __syncwarp();
      // A22 -= v w^T + w v^T (live column groups)
      const float4* ws4 = reinterpret_cast<const float4*>(ws);
#define LRD_UPDH(J)                                                                   \
  case J:                                                                             \
    if constexpr (J < NG) {                                                           \
      const float4 v4 = hv4[J];                                                       \
      const float4 w4 = ws4[J];                                                       \
      a0[4 * J + 0] = fmaf(-vr0, w4.x, fmaf(-wr0, v4.x, a0[4 * J + 0]));              \
      a0[4 * J + 1] = fmaf(-vr0, w4.y, fmaf(-wr0, v4.y, a0[4 * J + 1]));              \
      a0[4 * J + 2] = fmaf(-vr0, w4.z, fmaf(-wr0, v4.z, a0[4 * J + 2]));              \
      a0[4 * J + 3] = fmaf(-vr0, w4.w, fmaf(-wr0, v4.w, a0[4 * J + 3]));              \
      const float va = h ? v4.z : v4.x, vb = h ? v4.w : v4.y;                         \
      const float wa = h ? w4.z : w4.x, wb = h ? w4.w : w4.y;                         \
      a1[2 * J + 0] = fmaf(-vr1, wa, fmaf(-wr1, va, a1[2 * J + 0]));                  \
      a1[2 * J + 1] = fmaf(-vr1, wb, fmaf(-wr1, vb, a1[2 * J + 1]));                  \
    }
      switch (j4lo) {
        LRD_UPDH(0) LRD_UPDH(1) LRD_UPDH(2) LRD_UPDH(3) LRD_UPDH(4) LRD_UPDH(5)
        LRD_UPDH(6) LRD_UPDH(7) LRD_UPDH(8) LRD_UPDH(9) LRD_UPDH(10) LRD_UPDH(11)
        default: break;
      }
#undef LRD_UPDH
    }
    __syncwarp();  // xk, ws are rewritten by the next step
  }
  hbase_out = hbase;
}

// Body of one warp's matrix ``b`` (the launch's patch index; the patch is
// patch0 + b), shared by the single-volume kernel and the packed launch.
// HALF: the half-row tridiagonalisation (TMAX in (32, 48]; same results).
template <int TMAX, bool HALF = eigh_reg_half<TMAX>()>
__device__ __forceinline__ void eigh_reg_body(const float* gram, float* vecs, float* __restrict__ lam_out,
                                              int32_t* __restrict__ ranks, float* __restrict__ wgt,
                                              float* __restrict__ sig2, int n, int nvox, long long patch0,
                                              int* __restrict__ refine_count, int* __restrict__ refine_ids,
                                              long long b) {
  constexpr int NR = eigh_reg_nr<TMAX>();
  extern __shared__ __align__(16) float sr[];
  float* HV = sr;  // packed reflector vectors
  float* d = HV + eigh_hv_floats<TMAX>();
  float* e = d + TMAX;
  float* e2 = e + TMAX;
  float* tau = e2 + TMAX;
  float* lam = tau + TMAX;
  float* W = lam + TMAX;                 // LU (3 TMAX kInvGroup) / MP scratch (2 TMAX)
  float* Yt = W + 3 * TMAX * kInvGroup;  // TMAX x kLdy
  float* xk = W;                         // tridiagonalisation only: row k broadcast
  float* ws = W + TMAX;                  //   and the w vector
  const int lane = threadIdx.x;
  const float* G = gram + b * (long long)n * n;
  LRD_STAMP(0);

  // ---- load own rows (exact power-of-two scaling), Householder ---------------
  float unscale;
  int hbase;
  if constexpr (HALF) {
    tridiag_half<TMAX>(G, n, HV, d, e, tau, xk, ws, unscale, hbase);
  } else {
    // ---- load own rows, exact power-of-two scaling -----------------------------
    float a[NR][TMAX];
    float dmax = 0.f;
#pragma unroll
    for (int ri = 0; ri < NR; ++ri) {
      const int r = lane + 32 * ri;
      const bool rv = r < n;
#pragma unroll
      for (int j = 0; j < TMAX; ++j) a[ri][j] = (rv && j < n) ? G[(long long)r * n + j] : 0.f;
      if (rv) dmax = fmaxf(dmax, fabsf(G[(long long)r * n + r]));
    }
    dmax = warp_max(dmax);
    int ex = 0;
    if (dmax > 0.f && isfinite(dmax)) frexpf(dmax, &ex);
    const float scale = ldexpf(1.f, -ex);
    unscale = ldexpf(1.f, ex);
#pragma unroll
    for (int ri = 0; ri < NR; ++ri)
#pragma unroll
      for (int j = 0; j < TMAX; ++j) a[ri][j] *= scale;

    LRD_STAMP(1);
    // ---- Householder tridiagonalisation ---------------------------------------
    hbase = 0;  // packed offset of row k of HV
    for (int k = 0; k < n; ++k) {
      // owner of row k broadcasts it (= column k by symmetry)
      if (lane == (k & 31)) {
        if (NR == 1 || k < 32) {
#pragma unroll
          for (int j4 = 0; j4 < TMAX / 4; ++j4)
            reinterpret_cast<float4*>(xk)[j4] = make_float4(a[0][4 * j4], a[0][4 * j4 + 1], a[0][4 * j4 + 2],
                                                            a[0][4 * j4 + 3]);
        } else {
#pragma unroll
          for (int j4 = 0; j4 < TMAX / 4; ++j4)
            reinterpret_cast<float4*>(xk)[j4] = make_float4(a[NR - 1][4 * j4], a[NR - 1][4 * j4 + 1],
                                                            a[NR - 1][4 * j4 + 2], a[NR - 1][4 * j4 + 3]);
        }
      }
      __syncwarp();
      if (k >= n - 2) {
        if (lane == 0) {
          d[k] = xk[k];
          e[k] = (k == n - 2) ? xk[k + 1] : 0.f;
          tau[k] = 0.f;
        }
        __syncwarp();
        continue;
      }
      float xr[NR];
      float part = 0.f;
#pragma unroll
      for (int ri = 0; ri < NR; ++ri) {
        const int r = lane + 32 * ri;
        xr[ri] = (r < n) ? xk[r] : 0.f;
        if (r >= k + 2 && r < n) part = fmaf(xr[ri], xr[ri], part);
      }
      const float xnorm2 = warp_sum(part);
      const float alpha = xk[k + 1];
      float taui = 0.f, beta = alpha, sc = 0.f;
      if (xnorm2 > 0.f) {
        beta = -copysignf(sqrtf(fmaf(alpha, alpha, xnorm2)), alpha);
        taui = (beta - alpha) / beta;
        sc = 1.f / (alpha - beta);
      }
      if (lane == 0) {
        d[k] = xk[k];
        e[k] = beta;
        tau[k] = taui;
      }
      // row k from its first live column group j4lo on; hv[c] = column c
      const int j4lo = (k + 1) >> 2;
      float* hv = HV + hbase - 4 * j4lo;
      hbase += TMAX - 4 * j4lo;
      float vr[NR];
#pragma unroll
      for (int ri = 0; ri < NR; ++ri) {
        const int r = lane + 32 * ri;
        vr[ri] = (r == k + 1) ? 1.f : ((r >= k + 2 && r < n) ? xr[ri] * sc : 0.f);
        if (r >= 4 * j4lo && r < TMAX) hv[r] = vr[ri];
      }
      __syncwarp();
      if (taui != 0.f) {
        // p = taui * A22 v over own rows (columns j >= k+1; hv is 0 below).
        // The column groups j4 < j4lo are dead (and not stored): a switch on
        // j4lo enters the unrolled groups at the first live one (cases fall
        // through), so the register indices stay compile-time and the dead
        // groups cost nothing.
        // (both own rows in one pass over the groups: each hv group is read once)
        float pr[NR];
        float s0[NR], s1[NR], s2[NR], s3[NR];
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) s0[ri] = s1[ri] = s2[ri] = s3[ri] = 0.f;
#define LRD_MV(J)                                                   \
    case J:                                                           \
      if constexpr (J < TMAX / 4) {                                   \
        const float4 v4 = reinterpret_cast<const float4*>(hv)[J];     \
        _Pragma("unroll") for (int ri = 0; ri < NR; ++ri) {           \
          s0[ri] = fmaf(a[ri][4 * J + 0], v4.x, s0[ri]);              \
          s1[ri] = fmaf(a[ri][4 * J + 1], v4.y, s1[ri]);              \
          s2[ri] = fmaf(a[ri][4 * J + 2], v4.z, s2[ri]);              \
          s3[ri] = fmaf(a[ri][4 * J + 3], v4.w, s3[ri]);              \
        }                                                             \
      }
        switch (j4lo) {
          LRD_MV(0) LRD_MV(1) LRD_MV(2) LRD_MV(3) LRD_MV(4) LRD_MV(5) LRD_MV(6) LRD_MV(7)
          LRD_MV(8) LRD_MV(9) LRD_MV(10) LRD_MV(11) LRD_MV(12) LRD_MV(13) LRD_MV(14) LRD_MV(15)
          default: break;
        }
#undef LRD_MV
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) {
          const int r = lane + 32 * ri;
          pr[ri] = (r >= k + 1 && r < n) ? taui * ((s0[ri] + s1[ri]) + (s2[ri] + s3[ri])) : 0.f;
        }
        float part2 = 0.f;
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) part2 = fmaf(pr[ri], vr[ri], part2);
        const float kc = -0.5f * taui * warp_sum(part2);
        float wr[NR];
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) {
          const int r = lane + 32 * ri;
          wr[ri] = fmaf(kc, vr[ri], pr[ri]);
          if (r < TMAX) ws[r] = wr[ri];
        }
        __syncwarp();
        // A22 -= v w^T + w v^T on own rows, columns j >= k+1 (ws, hv zero
        // below), live column groups only as above
#define LRD_UPD(J)                                                                     \
    case J:                                                                              \
      if constexpr (J < TMAX / 4) {                                                      \
        const float4 v4 = reinterpret_cast<const float4*>(hv)[J];                        \
        const float4 w4 = reinterpret_cast<const float4*>(ws)[J];                        \
        _Pragma("unroll") for (int ri = 0; ri < NR; ++ri) {                              \
          a[ri][4 * J + 0] = fmaf(-vr[ri], w4.x, fmaf(-wr[ri], v4.x, a[ri][4 * J + 0])); \
          a[ri][4 * J + 1] = fmaf(-vr[ri], w4.y, fmaf(-wr[ri], v4.y, a[ri][4 * J + 1])); \
          a[ri][4 * J + 2] = fmaf(-vr[ri], w4.z, fmaf(-wr[ri], v4.z, a[ri][4 * J + 2])); \
          a[ri][4 * J + 3] = fmaf(-vr[ri], w4.w, fmaf(-wr[ri], v4.w, a[ri][4 * J + 3])); \
        }                                                                                \
      }
        switch (j4lo) {
          LRD_UPD(0) LRD_UPD(1) LRD_UPD(2) LRD_UPD(3) LRD_UPD(4) LRD_UPD(5) LRD_UPD(6) LRD_UPD(7)
          LRD_UPD(8) LRD_UPD(9) LRD_UPD(10) LRD_UPD(11) LRD_UPD(12) LRD_UPD(13) LRD_UPD(14) LRD_UPD(15)
          default: break;
        }
#undef LRD_UPD
      }
      __syncwarp();  // xk, ws are rewritten by the next step
    }
  }
  for (int i = lane; i < n; i += 32) e2[i] = (i < n - 1) ? e[i] * e[i] : 0.f;
  __syncwarp();

  LRD_STAMP(2);
  // ---- eigenvalues, MP rank ---------------------------------------------------
  float tnorm;
  bisect_reg<TMAX>(d, e, e2, lam, n, tnorm);
  LRD_STAMP(3);
  int p;
  const double margin = mp_rank<float>(lam, unscale, n, nvox, W, p, sig2 ? sig2 + b : nullptr);
  if (lane == 0) {
    ranks[b] = p;
    wgt[b] = (float)(1.0 / (2.0 + (double)p));
    if (refine_count != nullptr && margin < kRefineTol) refine_ids[atomicAdd(refine_count, 1)] = (int)(patch0 + b);
  }
  if (lam_out != nullptr)
    for (int i = lane; i < n; i += 32) lam_out[b * n + i] = lam[i] * unscale;
  LRD_STAMP(4);
  if (p == 0) return;
  __syncwarp();

  // ---- top-p eigenvectors, 8 at a time --------------------------------------
  const float pivtol = Num<float>::eps() * tnorm;
  float* RU0 = W;
  float* U1 = RU0 + TMAX * kInvGroup;
  float* ML = U1 + TMAX * kInvGroup;
  float* V = vecs + b * (long long)n * n;
  for (int j0 = 0; j0 < p; j0 += kInvGroup) {
    const int g = min(kInvGroup, p - j0);
    if (lane < g) {
      const int q = lane;
      const int j = j0 + q;
      const float sig = lam[n - 1 - j];
      // LU with partial pivoting of (T - sig I)
      float c = d[0] - sig, s = (n > 1) ? e[0] : 0.f;
      unsigned long long swb = 0;  // bit i: rows i and i + 1 swapped
      // (the lanes pivot differently: selects, not branches)
      for (int i = 0; i < n - 1; ++i) {
        const float ei = e[i];
        const float an = d[i + 1] - sig;
        const float en = (i + 1 < n - 1) ? e[i + 1] : 0.f;
        const bool keep = fabsf(c) >= fabsf(ei);
        const float num = keep ? ei : c, den = keep ? c : ei;
        const float m = (keep && ei == 0.f) ? 0.f : __fdividef(num, den);
        float piv = den;
        U1[i * kInvGroup + q] = keep ? s : an;
        ML[i * kInvGroup + q] = m;
        swb |= (unsigned long long)(!keep) << i;
        const float cn = keep ? fmaf(-m, s, an) : fmaf(-m, an, s);
        s = keep ? en : -m * en;
        c = cn;
        if (fabsf(piv) < pivtol) piv = (piv < 0.f) ? -pivtol : pivtol;
        RU0[i * kInvGroup + q] = __fdividef(1.f, piv);
      }
      if (fabsf(c) < pivtol) c = (c < 0.f) ? -pivtol : pivtol;
      RU0[(n - 1) * kInvGroup + q] = __fdividef(1.f, c);
      // the vector in shared memory (Yt column q)
      float* Y = Yt;
      for (int i = 0; i < n; ++i) Y[i * kLdy + q] = start_entry(i, j);
      // two solves: the shift is the eigenvalue to eps ||T||, so each solve
      // shrinks the other eigenvectors' share by about eps ||T|| / gap; a
      // solve grows the vector by about 1 / (eps ||T||) per eigenvalue that
      // close to the shift, so it is rescaled between solves only when it has
      // grown past 1e15, and normalised after the last one
      for (int iter = 0; iter < kInvSolves; ++iter) {
        for (int i = 0; i < n - 1; ++i) {
          const float yi = Y[i * kLdy + q], yn = Y[(i + 1) * kLdy + q];
          const float m = ML[i * kInvGroup + q];
          const bool sw = (swb >> i) & 1ull;
          Y[i * kLdy + q] = sw ? yn : yi;
          Y[(i + 1) * kLdy + q] = sw ? fmaf(-m, yn, yi) : fmaf(-m, yi, yn);
        }
        float x2 = Y[(n - 1) * kLdy + q] * RU0[(n - 1) * kInvGroup + q];
        Y[(n - 1) * kLdy + q] = x2;
        float x1 = x2, amax = fabsf(x2);
        if (n >= 2) {
          x1 = (Y[(n - 2) * kLdy + q] - U1[(n - 2) * kInvGroup + q] * x2) * RU0[(n - 2) * kInvGroup + q];
          Y[(n - 2) * kLdy + q] = x1;
          amax = fmaxf(amax, fabsf(x1));
        }
        for (int i = n - 3; i >= 0; --i) {
          const float u2 = ((swb >> i) & 1ull) ? e[i + 1] : 0.f;
          const float xi = (Y[i * kLdy + q] - U1[i * kInvGroup + q] * x1 - u2 * x2) * RU0[i * kInvGroup + q];
          Y[i * kLdy + q] = xi;
          amax = fmaxf(amax, fabsf(xi));
          x2 = x1;
          x1 = xi;
        }
        if (!(amax > 0.f) || !isfinite(amax)) {
          for (int i = 0; i < n; ++i) Y[i * kLdy + q] = start_entry(i, j + 977 * (iter + 1));
          continue;
        }
        if (iter + 1 < kInvSolves && amax < 1e15f) continue;  // rescale only a vector grown this far
        const float sa = 1.f / amax;
        float nrm = 0.f;
        for (int i = 0; i < n; ++i) {
          const float v = Y[i * kLdy + q] * sa;
          Y[i * kLdy + q] = v;
          nrm = fmaf(v, v, nrm);
        }
        const float inv = rsqrtf(nrm);
        for (int i = 0; i < n; ++i) Y[i * kLdy + q] *= inv;
      }
    }
    __syncwarp();
    LRD_STAMP(5);
    // row-distributed chunk: yr[ri][q] = vector q, row lane + 32 ri
    float yr[NR][kInvGroup];
#pragma unroll
    for (int ri = 0; ri < NR; ++ri) {
      const int r = lane + 32 * ri;
#pragma unroll
      for (int q = 0; q < kInvGroup; ++q) yr[ri][q] = (r < n && q < g) ? Yt[r * kLdy + q] : 0.f;
    }
    // back-transform x = H(0) ... H(n-3) y, on the first G = 4 or 8 vectors
    // of the chunk (G >= g)
    auto back_transform = [&](auto gtag) {
      constexpr int G = decltype(gtag)::value;
      int hb = hbase;  // end of the packed rows
      for (int k = n - 3; k >= 0; --k) {
        const int j4lo = (k + 1) >> 2;
        hb -= TMAX - 4 * j4lo;
        const float tk = tau[k];
        if (tk == 0.f) continue;
        const float* hrow = HV + hb - 4 * j4lo;
        float hr[NR];
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) {
          const int r = lane + 32 * ri;
          hr[ri] = (r >= 4 * j4lo && r < n) ? hrow[r] : 0.f;
        }
        float dq[G];
#pragma unroll
        for (int q = 0; q < G; ++q) {
          float s_ = 0.f;
#pragma unroll
          for (int ri = 0; ri < NR; ++ri) s_ = fmaf(hr[ri], yr[ri][q], s_);
          dq[q] = s_;
        }
        warp_allsum<G>(dq);
#pragma unroll
        for (int q = 0; q < G; ++q) {
          const float f = tk * dq[q];
#pragma unroll
          for (int ri = 0; ri < NR; ++ri) yr[ri][q] = fmaf(-f, hr[ri], yr[ri][q]);
        }
      }
    };
    if (g <= 4)
      back_transform(IntTag<4>{});
    else
      back_transform(IntTag<8>{});
    LRD_STAMP(6);
    // modified Gram-Schmidt in descending eigenvalue order
#pragma unroll
    for (int q = 0; q < kInvGroup; ++q) {
      if (q < g) {
        for (int i = 0; i < j0; ++i) {  // earlier chunks, from the output
          float s_ = 0.f;
          float vi[NR];
#pragma unroll
          for (int ri = 0; ri < NR; ++ri) {
            const int r = lane + 32 * ri;
            vi[ri] = (r < n) ? V[i * n + r] : 0.f;
            s_ = fmaf(vi[ri], yr[ri][q], s_);
          }
          const float dot = warp_sum(s_);
#pragma unroll
          for (int ri = 0; ri < NR; ++ri) yr[ri][q] = fmaf(-dot, vi[ri], yr[ri][q]);
        }
#pragma unroll
        for (int i = 0; i < kInvGroup; ++i) {
          if (i < q) {
            float s_ = 0.f;
#pragma unroll
            for (int ri = 0; ri < NR; ++ri) s_ = fmaf(yr[ri][i], yr[ri][q], s_);
            const float dot = warp_sum(s_);
#pragma unroll
            for (int ri = 0; ri < NR; ++ri) yr[ri][q] = fmaf(-dot, yr[ri][i], yr[ri][q]);
          }
        }
        float s_ = 0.f;
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) s_ = fmaf(yr[ri][q], yr[ri][q], s_);
        const float inv = rsqrtf(fmaxf(warp_sum(s_), FLT_MIN));
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) yr[ri][q] *= inv;
      }
    }
#pragma unroll
    for (int q = 0; q < kInvGroup; ++q)
      if (q < g)
#pragma unroll
        for (int ri = 0; ri < NR; ++ri) {
          const int r = lane + 32 * ri;
          if (r < n) V[(j0 + q) * n + r] = yr[ri][q];
        }
    __syncwarp();
  }
  LRD_STAMP(7);
}

// Warps per SM the single-volume eigh_reg_kernel<TMAX> reaches with the
// registers it is built with (94 / 128 / 168 at TMAX 32 / 48 / 64): the
// packed batch kernel's descriptor lookups must not lower it.
template <int TMAX>
__host__ __device__ constexpr int eigh_reg_min_blocks() {
  return TMAX <= 32 ? 20 : (TMAX <= 48 ? 16 : 12);
}

// At TMAX 48 the half-row tridiagonalisation measured 0.908 -> 0.885 ms on
// the 12600 headline Grams (bit-identical vectors and ranks) at the same 16
// warps per SM; capped below 128 registers (17 warps) it spilled and was
// slower (120: 0.922 ms, 112: 0.947 ms). The packed batch kernel keeps the
// two-row code, which its descriptor lookups leave fewer spills in.
template <int TMAX>
__global__ void __launch_bounds__(32, eigh_reg_min_blocks<TMAX>())
    eigh_reg_kernel(const float* gram, float* vecs, float* __restrict__ lam_out, int32_t* __restrict__ ranks,
                    float* __restrict__ wgt, float* __restrict__ sig2, int n, int nvox, long long patch0,
                    int* __restrict__ refine_count, int* __restrict__ refine_ids) {
  eigh_reg_body<TMAX>(gram, vecs, lam_out, ranks, wgt, sig2, n, nvox, patch0, refine_count, refine_ids,
                      (long long)blockIdx.x);
}

}  // namespace lrd
