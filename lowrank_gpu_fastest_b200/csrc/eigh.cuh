// Batched T x T symmetric eigensolver + Marchenko-Pastur rank + weight.
//
// Replaces the ladder's ``torch.linalg.eigh`` (step8_tuned.py:134; cuSOLVER),
// ``mp_keep`` (step8_tuned.py:96-113), the projector bmm (step8:136) and the
// weight (step8:137). One warp owns one patch's Gram matrix in shared memory:
//
//  1. exact power-of-two scaling so the largest diagonal entry is in [0.5, 1);
//  2. Householder reduction to tridiagonal form (lower, one reflector per
//     column; the reflector vectors stay in the strictly-lower part);
//  3. every eigenvalue by bisection on Sturm counts, two eigenvalues per lane
//     evaluated as two interleaved dependency chains;
//  4. the MP rank from the full spectrum, evaluated like step0_numpy_loop.py:
//     18-24: eigs = float32(max(lambda, 0) / N) in descending order with the
//     smallest (null) eigenvalue dropped (step4_gram_eigh.py:49), float32
//     suffix sums rcum, and the test
//       float64(float32(eigs_i - eigs_last)) * (t - i) * (N - i)
//         > float64(float32(4 * rcum_i)) * sqrt(float64(t * N))
//     counted over all i (NumPy promotes the ladder's test to float64);
//  5. the top-p eigenvectors, in chunks of 8: inverse iteration on the
//     tridiagonal matrix (partial-pivoting LU, three solves from distinct
//     pseudo-random starts), the Householder back-transform, then modified
//     Gram-Schmidt in descending eigenvalue order;
//  6. w = float32(1 / (2 + p)) (step0:36).
//
// The routine is templated on the working precision. The main pass runs it
// in float32 on the float32 Gram. A patch whose MP test has an index with
// |lhs/rhs - 1| below kRefineTol (a near-tie that float32 round-off could
// decide either way) is queued, and eigh_refine_kernel redoes it in float64:
// each voxel's time course centred in float64 from the input volume (the
// float64 mean of its float32 values), the Gram from float64 products with a
// float64 sum, then the same eigen/MP/eigenvector steps in float64 - so
// near-ties are decided as the float64 evaluation of the algorithm decides
// them, down to margins far below the float32 centred data's own rounding.
//
// Output per patch: the p eigenvectors (descending eigenvalue order) as the
// rows of a compact p x T block at the start of the patch's T x T slot (the
// projector of step8:136 is V_p V_p^T; the reconstruction applies it as
// (x V_p) V_p^T), the rank, the weight, optionally the ascending eigenvalues.
#pragma once

#include <float.h>

#include "lrd_common.cuh"

namespace lrd {

template <typename Real>
struct Num;
template <>
struct Num<float> {
  static __device__ __forceinline__ float eps() { return FLT_EPSILON * 0.5f; }
  static __device__ __forceinline__ float tiny() { return FLT_MIN; }
  static __device__ __forceinline__ float huge() { return FLT_MAX; }
  static __device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
  static __device__ __forceinline__ float rsq(float a) { return rsqrtf(a); }
};
template <>
struct Num<double> {
  static __device__ __forceinline__ double eps() { return DBL_EPSILON * 0.5; }
  static __device__ __forceinline__ double tiny() { return DBL_MIN; }
  static __device__ __forceinline__ double huge() { return DBL_MAX; }
  static __device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
  static __device__ __forceinline__ double rsq(double a) { return rsqrt(a); }
};

template <typename Real>
__device__ __forceinline__ Real warp_sum(Real v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename Real>
__device__ __forceinline__ Real warp_max(Real v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename Real>
__device__ __forceinline__ Real warp_min(Real v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Deterministic start vector entry in [-1, 1) for inverse iteration.
__device__ __forceinline__ float start_entry(int i, int j) {
  unsigned h = (unsigned)i * 0x9E3779B1u ^ ((unsigned)j + 0x7F4A7C15u) * 0x85EBCA77u;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  h *= 0x297A2D39u;
  h ^= h >> 15;
  return (float)(h >> 8) * (2.0f / 16777216.0f) - 1.0f;
}

constexpr int kInvGroup = 8;  // eigenvectors refined concurrently (one lane each)
constexpr int kInvSolves = 2;  // float32 solvers: inverse-iteration solves per eigenvector

// Floats of the packed Householder reflector rows of the float32 solvers: row
// k (k < n - 2 <= TMAX - 2) is stored from its first live 4-column group on,
// columns [4 * ((k + 1) >> 2), TMAX), about half of TMAX x TMAX.
template <int TMAX>
__host__ __device__ constexpr size_t eigh_hv_floats() {
  size_t f = 0;
  for (int k = 0; k < TMAX - 2; ++k) f += (size_t)(TMAX - 4 * ((k + 1) >> 2));
  return f;
}
constexpr int kLdy = kInvGroup + 1;  // eigenvector chunk row stride
constexpr double kRefineTol = 1e-4;  // MP-test margin below which float64 redoes the patch
// Margin of the float64 pass's step-0 emulation below which its decision is
// taken from the test in float64 throughout (within float32 resolution of the
// data, step 0's float32 arithmetic could decide either way).
constexpr double kTieFloor = 1e-6;

__host__ __device__ inline int eigh_lda(int n) { return n + ((n & 1) ? 2 : 1); }

// Shared-memory elements (of the working type) per warp: A (n x lda),
// eigenvector chunk (n x kLdy), d, e, e2, tau, lam (5n), LU of the chunk's
// shifted tridiagonals (4 n kInvGroup).
__host__ __device__ inline size_t eigh_smem_elems(int n) {
  return (size_t)n * eigh_lda(n) + (size_t)n * kLdy + 5 * (size_t)n + (size_t)4 * n * kInvGroup;
}

// MP rank from the ascending eigenvalues lam * unscale, evaluated like
// step0_numpy_loop.py:18-24 (float32 eigs and suffix sums, float64 test,
// a count over all indices); W holds 2n floats of scratch (4n + 2 in the
// float64 instantiation, whose W is 8-byte aligned). Returns the
// smallest |lhs/rhs - 1| over the indices. With ``sig2_out`` lane 0 also
// writes the patch's noise variance estimate, the mean of the t - p noise
// eigenvalues: rcum_p / (t - p) in float32 (0 when p = t). One warp.
template <typename Real>
__device__ double mp_rank(const Real* lam, Real unscale, int n, int nvox, float* W, int& p_out,
                          float* sig2_out = nullptr) {
  const int lane = threadIdx.x & 31;
  // eigs = float32(max(lambda, 0) / N), as step 0's float32 s**2 / n.
  const int t = n - 1;
  float* eg = W;                             // descending eigs, t entries
  float* rc = eg + n;                        // float32 suffix sums
  for (int i = lane; i < t; i += 32) {
    const Real l = fmax(lam[n - 1 - i] * unscale, Real(0));
    eg[i] = (sizeof(Real) == 4) ? __fdiv_rn((float)l, (float)nvox) : (float)(l / (Real)nvox);
  }
  __syncwarp();
  if (lane == 0) {
    float acc = eg[t - 1];
    rc[t - 1] = acc;
    for (int i = t - 2; i >= 0; --i) {
      acc = __fadd_rn(acc, eg[i]);
      rc[i] = acc;
    }
  }
  __syncwarp();
  int p = 0;
  double margin = DBL_MAX;
  {
    const double sq = sqrt((double)((long long)t * (long long)nvox));
    const float elast = eg[t - 1];
    for (int i0 = 0; i0 < t; i0 += 32) {
      const int i = i0 + lane;
      bool sig = false;
      if (i < t) {
        const double lhs = (double)__fsub_rn(eg[i], elast) * (double)(t - i) * (double)(nvox - i);
        const double rhs = (double)__fmul_rn(4.f, rc[i]) * sq;
        sig = lhs > rhs;
        if (rhs > 0.0) margin = fmin(margin, fabs(lhs - rhs) / rhs);
      }
      p += __popc(__ballot_sync(0xffffffffu, sig));
    }
    margin = warp_min(margin);
  }
  if constexpr (sizeof(Real) == 8) {
    // The float64 near-tie pass. Below a margin of kTieFloor the step-0
    // emulation (float32 eigs and sums) decides within float32 resolution of
    // the data - step 0's own float32 SVD could land either way - so the
    // count is taken from the test in float64 throughout (eigs, suffix sums
    // and products), the decision of the float64 run of the algorithm.
    if (margin < kTieFloor) {
      double* e64 = reinterpret_cast<double*>(rc + n);  // past the float32 arrays (float offset 2n: 8-byte aligned)
      for (int i = lane; i < t; i += 32) e64[i] = fmax((double)lam[n - 1 - i] * (double)unscale, 0.0) / nvox;
      __syncwarp();
      double r64 = 0.0, tail = 0.0;
      const double sq = sqrt((double)((long long)t * (long long)nvox));
      int p64 = 0;
      // suffix sums in double by lane 0 (t <= 127 terms), then the count
      if (lane == 0) {
        for (int i = t - 1; i >= 0; --i) {
          r64 += e64[i];
          const double lhs = (e64[i] - e64[t - 1]) * (double)(t - i) * (double)(nvox - i);
          p64 += lhs > 4.0 * r64 * sq;
        }
        tail = (double)p64;
      }
      p = (int)__shfl_sync(0xffffffffu, tail, 0);
      __syncwarp();
    }
  }
  p_out = p;
  if (sig2_out != nullptr && lane == 0) *sig2_out = (p < t) ? __fdiv_rn(rc[p], (float)(t - p)) : 0.f;
  return margin;
}

// One CTA of 128 threads, any n <= 128: eigen-decomposition of the symmetric
// n x n matrix the caller put in the first n*lda elements of ``sm`` (used in
// float64 by the near-tie pass), MP rank and weight, top-p eigenvectors (rows
// of the compact p x n block ``V``), optionally the ascending eigenvalues.
// Exact power-of-two scaling; Householder tridiagonalisation with the matrix
// in shared memory (odd row stride: a warp's threads, one row each, hit
// distinct banks), thread i owning row i of the trailing block, the two dot
// products per step block reductions; thread j bisects eigenvalue j on
// Sturm counts; the MP test on warp 0; inverse iteration on the tridiagonal
// (one lane per vector, partial pivoting), the back-transform (warp w:
// vectors w and w + 4) and modified Gram-Schmidt in descending eigenvalue
// order against the vectors already written. ``red`` = 8 elements of
// scratch. Returns the MP margin (warp 0; 0 on the other warps).
template <typename Real>
__device__ Real block_sum128(Real v, Real* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  return (red[0] + red[1]) + (red[2] + red[3]);
}

template <typename Real>
__device__ Real block_max128(Real v, Real* red) {
  v = warp_max(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  return fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
}

template <typename Real>
__device__ Real block_min128(Real v, Real* red) {
  v = warp_min(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  return fmin(fmin(red[0], red[1]), fmin(red[2], red[3]));
}

template <typename Real>
__device__ __forceinline__ int sturm_count1_r(const Real* d, const Real* e2, int n, Real x, Real pivmin) {
  Real q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int a = q < Real(0);
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - Num<Real>::fdiv(e2[i - 1], q);
    if (fabs(q) < pivmin) q = -pivmin;
    a += q < Real(0);
  }
  return a;
}

template <typename Real>
__device__ double eigh_mp_block(Real* sm, Real* red, int n, int nvox, float* V, float* lam_out, int32_t* rank_out,
                                float* w_out, float* s2_out) {
  constexpr int NT = 128;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int lda = eigh_lda(n);
  Real* A = sm;
  Real* Y = A + n * lda;
  Real* d = Y + n * kLdy;
  Real* e = d + n;
  Real* e2 = e + n;
  Real* tau = e2 + n;
  Real* lam = tau + n;
  Real* W = lam + n;
  const Real eps = Num<Real>::eps();

  Real dm = 0;
  for (int i = tid; i < n; i += NT) dm = fmax(dm, fabs(A[i * lda + i]));
  dm = block_max128(dm, red);
  int ex = 0;
  if (dm > Real(0) && isfinite(dm)) frexp(dm, &ex);
  const Real scale = ldexp(Real(1), -ex), unscale = ldexp(Real(1), ex);
  for (int idx = tid; idx < n * n; idx += NT) {
    const int r = idx / n, c = idx - r * n;
    A[r * lda + c] *= scale;
  }
  __syncthreads();

  Real* vv = W;
  Real* pp = W + n;
  Real* ww = W + 2 * n;
  for (int k = 0; k < n - 2; ++k) {
    const int L = n - k - 1;
    Real part = 0;
    for (int i = 1 + tid; i < L; i += NT) {
      const Real v = A[(k + 1 + i) * lda + k];
      part = fma(v, v, part);
    }
    const Real xnorm2 = block_sum128(part, red);
    const Real alpha = A[(k + 1) * lda + k];
    Real taui = 0, beta = alpha, scv = 0;
    if (xnorm2 > Real(0)) {
      beta = -copysign(sqrt(fma(alpha, alpha, xnorm2)), alpha);
      taui = (beta - alpha) / beta;
      scv = Real(1) / (alpha - beta);
    }
    for (int i = tid; i < L; i += NT) {
      if (i == 0) {
        vv[0] = Real(1);
      } else if (xnorm2 > Real(0)) {
        const Real v = A[(k + 1 + i) * lda + k] * scv;
        A[(k + 1 + i) * lda + k] = v;
        vv[i] = v;
      }
    }
    if (tid == 0) {
      e[k] = beta;
      d[k] = A[k * lda + k];
      tau[k] = taui;
    }
    __syncthreads();
    if (taui != Real(0)) {
      for (int i = tid; i < L; i += NT) {
        const Real* row = A + (k + 1 + i) * lda + (k + 1);
        Real s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        int j = 0;
        for (; j + 4 <= L; j += 4) {
          s0 = fma(row[j], vv[j], s0);
          s1 = fma(row[j + 1], vv[j + 1], s1);
          s2 = fma(row[j + 2], vv[j + 2], s2);
          s3 = fma(row[j + 3], vv[j + 3], s3);
        }
        for (; j < L; ++j) s0 = fma(row[j], vv[j], s0);
        pp[i] = taui * ((s0 + s1) + (s2 + s3));
      }
      __syncthreads();
      Real part2 = 0;
      for (int i = tid; i < L; i += NT) part2 = fma(pp[i], vv[i], part2);
      const Real kc = Real(-0.5) * taui * block_sum128(part2, red);
      for (int i = tid; i < L; i += NT) ww[i] = fma(kc, vv[i], pp[i]);
      __syncthreads();
      for (int i = tid; i < L; i += NT) {
        const Real vi = vv[i], wi = ww[i];
        Real* row = A + (k + 1 + i) * lda + (k + 1);
        for (int j = 0; j < L; ++j) row[j] = fma(-vi, ww[j], fma(-wi, vv[j], row[j]));
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A[(n - 2) * lda + (n - 2)];
      e[n - 2] = A[(n - 1) * lda + (n - 2)];
      tau[n - 2] = 0;
    }
    d[n - 1] = A[(n - 1) * lda + (n - 1)];
    e[n - 1] = 0;
    tau[n - 1] = 0;
  }
  __syncthreads();
  for (int i = tid; i < n; i += NT) e2[i] = (i < n - 1) ? e[i] * e[i] : Real(0);
  __syncthreads();

  // bisection, thread j = eigenvalue j, after a multisection pass (counts at
  // 128 evenly spaced points of the Gerschgorin interval bracket every
  // eigenvalue at once). The float64 pass exists to settle the MP test and the
  // top eigenvectors, so it stops at 100 eps (1e-14 relative to the norm
  // bound, and to the eigenvalue): ~40 steps instead of ~57.
  Real tnorm;
  {
    Real glo = Num<Real>::huge(), ghi = -Num<Real>::huge();
    for (int i = tid; i < n; i += NT) {
      const Real r = (i > 0 ? fabs(e[i - 1]) : Real(0)) + (i < n - 1 ? fabs(e[i]) : Real(0));
      glo = fmin(glo, d[i] - r);
      ghi = fmax(ghi, d[i] + r);
    }
    glo = block_min128(glo, red);
    ghi = block_max128(ghi, red);
    tnorm = fmax(fmax(fabs(glo), fabs(ghi)), Num<Real>::tiny());
    glo -= Real(4) * eps * tnorm * n;
    ghi += Real(4) * eps * tnorm * n;
    const Real pivmin = Num<Real>::tiny() * Real(4);
    const Real loose = Real(100) * eps;
    const Real abstol = loose * tnorm;
    const Real h = (ghi - glo) / Real(NT + 1);
    int* cnt = reinterpret_cast<int*>(W);
    cnt[tid] = sturm_count1_r(d, e2, n, glo + Real(tid + 1) * h, pivmin);
    __syncthreads();
    for (int j = tid; j < n; j += NT) {
      int lo_m = -1, hi_m = NT;  // cnt[lo_m] <= j < cnt[hi_m] holds along the search
      while (hi_m - lo_m > 1) {
        const int mid = (lo_m + hi_m) >> 1;
        if (cnt[mid] <= j) lo_m = mid; else hi_m = mid;
      }
      Real lo = lo_m >= 0 ? glo + Real(lo_m + 1) * h : glo;
      Real hi = hi_m < NT ? glo + Real(hi_m + 1) * h : ghi;
      for (int it = 0; it < 200; ++it) {
        const Real tol = fmax(abstol, Real(2) * loose * fmax(fabs(lo), fabs(hi)));
        const Real mid = Real(0.5) * (lo + hi);
        if (!(hi - lo > tol && mid > lo && mid < hi)) break;
        if (sturm_count1_r(d, e2, n, mid, pivmin) > j) hi = mid; else lo = mid;
      }
      lam[j] = Real(0.5) * (lo + hi);
    }
  }
  __syncthreads();

  int* pshare = reinterpret_cast<int*>(red + 4);
  double margin = 0.0;
  if (warp == 0) {
    int p;
    margin = mp_rank<Real>(lam, unscale, n, nvox, reinterpret_cast<float*>(W), p, s2_out);
    if (lane == 0) {
      *rank_out = p;
      *w_out = (float)(1.0 / (2.0 + (double)p));
      *pshare = p;
    }
  }
  if (lam_out != nullptr)
    for (int i = tid; i < n; i += NT) lam_out[i] = (float)(lam[i] * unscale);
  __syncthreads();
  const int p = *pshare;
  if (p == 0) return margin;

  const Real pivtol = eps * tnorm;
  Real* RU0 = W;
  Real* U1 = RU0 + n * kInvGroup;
  Real* ML = U1 + n * kInvGroup;
  Real* SW = ML + n * kInvGroup;
  for (int j0 = 0; j0 < p; j0 += kInvGroup) {
    const int g = min(kInvGroup, p - j0);
    __syncthreads();
    if (warp == 0 && lane < g) {
      const int q = lane;
      const int j = j0 + q;
      const Real sig = lam[n - 1 - j];
      Real c = d[0] - sig, s = (n > 1) ? e[0] : Real(0);
      for (int i = 0; i < n - 1; ++i) {
        const Real ei = e[i];
        const Real an = d[i + 1] - sig;
        const Real en = (i + 1 < n - 1) ? e[i + 1] : Real(0);
        const bool keep = fabs(c) >= fabs(ei);
        const Real m = keep ? ((ei == Real(0)) ? Real(0) : ei / c) : c / ei;
        Real piv = keep ? c : ei;
        U1[i * kInvGroup + q] = keep ? s : an;
        ML[i * kInvGroup + q] = m;
        SW[i * kInvGroup + q] = keep ? Real(0) : Real(1);
        const Real cn = keep ? fma(-m, s, an) : fma(-m, an, s);
        s = keep ? en : -m * en;
        c = cn;
        if (fabs(piv) < pivtol) piv = (piv < Real(0)) ? -pivtol : pivtol;
        RU0[i * kInvGroup + q] = Real(1) / piv;
      }
      if (fabs(c) < pivtol) c = (c < Real(0)) ? -pivtol : pivtol;
      RU0[(n - 1) * kInvGroup + q] = Real(1) / c;
      for (int i = 0; i < n; ++i) Y[i * kLdy + q] = start_entry(i, j);
      for (int iter = 0; iter < 3; ++iter) {
        for (int i = 0; i < n - 1; ++i) {
          const Real yi = Y[i * kLdy + q], yn = Y[(i + 1) * kLdy + q];
          const Real m = ML[i * kInvGroup + q];
          const bool sw = SW[i * kInvGroup + q] != Real(0);
          Y[i * kLdy + q] = sw ? yn : yi;
          Y[(i + 1) * kLdy + q] = sw ? fma(-m, yn, yi) : fma(-m, yi, yn);
        }
        Real x2 = Y[(n - 1) * kLdy + q] * RU0[(n - 1) * kInvGroup + q];
        Y[(n - 1) * kLdy + q] = x2;
        Real x1 = x2, amax = fabs(x2);
        if (n >= 2) {
          x1 = (Y[(n - 2) * kLdy + q] - U1[(n - 2) * kInvGroup + q] * x2) * RU0[(n - 2) * kInvGroup + q];
          Y[(n - 2) * kLdy + q] = x1;
          amax = fmax(amax, fabs(x1));
        }
        for (int i = n - 3; i >= 0; --i) {
          const Real u2 = (SW[i * kInvGroup + q] != Real(0)) ? e[i + 1] : Real(0);
          const Real xi = (Y[i * kLdy + q] - U1[i * kInvGroup + q] * x1 - u2 * x2) * RU0[i * kInvGroup + q];
          Y[i * kLdy + q] = xi;
          amax = fmax(amax, fabs(xi));
          x2 = x1;
          x1 = xi;
        }
        if (!(amax > Real(0)) || !isfinite(amax)) {
          for (int i = 0; i < n; ++i) Y[i * kLdy + q] = start_entry(i, j + 977 * (iter + 1));
          continue;
        }
        const Real sa = Real(1) / amax;
        Real nrm = 0;
        for (int i = 0; i < n; ++i) {
          const Real v = Y[i * kLdy + q] * sa;
          Y[i * kLdy + q] = v;
          nrm = fma(v, v, nrm);
        }
        const Real inv = Num<Real>::rsq(nrm);
        for (int i = 0; i < n; ++i) Y[i * kLdy + q] *= inv;
      }
    }
    __syncthreads();
    for (int q = warp; q < g; q += 4) {
      for (int k = n - 3; k >= 0; --k) {
        const Real tk = tau[k];
        if (tk == Real(0)) continue;
        const int L = n - k - 1;
        Real part = 0;
        for (int i = lane; i < L; i += 32) {
          const Real v = (i == 0) ? Real(1) : A[(k + 1 + i) * lda + k];
          part = fma(v, Y[(k + 1 + i) * kLdy + q], part);
        }
        const Real f = tk * warp_sum(part);
        for (int i = lane; i < L; i += 32) {
          const Real v = (i == 0) ? Real(1) : A[(k + 1 + i) * lda + k];
          Y[(k + 1 + i) * kLdy + q] = fma(-f, v, Y[(k + 1 + i) * kLdy + q]);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (warp == 0) {
      for (int q = 0; q < g; ++q) {
        const int j = j0 + q;
        for (int i = 0; i < j; ++i) {
          Real part = 0;
          if (i < j0) {
            for (int r = lane; r < n; r += 32) part = fma((Real)V[i * n + r], Y[r * kLdy + q], part);
          } else {
            for (int r = lane; r < n; r += 32) part = fma(Y[r * kLdy + (i - j0)], Y[r * kLdy + q], part);
          }
          const Real dot = warp_sum(part);
          if (i < j0) {
            for (int r = lane; r < n; r += 32) Y[r * kLdy + q] = fma(-dot, (Real)V[i * n + r], Y[r * kLdy + q]);
          } else {
            for (int r = lane; r < n; r += 32) Y[r * kLdy + q] = fma(-dot, Y[r * kLdy + (i - j0)], Y[r * kLdy + q]);
          }
          __syncwarp();
        }
        Real part = 0;
        for (int r = lane; r < n; r += 32) part = fma(Y[r * kLdy + q], Y[r * kLdy + q], part);
        const Real inv = Num<Real>::rsq(fmax(warp_sum(part), Num<Real>::tiny()));
        for (int r = lane; r < n; r += 32) Y[r * kLdy + q] *= inv;
        __syncwarp();
      }
    }
    __syncthreads();
    for (int idx = tid; idx < n * g; idx += NT) {
      const int c = idx / n, r = idx - c * n;
      V[(j0 + c) * n + r] = (float)Y[r * kLdy + c];
    }
  }
  __syncthreads();
  return margin;
}

// Shared memory bytes of eigh_refine_kernel: the float64 eigensolver's arrays
// plus two staged z-runs of the patch (pz*T values each, held as float64).
__host__ __device__ inline size_t eigh_refine_smem_bytes(int n, int pz) {
  return sizeof(double) * (eigh_smem_elems(n) + 8) + 2 * sizeof(double) * (size_t)pz * n;
}

constexpr int kRefineEntries = 24;  // Gram entries per thread per pass over the patch
constexpr int kRefinePrefetch = 16; // floats of the next z-run a thread prefetches

// Float64 pass over the queued near-tie patches not yet refined:
// refine_count[0] = entries queued, refine_count[1] = entries already refined
// (advanced by refine_advance_kernel after this kernel). Persistent grid, one
// patch per block at a time (128 threads). The block forms G = Xc^T Xc in
// float64 (products of the float32 centred values are exact in float64, the
// sum is float64) in passes of kRefineEntries entries per thread over the
// patch's z-runs, each run converted to float64 once as it is staged (the
// conversions inside the product loop bound this step: 1.6 M cycles at
// T = 64) and the next run prefetched through registers into a second
// buffer; then the block's float64 eigensolver (eigh_mp_block) overwrites the
// patch's rank, weight, eigenvectors (and eigenvalues if requested). A queue
// holds a handful of patches per volume, so this pass is one patch's latency:
// every step of it is spread over the block.
// Body: this block is block ``bid`` of ``nblocks`` working on one volume's queue.
// ``vol`` (nullable): the input volume - its voxel rows are centred here in
// float64; without it the float32 centred rows ``xc`` are used as they are.
__device__ __forceinline__ void eigh_refine_body(const float* __restrict__ vol, const float* __restrict__ xc,
                                                 float* vecs,
                                                 float* __restrict__ lam_out, int32_t* __restrict__ ranks,
                                                 float* __restrict__ wgt, float* __restrict__ sig2, const Geom& g,
                                                 const AxisTables& tab, const int* __restrict__ refine_count,
                                                 const int* __restrict__ refine_ids, int bid, int nblocks) {
  extern __shared__ double sm_ref[];
  const int n = g.nt;
  const int lda = eigh_lda(n);
  double* A = sm_ref;
  double* red = sm_ref + eigh_smem_elems(n);  // block reductions
  double* runs = red + 8;  // two z-run buffers, converted to float64 once when staged
  const int runlen = g.pz * n;
  const int count = refine_count[0];
  const int first = refine_count[1];
  const int tid = threadIdx.x;
  const int nth = blockDim.x;
  const int nent = n * (n + 1) / 2;
  const int nruns = g.px * g.py;
  // the next run goes through registers while this one is used (one barrier
  // per run) when a thread's share fits kRefinePrefetch floats
  const bool prefetch = runlen <= kRefinePrefetch * nth;
  for (int w = first + bid; w < count; w += nblocks) {
    const long long pid = refine_ids[w];
    int ci, cj, ck;
    patch_axes(g, pid, ci, cj, ck);
    const int cx = tab.corners[0][ci], cy = tab.corners[1][cj], cz = tab.corners[2][ck];
    const float* src0 = vol != nullptr ? vol : xc;
    auto run_src = [&](int q) { return src0 + voxel_row(g, cx + q / g.py, cy + q % g.py, cz) * n; };
    // the staged run's voxel rows centred in float64 (float32 input values are
    // exact in float64; the mean is their float64 sum / T)
    auto centre_run = [&](double* run) {
      if (vol == nullptr) return;
      __syncthreads();
      for (int r = tid; r < g.pz; r += nth) {
        double* row = run + (size_t)r * n;
        double sum = 0.0;
        for (int t = 0; t < n; ++t) sum += row[t];
        const double m = sum / n;
        for (int t = 0; t < n; ++t) row[t] -= m;
      }
    };
    // G = Xc^T Xc in float64 (products of float32 values are exact in float64);
    // entry (r, c), r <= c, sums over the runs in x-major voxel order
    for (int base = 0; base < nent; base += kRefineEntries * nth) {
      uint32_t rc[kRefineEntries];
      double acc[kRefineEntries];
#pragma unroll
      for (int u = 0; u < kRefineEntries; ++u) {
        int e = base + tid + u * nth, r = 0;
        if (e < nent) {
          while (e >= n - r) {
            e -= n - r;
            ++r;
          }
          rc[u] = (uint32_t)r | ((uint32_t)(r + e) << 16);
        } else {
          rc[u] = 0xffffffffu;
        }
        acc[u] = 0.0;
      }
      __syncthreads();  // the run buffers are free
      {
        const float* src = run_src(0);
        for (int e = tid; e < runlen; e += nth) runs[e] = (double)src[e];
      }
      centre_run(runs);
      __syncthreads();
      for (int q = 0; q < nruns; ++q) {
        const double* cur = runs + (size_t)(q & 1) * runlen;
        float pre[kRefinePrefetch];
        if (prefetch && q + 1 < nruns) {
          const float* src = run_src(q + 1);
#pragma unroll
          for (int i = 0; i < kRefinePrefetch; ++i) {
            const int e = tid + i * nth;
            pre[i] = e < runlen ? src[e] : 0.f;
          }
        }
#pragma unroll
        for (int u = 0; u < kRefineEntries; ++u) {
          if (rc[u] == 0xffffffffu) continue;
          const int r = (int)(rc[u] & 0xffffu), c = (int)(rc[u] >> 16);
          double s_ = acc[u];
          for (int rr = 0; rr < g.pz; ++rr) s_ = fma(cur[rr * n + r], cur[rr * n + c], s_);
          acc[u] = s_;
        }
        if (q + 1 < nruns) {
          double* nxt = runs + (size_t)((q + 1) & 1) * runlen;
          if (prefetch) {
#pragma unroll
            for (int i = 0; i < kRefinePrefetch; ++i) {
              const int e = tid + i * nth;
              if (e < runlen) nxt[e] = (double)pre[i];
            }
          } else {
            __syncthreads();  // everyone is done with the previous use of nxt
            const float* src = run_src(q + 1);
            for (int e = tid; e < runlen; e += nth) nxt[e] = (double)src[e];
          }
          centre_run(nxt);
        }
        __syncthreads();
      }
#pragma unroll
      for (int u = 0; u < kRefineEntries; ++u) {
        if (rc[u] == 0xffffffffu) continue;
        const int r = (int)(rc[u] & 0xffffu), c = (int)(rc[u] >> 16);
        A[r * lda + c] = acc[u];
        A[c * lda + r] = acc[u];
      }
    }
    __syncthreads();
    eigh_mp_block<double>(A, red, n, g.nvox_patch, vecs + pid * (long long)n * n,
                          lam_out ? lam_out + pid * n : nullptr, ranks + pid, wgt + pid,
                          sig2 ? sig2 + pid : nullptr);
    __syncthreads();
  }
}

__global__ void eigh_refine_kernel(const float* __restrict__ vol, const float* __restrict__ xc, float* vecs,
                                   float* __restrict__ lam_out,
                                   int32_t* __restrict__ ranks, float* __restrict__ wgt, float* __restrict__ sig2,
                                   Geom g, AxisTables tab, const int* __restrict__ refine_count,
                                   const int* __restrict__ refine_ids) {
  eigh_refine_body(vol, xc, vecs, lam_out, ranks, wgt, sig2, g, tab, refine_count, refine_ids, (int)blockIdx.x,
                   (int)gridDim.x);
}

// Marks every queued near-tie patch as refined (one thread).
__global__ void refine_advance_kernel(int* refine_count) { refine_count[1] = refine_count[0]; }

}  // namespace lrd
