// Block eigensolver for 64 < T <= 128: one CTA of TMAX threads (TMAX = 96
// or 128) per matrix, thread i owning row i.
//
// The algorithm is eigh_reg_kernel's (eigh_reg.cuh) - Householder
// tridiagonalisation, bisection with Sturm counts, the MP rank test, inverse
// iteration, back-transform, modified Gram-Schmidt - with a row per thread
// instead of rows per lane:
//
//  * Householder: row i of the working matrix in thread i's registers
//    (a[TMAX], every column index compile-time); at step k the owner of row k
//    broadcasts it through shared memory (= column k by symmetry); the
//    reflectors go to shared memory (HV, one row per step, stored from its
//    first live 4-column group on) for the back-transform; the two dot
//    products per step are block reductions;
//  * bisection: thread j owns eigenvalue j, after a multisection pass (counts
//    at TMAX evenly spaced points of the Gerschgorin interval bracket every
//    eigenvalue at once);
//  * MP rank and inverse iteration (one lane per eigenvector, vector in
//    registers) on warp 0; the back-transform and Gram-Schmidt row-distributed
//    over the CTA (thread i holds row i of the chunk's vectors) with block
//    reductions.
//
// The results agree with the one-warp routines to float32 round-off, and the
// same near-tie test queues patches for the float64 pass.
#pragma once

#include "eigh.cuh"

namespace lrd {

// Shared-memory floats: packed HV, d, e, e2, tau, lam (5 TMAX), LU / MP
// scratch / multisection counts (4 TMAX kInvGroup; during the
// tridiagonalisation the row broadcast and the w vector), eigenvector chunk
// (TMAX x kLdy), reductions (kInvGroup x 4 + 8).
template <int TMAX>
__host__ __device__ constexpr size_t eigh_cta_smem_floats() {
  return eigh_hv_floats<TMAX>() + 5 * (size_t)TMAX + (size_t)4 * TMAX * kInvGroup + (size_t)TMAX * kLdy +
         4 * kInvGroup + 8;
}

template <int NW>
__device__ __forceinline__ float cta_sum(float v, float* red) {
  v = warp_sum(v);
  __syncthreads();  // red is free (its previous readers are past this point)
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = red[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) s += red[w];
  return s;
}

template <int NW>
__device__ __forceinline__ float cta_max(float v, float* red) {
  v = warp_max(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = red[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) s = fmaxf(s, red[w]);
  return s;
}

template <int NW>
__device__ __forceinline__ float cta_min(float v, float* red) {
  v = warp_min(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = red[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) s = fminf(s, red[w]);
  return s;
}

// Eigenvalues of the tridiagonal below x (one chain): sturm2_reg's pivot
// recurrence (eigh_reg.cuh) on the tridiagonal in shared memory.
__device__ __forceinline__ int sturm_count1(const float* __restrict__ d, const float* __restrict__ e2, int n, float x,
                                            float pivmin) {
  float q = d[0] - x;
  if (fabsf(q) < pivmin) q = -pivmin;
  int a = (int)(__float_as_uint(q) >> 31);
#pragma unroll 4
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - __fdividef(e2[i - 1], q);
    if (fabsf(q) < pivmin) q = -pivmin;
    a += (int)(__float_as_uint(q) >> 31);
  }
  return a;
}

// One CTA of TMAX threads per patch: the body solves the launch's patch ``b``
// (patch index patch0 + b), n <= TMAX. ``gram`` (read) and ``vecs`` (written) may
// alias: the CTA reads its whole matrix before writing.
template <int TMAX>
__device__ __forceinline__ void eigh_cta_body(const float* gram, float* vecs, float* __restrict__ lam_out,
                                              int32_t* __restrict__ ranks, float* __restrict__ wgt,
                                              float* __restrict__ sig2, int n, int nvox, long long patch0,
                                              int* __restrict__ refine_count, int* __restrict__ refine_ids,
                                              long long b) {
  constexpr int NW = TMAX / 32;
  extern __shared__ __align__(16) float sc[];
  float* HV = sc;  // packed reflector vectors
  float* d = HV + eigh_hv_floats<TMAX>();
  float* e = d + TMAX;
  float* e2 = e + TMAX;
  float* tau = e2 + TMAX;
  float* lam = tau + TMAX;
  float* W = lam + TMAX;                  // LU (4 TMAX kInvGroup) / MP scratch / counts
  float* Yt = W + 4 * TMAX * kInvGroup;   // TMAX x kLdy
  float* red = Yt + TMAX * kLdy;          // 4 kInvGroup + 8
  float* xk = W;                          // tridiagonalisation only: row k broadcast
  float* ws = W + TMAX;                   //   and the w vector
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float* G = gram + b * (long long)n * n;
  const bool rv = tid < n;
  LRD_STAMP(0);

  // ---- own row, exact power-of-two scaling ------------------------------------
  float a[TMAX];
#pragma unroll
  for (int j = 0; j < TMAX; ++j) a[j] = (rv && j < n) ? G[(long long)tid * n + j] : 0.f;
  const float dmax = cta_max<NW>(rv ? fabsf(G[(long long)tid * n + tid]) : 0.f, red);
  int ex = 0;
  if (dmax > 0.f && isfinite(dmax)) frexpf(dmax, &ex);
  const float scale = ldexpf(1.f, -ex), unscale = ldexpf(1.f, ex);
#pragma unroll
  for (int j = 0; j < TMAX; ++j) a[j] *= scale;
  LRD_STAMP(1);

  // ---- Householder tridiagonalisation -------------------------------------------
  int hbase = 0;  // packed offset of row k of HV
  for (int k = 0; k < n; ++k) {
    if (tid == k) {
#pragma unroll
      for (int j4 = 0; j4 < TMAX / 4; ++j4)
        reinterpret_cast<float4*>(xk)[j4] = make_float4(a[4 * j4], a[4 * j4 + 1], a[4 * j4 + 2], a[4 * j4 + 3]);
    }
    __syncthreads();
    if (k >= n - 2) {
      if (tid == 0) {
        d[k] = xk[k];
        e[k] = (k == n - 2) ? xk[k + 1] : 0.f;
        tau[k] = 0.f;
      }
      __syncthreads();
      continue;
    }
    const float xr = rv ? xk[tid] : 0.f;
    const float xnorm2 = cta_sum<NW>((tid >= k + 2 && rv) ? xr * xr : 0.f, red);
    const float alpha = xk[k + 1];
    float taui = 0.f, beta = alpha, scv = 0.f;
    if (xnorm2 > 0.f) {
      beta = -copysignf(sqrtf(fmaf(alpha, alpha, xnorm2)), alpha);
      taui = (beta - alpha) / beta;
      scv = 1.f / (alpha - beta);
    }
    if (tid == 0) {
      d[k] = xk[k];
      e[k] = beta;
      tau[k] = taui;
    }
    const float vr = (tid == k + 1) ? 1.f : ((tid >= k + 2 && rv) ? xr * scv : 0.f);
    // row k from its first live column group j4lo on; hv[c] = column c
    const int j4lo = (k + 1) >> 2;
    float* hv = HV + hbase - 4 * j4lo;
    hbase += TMAX - 4 * j4lo;
    if (tid >= 4 * j4lo) hv[tid] = vr;
    __syncthreads();
    if (taui != 0.f) {
      // p = taui * A22 v on the own row; column groups below j4lo are dead and
      // not stored (a switch enters the unrolled groups at the first live one)
      float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#define LRD_CMV(J)                                                 \
  case J:                                                          \
    if constexpr (J < TMAX / 4) {                                  \
      const float4 v4 = reinterpret_cast<const float4*>(hv)[J];    \
      s0 = fmaf(a[4 * J + 0], v4.x, s0);                           \
      s1 = fmaf(a[4 * J + 1], v4.y, s1);                           \
      s2 = fmaf(a[4 * J + 2], v4.z, s2);                           \
      s3 = fmaf(a[4 * J + 3], v4.w, s3);                           \
    }
      switch (j4lo) {
        LRD_CMV(0) LRD_CMV(1) LRD_CMV(2) LRD_CMV(3) LRD_CMV(4) LRD_CMV(5) LRD_CMV(6) LRD_CMV(7)
        LRD_CMV(8) LRD_CMV(9) LRD_CMV(10) LRD_CMV(11) LRD_CMV(12) LRD_CMV(13) LRD_CMV(14) LRD_CMV(15)
        LRD_CMV(16) LRD_CMV(17) LRD_CMV(18) LRD_CMV(19) LRD_CMV(20) LRD_CMV(21) LRD_CMV(22) LRD_CMV(23)
        LRD_CMV(24) LRD_CMV(25) LRD_CMV(26) LRD_CMV(27) LRD_CMV(28) LRD_CMV(29) LRD_CMV(30) LRD_CMV(31)
        default: break;
      }
#undef LRD_CMV
      const float pr = (tid >= k + 1 && rv) ? taui * ((s0 + s1) + (s2 + s3)) : 0.f;
      const float kc = -0.5f * taui * cta_sum<NW>(pr * vr, red);
      const float wr = fmaf(kc, vr, pr);
      ws[tid] = wr;
      __syncthreads();
#define LRD_CUPD(J)                                                             \
  case J:                                                                       \
    if constexpr (J < TMAX / 4) {                                               \
      const float4 v4 = reinterpret_cast<const float4*>(hv)[J];                 \
      const float4 w4 = reinterpret_cast<const float4*>(ws)[J];                 \
      a[4 * J + 0] = fmaf(-vr, w4.x, fmaf(-wr, v4.x, a[4 * J + 0]));            \
      a[4 * J + 1] = fmaf(-vr, w4.y, fmaf(-wr, v4.y, a[4 * J + 1]));            \
      a[4 * J + 2] = fmaf(-vr, w4.z, fmaf(-wr, v4.z, a[4 * J + 2]));            \
      a[4 * J + 3] = fmaf(-vr, w4.w, fmaf(-wr, v4.w, a[4 * J + 3]));            \
    }
      switch (j4lo) {
        LRD_CUPD(0) LRD_CUPD(1) LRD_CUPD(2) LRD_CUPD(3) LRD_CUPD(4) LRD_CUPD(5) LRD_CUPD(6) LRD_CUPD(7)
        LRD_CUPD(8) LRD_CUPD(9) LRD_CUPD(10) LRD_CUPD(11) LRD_CUPD(12) LRD_CUPD(13) LRD_CUPD(14) LRD_CUPD(15)
        LRD_CUPD(16) LRD_CUPD(17) LRD_CUPD(18) LRD_CUPD(19) LRD_CUPD(20) LRD_CUPD(21) LRD_CUPD(22) LRD_CUPD(23)
        LRD_CUPD(24) LRD_CUPD(25) LRD_CUPD(26) LRD_CUPD(27) LRD_CUPD(28) LRD_CUPD(29) LRD_CUPD(30) LRD_CUPD(31)
        default: break;
      }
#undef LRD_CUPD
    }
    __syncthreads();  // xk, ws are rewritten by the next step
  }
  if (tid < n) e2[tid] = (tid < n - 1) ? e[tid] * e[tid] : 0.f;
  __syncthreads();
  LRD_STAMP(2);

  // ---- eigenvalues: multisection pass, then bisection, thread j = eigenvalue j
  const float eps = Num<float>::eps();
  float tnorm;
  {
    float glo = FLT_MAX, ghi = -FLT_MAX;
    if (rv) {
      const float r = (tid > 0 ? fabsf(e[tid - 1]) : 0.f) + (tid < n - 1 ? fabsf(e[tid]) : 0.f);
      glo = d[tid] - r;
      ghi = d[tid] + r;
    }
    glo = cta_min<NW>(glo, red);
    ghi = cta_max<NW>(ghi, red);
    tnorm = fmaxf(fmaxf(fabsf(glo), fabsf(ghi)), FLT_MIN);
    glo -= 4.f * eps * tnorm * n;
    ghi += 4.f * eps * tnorm * n;
    const float pivmin = FLT_MIN * 4.f;
    const float abstol = eps * tnorm;  // as bisect_reg
    const float h = (ghi - glo) * (1.f / (TMAX + 1));
    int* cnt = reinterpret_cast<int*>(W);
    cnt[tid] = sturm_count1(d, e2, n, fmaf((float)(tid + 1), h, glo), pivmin);
    __syncthreads();
    const int j = tid;
    // cnt[lo_m] <= j < cnt[hi_m] (-1 = glo, TMAX = ghi) holds along the search
    int lo_m = -1, hi_m = TMAX;
    while (hi_m - lo_m > 1) {
      const int mid = (lo_m + hi_m) >> 1;
      if (cnt[mid] <= j) lo_m = mid; else hi_m = mid;
    }
    float lo = lo_m >= 0 ? fmaf((float)(lo_m + 1), h, glo) : glo;
    float hi = hi_m < TMAX ? fmaf((float)(hi_m + 1), h, glo) : ghi;
    bool run = j < n;
    for (int it = 0; it < 200 && run; ++it) {
      const float tol = fmaxf(abstol, 2.f * eps * fmaxf(fabsf(lo), fabsf(hi)));
      const float mid = 0.5f * (lo + hi);
      run = hi - lo > tol && mid > lo && mid < hi;
      if (!run) break;
      if (sturm_count1(d, e2, n, mid, pivmin) > j) hi = mid; else lo = mid;
    }
    if (j < n) lam[j] = 0.5f * (lo + hi);
  }
  __syncthreads();
  LRD_STAMP(3);

  // ---- MP rank (warp 0) ---------------------------------------------------------
  int* pshare = reinterpret_cast<int*>(red + 4 * kInvGroup + 4);
  if (warp == 0) {
    int p;
    const double margin = mp_rank<float>(lam, unscale, n, nvox, W, p, sig2 ? sig2 + b : nullptr);
    if (lane == 0) {
      ranks[b] = p;
      wgt[b] = (float)(1.0 / (2.0 + (double)p));
      if (refine_count != nullptr && margin < kRefineTol) refine_ids[atomicAdd(refine_count, 1)] = (int)(patch0 + b);
      *pshare = p;
    }
  }
  if (lam_out != nullptr && rv) lam_out[b * n + tid] = lam[tid] * unscale;
  __syncthreads();
  const int p = *pshare;
  LRD_STAMP(4);
  if (p == 0) return;

  // ---- top-p eigenvectors, in chunks of kInvGroup ------------------------------
  const float pivtol = eps * tnorm;
  float* RU0 = W;
  float* U1 = RU0 + TMAX * kInvGroup;
  float* ML = U1 + TMAX * kInvGroup;
  float* SW = ML + TMAX * kInvGroup;
  float* V = vecs + b * (long long)n * n;
  for (int j0 = 0; j0 < p; j0 += kInvGroup) {
    const int g = min(kInvGroup, p - j0);
    __syncthreads();  // W and Yt are free
    if (warp == 0 && lane < g) {
      // inverse iteration on the tridiagonal, one lane per eigenvector
      const int q = lane;
      const int j = j0 + q;
      const float sig = lam[n - 1 - j];
      float c = d[0] - sig, s = (n > 1) ? e[0] : 0.f;
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
        SW[i * kInvGroup + q] = keep ? 0.f : 1.f;
        const float cn = keep ? fmaf(-m, s, an) : fmaf(-m, an, s);
        s = keep ? en : -m * en;
        c = cn;
        if (fabsf(piv) < pivtol) piv = (piv < 0.f) ? -pivtol : pivtol;
        RU0[i * kInvGroup + q] = __fdividef(1.f, piv);
      }
      if (fabsf(c) < pivtol) c = (c < 0.f) ? -pivtol : pivtol;
      RU0[(n - 1) * kInvGroup + q] = __fdividef(1.f, c);
      // the vector in shared memory (Yt column q): at T > 64 the register form's
      // fully unrolled loops measured slower (104 K vs 66 K cycles per matrix)
      float* Y = Yt;
      for (int i = 0; i < n; ++i) Y[i * kLdy + q] = start_entry(i, j);
      // two solves, rescaled in between only when grown past 1e15 (as the
      // one-warp solver)
      for (int iter = 0; iter < kInvSolves; ++iter) {
        for (int i = 0; i < n - 1; ++i) {
          const float yi = Y[i * kLdy + q], yn = Y[(i + 1) * kLdy + q];
          const float m = ML[i * kInvGroup + q];
          const bool sw = SW[i * kInvGroup + q] != 0.f;
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
          const float u2 = (SW[i * kInvGroup + q] != 0.f) ? e[i + 1] : 0.f;
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
        if (iter + 1 < kInvSolves && amax < 1e15f) continue;
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
    __syncthreads();
    LRD_STAMP(5);
    // row-distributed chunk: yr[q] = vector q, row tid
    float yr[kInvGroup];
#pragma unroll
    for (int q = 0; q < kInvGroup; ++q) yr[q] = (rv && q < g) ? Yt[tid * kLdy + q] : 0.f;
    float* rq = red;  // NW x kInvGroup partial sums
    // back-transform x = H(0) ... H(n-3) y
    int hb = hbase;  // end of the packed rows
    for (int k = n - 3; k >= 0; --k) {
      const int j4lo = (k + 1) >> 2;
      hb -= TMAX - 4 * j4lo;
      const float tk = tau[k];
      if (tk == 0.f) continue;
      const float hr = (rv && tid >= 4 * j4lo) ? HV[hb - 4 * j4lo + tid] : 0.f;
      float dq[kInvGroup];
#pragma unroll
      for (int q = 0; q < kInvGroup; ++q) dq[q] = hr * yr[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < kInvGroup; ++q) dq[q] += __shfl_xor_sync(0xffffffffu, dq[q], o);
      __syncthreads();  // rq is free
      if (lane < kInvGroup) {
        float v = dq[0];
#pragma unroll
        for (int q = 1; q < kInvGroup; ++q)
          if (lane == q) v = dq[q];
        rq[warp * kInvGroup + lane] = v;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kInvGroup; ++q) {
        float s_ = rq[q];
#pragma unroll
        for (int w = 1; w < NW; ++w) s_ += rq[w * kInvGroup + q];
        yr[q] = fmaf(-tk * s_, hr, yr[q]);
      }
    }
    LRD_STAMP(6);
    // modified Gram-Schmidt in descending eigenvalue order
    for (int q = 0; q < g; ++q) {
      for (int i = 0; i < j0; ++i) {  // earlier chunks, from the output
        const float vi = rv ? V[i * n + tid] : 0.f;
        float yq = 0.f;
#pragma unroll
        for (int u = 0; u < kInvGroup; ++u)
          if (u == q) yq = yr[u];
        const float dot = cta_sum<NW>(vi * yq, red + 4 * kInvGroup);
#pragma unroll
        for (int u = 0; u < kInvGroup; ++u)
          if (u == q) yr[u] = fmaf(-dot, vi, yr[u]);
      }
      for (int i = 0; i < q; ++i) {
        float yi = 0.f, yq = 0.f;
#pragma unroll
        for (int u = 0; u < kInvGroup; ++u) {
          if (u == i) yi = yr[u];
          if (u == q) yq = yr[u];
        }
        const float dot = cta_sum<NW>(yi * yq, red + 4 * kInvGroup);
#pragma unroll
        for (int u = 0; u < kInvGroup; ++u)
          if (u == q) yr[u] = fmaf(-dot, yi, yr[u]);
      }
      float yq = 0.f;
#pragma unroll
      for (int u = 0; u < kInvGroup; ++u)
        if (u == q) yq = yr[u];
      const float inv = rsqrtf(fmaxf(cta_sum<NW>(yq * yq, red + 4 * kInvGroup), FLT_MIN));
#pragma unroll
      for (int u = 0; u < kInvGroup; ++u)
        if (u == q) yr[u] *= inv;
    }
#pragma unroll
    for (int q = 0; q < kInvGroup; ++q)
      if (q < g && rv) V[(j0 + q) * n + tid] = yr[q];
    __syncthreads();  // the next chunk's Gram-Schmidt reads these rows
  }
  LRD_STAMP(7);
}

template <int TMAX>
__global__ void __launch_bounds__(TMAX)
    eigh_cta_kernel(const float* gram, float* vecs, float* __restrict__ lam_out, int32_t* __restrict__ ranks,
                    float* __restrict__ wgt, float* __restrict__ sig2, int n, int nvox, long long patch0,
                    int* __restrict__ refine_count, int* __restrict__ refine_ids) {
  eigh_cta_body<TMAX>(gram, vecs, lam_out, ranks, wgt, sig2, n, nvox, patch0, refine_count, refine_ids,
                      (long long)blockIdx.x);
}

}  // namespace lrd
