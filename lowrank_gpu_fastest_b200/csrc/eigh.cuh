// Batched T x T symmetric eigensolver + Marchenko-Pastur rank + weight.
//
// Replaces the ladder's ``torch.linalg.eigh`` (step8_tuned.py:134; cuSOLVER),
// ``mp_keep`` (step8_tuned.py:96-113), the projector bmm (step8:136) and the
// weight (step8:137). One warp owns one patch's Gram matrix in shared memory:
//
//  1. exact power-of-two scaling so the largest diagonal entry is in [0.5, 1);
//  2. Householder reduction to tridiagonal form (lower, one reflector per
//     column; the reflector vectors stay in the strictly-lower part);
//  3. every eigenvalue by bisection on Sturm counts, one eigenvalue per lane;
//  4. the MP rank from the full spectrum, evaluated like step0_numpy_loop.py:
//     18-24: eigs = float32(max(lambda, 0) / N) in descending order with the
//     smallest (null) eigenvalue dropped (step4_gram_eigh.py:49), float32
//     suffix sums rcum, and the test
//       float64(float32(eigs_i - eigs_last)) * (t - i) * (N - i)
//         > float64(float32(4 * rcum_i)) * sqrt(float64(t * N))
//     counted over all i (NumPy promotes the ladder's test to float64);
//  5. the top-p eigenvectors by inverse iteration on the tridiagonal matrix
//     (partial-pivoting LU, three solves from distinct pseudo-random starts),
//     modified Gram-Schmidt in descending eigenvalue order, then the
//     Householder back-transform;
//  6. w = float32(1 / (2 + p)) (step0:36).
//
// Output per patch: the p eigenvectors as a compact row-major T x p matrix at
// the start of the patch's T x T slot (the projector of step8:136 is V_p V_p^T; the reconstruction applies
// it as (x V_p) V_p^T), the rank, the weight, optionally the ascending
// eigenvalues.
#pragma once

#include <float.h>

#include "lrd_common.cuh"

namespace lrd {

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Number of eigenvalues of the tridiagonal (d, e^2) smaller than x.
__device__ __forceinline__ int sturm_count(const float* __restrict__ d, const float* __restrict__ e2,
                                           int n, float x, float pivmin) {
  float q = d[0] - x;
  if (fabsf(q) < pivmin) q = -pivmin;
  int c = q < 0.f;
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - __fdividef(e2[i - 1], q);
    if (fabsf(q) < pivmin) q = -pivmin;
    c += q < 0.f;
  }
  return c;
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

__host__ __device__ inline int eigh_lda(int n) { return n + ((n & 1) ? 2 : 1); }

// Shared-memory floats per warp.
__host__ __device__ inline size_t eigh_smem_floats(int n) {
  const int lda = eigh_lda(n);
  return (size_t)2 * n * lda + 5 * (size_t)n + (size_t)5 * n * kInvGroup;
}

// grid: one block of 32 threads per patch. ``gram`` (read) and ``vecs``
// (written) may alias: the block reads its whole matrix before writing.
__global__ void __launch_bounds__(32)
    eigh_mp_kernel(const float* gram, float* vecs, float* __restrict__ lam_out,
                   int32_t* __restrict__ ranks, float* __restrict__ wgt, int n, int nvox) {
  extern __shared__ float sm_eig[];
  const int lane = threadIdx.x;
  const long long b = blockIdx.x;
  const int lda = eigh_lda(n);
  float* A = sm_eig;             // n x lda, symmetric working matrix
  float* Y = A + n * lda;        // n x lda, eigenvector j in column j
  float* d = Y + n * lda;        // tridiagonal diagonal
  float* e = d + n;              // sub-diagonal e[0..n-2]
  float* e2 = e + n;             // e^2
  float* tau = e2 + n;           // reflector scalars
  float* lam = tau + n;          // ascending eigenvalues (scaled)
  float* W = lam + n;            // scratch: 5 * n * kInvGroup floats

  // ---- load and scale -----------------------------------------------------
  const float* G = gram + b * (long long)n * n;
  float dmax = 0.f;
  for (int idx = lane; idx < n * n; idx += 32) {
    const int r = idx / n, c = idx - r * n;
    const float v = G[idx];
    A[r * lda + c] = v;
    if (r == c) dmax = fmaxf(dmax, fabsf(v));
  }
  dmax = warp_max(dmax);
  int ex = 0;
  if (dmax > 0.f && isfinite(dmax)) frexpf(dmax, &ex);
  const float scale = ldexpf(1.f, -ex), unscale = ldexpf(1.f, ex);
  __syncwarp();
  for (int idx = lane; idx < n * n; idx += 32) {
    const int r = idx / n, c = idx - r * n;
    A[r * lda + c] *= scale;
  }
  __syncwarp();

  // ---- Householder tridiagonalisation ---------------------------------------
  float* vv = W;
  float* pp = W + n;
  float* ww = W + 2 * n;
  for (int k = 0; k < n - 2; ++k) {
    const int L = n - k - 1;
    float part = 0.f;
    for (int i = 1 + lane; i < L; i += 32) {
      const float v = A[(k + 1 + i) * lda + k];
      part = fmaf(v, v, part);
    }
    const float xnorm2 = warp_sum(part);
    const float alpha = A[(k + 1) * lda + k];
    float taui = 0.f, beta = alpha;
    if (xnorm2 > 0.f) {
      beta = -copysignf(sqrtf(fmaf(alpha, alpha, xnorm2)), alpha);
      taui = (beta - alpha) / beta;
      const float sc = 1.f / (alpha - beta);
      for (int i = 1 + lane; i < L; i += 32) A[(k + 1 + i) * lda + k] *= sc;
    }
    if (lane == 0) {
      e[k] = beta;
      d[k] = A[k * lda + k];
      tau[k] = taui;
    }
    __syncwarp();
    if (taui != 0.f) {
      for (int i = lane; i < L; i += 32) vv[i] = (i == 0) ? 1.f : A[(k + 1 + i) * lda + k];
      __syncwarp();
      for (int i = lane; i < L; i += 32) {
        const float* row = A + (k + 1 + i) * lda + (k + 1);
        float s = 0.f;
        for (int j = 0; j < L; ++j) s = fmaf(row[j], vv[j], s);
        pp[i] = taui * s;
      }
      __syncwarp();
      float part2 = 0.f;
      for (int i = lane; i < L; i += 32) part2 = fmaf(pp[i], vv[i], part2);
      const float kc = -0.5f * taui * warp_sum(part2);
      for (int i = lane; i < L; i += 32) ww[i] = fmaf(kc, vv[i], pp[i]);
      __syncwarp();
      for (int i = lane; i < L; i += 32) {
        const float vi = vv[i], wi = ww[i];
        float* row = A + (k + 1 + i) * lda + (k + 1);
        for (int j = 0; j < L; ++j) row[j] = fmaf(-vi, ww[j], fmaf(-wi, vv[j], row[j]));
      }
      __syncwarp();
    }
  }
  if (lane == 0) {
    if (n >= 2) {
      d[n - 2] = A[(n - 2) * lda + (n - 2)];
      e[n - 2] = A[(n - 1) * lda + (n - 2)];
      tau[n - 2] = 0.f;
    }
    d[n - 1] = A[(n - 1) * lda + (n - 1)];
    e[n - 1] = 0.f;
    tau[n - 1] = 0.f;
  }
  __syncwarp();
  for (int i = lane; i < n; i += 32) e2[i] = (i < n - 1) ? e[i] * e[i] : 0.f;

  // ---- eigenvalues: bisection on Sturm counts -------------------------------
  float glo = FLT_MAX, ghi = -FLT_MAX;
  for (int i = lane; i < n; i += 32) {
    const float r = (i > 0 ? fabsf(e[i - 1]) : 0.f) + (i < n - 1 ? fabsf(e[i]) : 0.f);
    glo = fminf(glo, d[i] - r);
    ghi = fmaxf(ghi, d[i] + r);
  }
  glo = warp_min(glo);
  ghi = warp_max(ghi);
  const float tnorm = fmaxf(fmaxf(fabsf(glo), fabsf(ghi)), FLT_MIN);
  const float eps = FLT_EPSILON * 0.5f;
  glo -= 4.f * eps * tnorm * n;
  ghi += 4.f * eps * tnorm * n;
  const float pivmin = FLT_MIN * 4.f;
  const float abstol = 0.1f * eps * tnorm;
  __syncwarp();
  for (int j = lane; j < n; j += 32) {
    float lo = glo, hi = ghi;
    for (int it = 0; it < 80; ++it) {
      const float tol = fmaxf(abstol, 2.f * eps * fmaxf(fabsf(lo), fabsf(hi)));
      if (hi - lo <= tol) break;
      const float mid = 0.5f * (lo + hi);
      if (mid <= lo || mid >= hi) break;
      if (sturm_count(d, e2, n, mid, pivmin) > j)
        hi = mid;
      else
        lo = mid;
    }
    lam[j] = 0.5f * (lo + hi);
  }
  __syncwarp();

  // ---- MP rank (step0_numpy_loop.py:18-24) ---------------------------------
  const int t = n - 1;
  float* eg = W;      // descending eigs, t entries
  float* rc = W + n;  // suffix sums
  for (int i = lane; i < t; i += 32)
    eg[i] = __fdiv_rn(fmaxf(lam[n - 1 - i] * unscale, 0.f), (float)nvox);
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
      }
      p += __popc(__ballot_sync(0xffffffffu, sig));
    }
  }
  if (lane == 0) {
    ranks[b] = p;
    wgt[b] = (float)(1.0 / (2.0 + (double)p));
  }
  if (lam_out != nullptr)
    for (int i = lane; i < n; i += 32) lam_out[b * n + i] = lam[i] * unscale;
  if (p == 0) return;
  __syncwarp();

  // ---- top-p eigenvectors: inverse iteration on the tridiagonal -------------
  const float pivtol = eps * tnorm;
  float* U0 = W;
  float* U1 = U0 + n * kInvGroup;
  float* U2 = U1 + n * kInvGroup;
  float* ML = U2 + n * kInvGroup;
  float* SW = ML + n * kInvGroup;
  for (int j0 = 0; j0 < p; j0 += kInvGroup) {
    const int g = min(kInvGroup, p - j0);
    if (lane < g) {
      const int j = j0 + lane;        // descending index
      const float sig = lam[n - 1 - j];
      const int q = lane;
      // LU with partial pivoting of (T - sig I)
      float c = d[0] - sig, s = (n > 1) ? e[0] : 0.f;
      for (int i = 0; i < n - 1; ++i) {
        const float ei = e[i];
        const float an = d[i + 1] - sig;
        const float en = (i + 1 < n - 1) ? e[i + 1] : 0.f;
        if (fabsf(c) >= fabsf(ei)) {
          const float m = (ei == 0.f) ? 0.f : ei / c;
          U0[i * kInvGroup + q] = c;
          U1[i * kInvGroup + q] = s;
          U2[i * kInvGroup + q] = 0.f;
          ML[i * kInvGroup + q] = m;
          SW[i * kInvGroup + q] = 0.f;
          c = fmaf(-m, s, an);
          s = en;
        } else {
          const float m = c / ei;
          U0[i * kInvGroup + q] = ei;
          U1[i * kInvGroup + q] = an;
          U2[i * kInvGroup + q] = en;
          ML[i * kInvGroup + q] = m;
          SW[i * kInvGroup + q] = 1.f;
          c = fmaf(-m, an, s);
          s = -m * en;
        }
      }
      U0[(n - 1) * kInvGroup + q] = c;
      for (int i = 0; i < n; ++i) {
        const float u = U0[i * kInvGroup + q];
        if (fabsf(u) < pivtol) U0[i * kInvGroup + q] = (u < 0.f) ? -pivtol : pivtol;
      }
      // start vector
      for (int i = 0; i < n; ++i) Y[i * lda + j] = start_entry(i, j);
      for (int iter = 0; iter < 3; ++iter) {
        for (int i = 0; i < n - 1; ++i) {
          const float bi = Y[i * lda + j], bi1 = Y[(i + 1) * lda + j];
          const float m = ML[i * kInvGroup + q];
          if (SW[i * kInvGroup + q] != 0.f) {
            Y[i * lda + j] = bi1;
            Y[(i + 1) * lda + j] = fmaf(-m, bi1, bi);
          } else {
            Y[(i + 1) * lda + j] = fmaf(-m, bi, bi1);
          }
        }
        float x2 = Y[(n - 1) * lda + j] / U0[(n - 1) * kInvGroup + q];
        Y[(n - 1) * lda + j] = x2;
        float x1 = x2, amax = fabsf(x2);
        if (n >= 2) {
          x1 = (Y[(n - 2) * lda + j] - U1[(n - 2) * kInvGroup + q] * x2) / U0[(n - 2) * kInvGroup + q];
          Y[(n - 2) * lda + j] = x1;
          amax = fmaxf(amax, fabsf(x1));
        }
        for (int i = n - 3; i >= 0; --i) {
          const float xi = (Y[i * lda + j] - U1[i * kInvGroup + q] * x1 - U2[i * kInvGroup + q] * x2) /
                           U0[i * kInvGroup + q];
          Y[i * lda + j] = xi;
          amax = fmaxf(amax, fabsf(xi));
          x2 = x1;
          x1 = xi;
        }
        // normalise with a max-abs prescale (the solve can grow by 1/pivtol per
        // tiny pivot); a non-finite solve restarts from a fresh start vector
        if (!(amax > 0.f) || !isfinite(amax)) {
          for (int i = 0; i < n; ++i) Y[i * lda + j] = start_entry(i, j + 977 * (iter + 1));
          continue;
        }
        const float sa = 1.f / amax;
        float nrm = 0.f;
        for (int i = 0; i < n; ++i) {
          const float v = Y[i * lda + j] * sa;
          Y[i * lda + j] = v;
          nrm = fmaf(v, v, nrm);
        }
        const float inv = rsqrtf(nrm);
        for (int i = 0; i < n; ++i) Y[i * lda + j] *= inv;
      }
    }
    __syncwarp();
  }

  // ---- modified Gram-Schmidt, descending eigenvalue order --------------------
  for (int j = 0; j < p; ++j) {
    for (int i = 0; i < j; ++i) {
      float part = 0.f;
      for (int r = lane; r < n; r += 32) part = fmaf(Y[r * lda + i], Y[r * lda + j], part);
      const float dot = warp_sum(part);
      for (int r = lane; r < n; r += 32) Y[r * lda + j] = fmaf(-dot, Y[r * lda + i], Y[r * lda + j]);
      __syncwarp();
    }
    float part = 0.f;
    for (int r = lane; r < n; r += 32) part = fmaf(Y[r * lda + j], Y[r * lda + j], part);
    const float inv = rsqrtf(fmaxf(warp_sum(part), FLT_MIN));
    for (int r = lane; r < n; r += 32) Y[r * lda + j] *= inv;
    __syncwarp();
  }

  // ---- back-transform: x = H(0) H(1) ... H(n-3) y, one lane per vector ------
  for (int j = lane; j < p; j += 32) {
    for (int k = n - 3; k >= 0; --k) {
      const float tk = tau[k];
      if (tk == 0.f) continue;
      const int L = n - k - 1;
      float dot = Y[(k + 1) * lda + j];
      for (int i = 1; i < L; ++i) dot = fmaf(A[(k + 1 + i) * lda + k], Y[(k + 1 + i) * lda + j], dot);
      const float f = tk * dot;
      Y[(k + 1) * lda + j] -= f;
      for (int i = 1; i < L; ++i) Y[(k + 1 + i) * lda + j] = fmaf(-f, A[(k + 1 + i) * lda + k], Y[(k + 1 + i) * lda + j]);
    }
  }
  __syncwarp();
  // compact row-major n x p block at the start of the patch's n x n slot
  float* V = vecs + b * (long long)n * n;
  for (int idx = lane; idx < n * p; idx += 32) {
    const int r = idx / p, c = idx - r * p;
    V[idx] = Y[r * lda + c];
  }
}

}  // namespace lrd
