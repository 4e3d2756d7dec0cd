// Packed multi-volume launches of the batched form (lrd_batch_*): one grid
// per phase and kernel class covers every volume of the batch.
//
// Each volume of a batch has a descriptor (BatchVol: its buffers, geometry,
// index tables and the TMA plane map over its centred volume) in one device
// array. A launch covers a list of volumes; volume list[i] owns the launch's
// blocks [off[i], off[i + 1]), so a block finds its volume by a binary search
// over the offsets and runs the single-volume kernel body (the same device
// function the per-volume kernels run) with its block index within that
// volume. Volumes therefore compute exactly what a single-volume call
// computes - the batch only changes how the blocks are launched: 24 volumes
// of mixed shapes take one grid per phase and frame-count class instead of
// six launches each.
#pragma once

#include <cuda.h>

#include "center.cuh"
#include "eigh.cuh"
#include "eigh_cta.cuh"
#include "eigh_reg.cuh"
#include "gram_z.cuh"
#include "lrd_common.cuh"
#include "recon_warp.cuh"

namespace lrd {

struct alignas(64) BatchVol {
  CUtensorMap map;       // plane map over xc (gram_z), 64-byte aligned: first member
  const float* vol;      // input volume
  float* out;            // output volume
  int32_t* ranks_out;    // nullable
  float* mean;           // workspace buffers of this volume
  float* xc;
  float* gv;             // Gram blocks, overwritten by the top-p eigenvectors
  int32_t* rank;
  float* wgt;
  float* sig2;
  int* status;
  int* refine;           // [count, refined, 62 unused, ids...]
  Geom g;
  AxisTables tab;
  int ring;              // gram_z window slots
};

// Index i of the list entry whose block range holds block b (off has n + 1
// entries, off[0] = 0, nondecreasing).
__device__ __forceinline__ int batch_find(const long long* __restrict__ off, int n, long long b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Clears every volume's status word and near-tie queue cursor (what the
// single-volume call does with two memsets).
__global__ void batch_reset_kernel(const BatchVol* __restrict__ vols, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    *vols[i].status = 0;
    vols[i].refine[0] = 0;
    vols[i].refine[1] = 0;
  }
}

__global__ void center_batch_kernel(const BatchVol* __restrict__ vols, const int* __restrict__ list,
                                    const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  const long long nvox = (long long)V.g.nx * V.g.ny * V.g.nz;
  center_body(V.vol, V.xc, V.mean, nvox, V.g.nt, (long long)blockIdx.x - off[i]);
}

// Column Gram, every column of each listed volume (no short-last-wave cut:
// the batch's columns fill the device).
template <int KS>
__global__ void __maxnreg__(64) gram_z_batch_kernel(const BatchVol* __restrict__ vols, const int* __restrict__ list,
                                                    const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  if (threadIdx.x == 0)  // the map was written by a copy before this launch; order it for the TMA unit
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&V.map) : "memory");
  const long long ncols = (long long)V.g.ncx * V.g.ncy;
  gram_z_body<KS>(&V.map, V.gv, V.g, V.tab, 0, V.ring, (int)ncols, 1, V.status, (int)(blockIdx.x - off[i]));
}

template <int TMAX>
__global__ void __launch_bounds__(32, eigh_reg_min_blocks<TMAX>()) eigh_reg_batch_kernel(const BatchVol* __restrict__ vols,
                                                            const int* __restrict__ list,
                                                            const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  eigh_reg_body<TMAX, false>(V.gv, V.gv, nullptr, V.rank, V.wgt, V.sig2, V.g.nt, V.g.nvox_patch, 0, V.refine,
                      V.refine + 64, (long long)blockIdx.x - off[i]);
}

template <int TMAX>
__global__ void __launch_bounds__(TMAX) eigh_cta_batch_kernel(const BatchVol* __restrict__ vols,
                                                              const int* __restrict__ list,
                                                              const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  eigh_cta_body<TMAX>(V.gv, V.gv, nullptr, V.rank, V.wgt, V.sig2, V.g.nt, V.g.nvox_patch, 0, V.refine,
                      V.refine + 64, (long long)blockIdx.x - off[i]);
}

// Float64 near-tie pass: each listed volume's queue is worked by its blocks.
__global__ void eigh_refine_batch_kernel(const BatchVol* __restrict__ vols, const int* __restrict__ list,
                                         const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  eigh_refine_body(V.vol, V.xc, V.gv, nullptr, V.rank, V.wgt, V.sig2, V.g, V.tab, V.refine, V.refine + 64,
                   (int)(blockIdx.x - off[i]), (int)(off[i + 1] - off[i]));
}

__global__ void refine_advance_batch_kernel(const BatchVol* __restrict__ vols, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    vols[i].refine[1] = vols[i].refine[0];
}

template <int Q, bool ACCURATE>
__global__ void __launch_bounds__(32 * kReconWarps)
    recon_warp_batch_kernel(const BatchVol* __restrict__ vols, const int* __restrict__ list,
                            const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  const SlabIO io{0, V.g.nx, 0, nullptr, V.g.nx, nullptr};
  recon_warp_body<Q, ACCURATE>(V.xc, V.mean, V.gv, V.rank, V.wgt, V.out, V.g, V.tab, 0, io,
                               (int)(blockIdx.x - off[i]));
}

// Ranks of every listed volume that asked for them, into its rank array.
__global__ void ranks_batch_kernel(const BatchVol* __restrict__ vols, const int* __restrict__ list,
                                   const long long* __restrict__ off, int n) {
  const int i = batch_find(off, n, blockIdx.x);
  const BatchVol& V = vols[list[i]];
  const long long p = (long long)(blockIdx.x - off[i]) * blockDim.x + threadIdx.x;
  if (V.ranks_out != nullptr && p < V.g.npatch) V.ranks_out[p] = V.rank[p];
}

}  // namespace lrd
