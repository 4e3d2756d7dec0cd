// C ABI of the MP-PCA denoiser: plans, workspace, launches (include/lrd.h).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lrd.h"
#include "center.cuh"
#include "eigh.cuh"
#include "eigh_reg.cuh"
#include "eigh_cta.cuh"
#include "noise.cuh"
#include "gram.cuh"
#include "gram_tc.cuh"
#include "gram_z.cuh"
#include "lrd_common.cuh"
#include "recon.cuh"
#include "recon_tc.cuh"
#include "recon_warp.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t err, const char* what) {
  return fail(LRD_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(err), cudaGetErrorName(err));
}

#define LRD_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Sorted corner positions along one axis (common.py:40-43):
// sorted({*range(0, s - p + 1, step), s - p}).
std::vector<int32_t> axis_corners(int size, int patch, int stride) {
  std::vector<int32_t> c;
  for (int v = 0; v <= size - patch; v += stride) c.push_back(v);
  if (c.empty() || c.back() != size - patch) c.push_back(size - patch);
  return c;
}

}  // namespace

struct lrd_plan {
  lrd_problem prob;
  lrd::Geom g;
  int device;
  long long nvox;
  int tpt;                 // recon frames per thread
  int split;               // recon threads per voxel
  bool recon_warp = false; // reconstruction by recon_warp_kernel (2 x 2 x 2 voxels per warp)
  bool recon_tc = false;   // reconstruction by recon_tc_kernel (tensor forms: 4 x 4 x 8 bricks on tcgen05)
  size_t smem_recon_tc = 0;
  int gram_threads;
  bool use_gramz;          // column Gram kernel (TMA-staged z-planes) instead of per-patch
  bool use_gramtc;         // the column Gram on tcgen05 (tensor forms)
  bool gramtc_bf16 = false; // ... with BF16 3-term split operands instead of 3xTF32
  size_t smem_gramtc;
  int gramz_ring;          // window accumulator slots
  int gramz_ks = 1;        // voxel-row split per 4x4 Gram block (threads per block)
  bool eigh_cta = false;   // eigensolver: one CTA per matrix (else one warp)
  size_t smem_gramz;
  int gramz_slots = 0;     // column CTAs resident at once on the device (0: never cut columns)
  int gramtc_slots = 0;    // the same for the tensor-core column Gram
  int sms = 0;             // multiprocessors of the device
  size_t smem_center, smem_gram, smem_eigh, smem_recon;
  int center_warps;
  // workspace offsets (bytes)
  size_t off_mean, off_xc, off_gv, off_rank, off_wgt, off_sig2, off_status, off_refine, ws_bytes;
  size_t smem_refine;
  int refine_blocks;
  // device tables (one allocation)
  void* d_tables;
  lrd::AxisTables tab;
  // host copies of the x-axis tables (host-buffer pipeline) and its streams/events
  std::vector<int32_t> h_corner_x, h_brick_x;
  cudaStream_t io_in = nullptr, io_out = nullptr;
  cudaStream_t io_prep[3] = {nullptr, nullptr, nullptr};  // centre + Gram of slab s on io_prep[s % 3]
  cudaStream_t io_recon = nullptr;                         // reconstruction of the slabs (even ones in
  cudaStream_t io_recon2 = nullptr;                        //   the host pipeline; odd ones on io_recon2)
  cudaStream_t io_solve = nullptr;                         // solves of odd slabs (even ones: the caller's;
  cudaStream_t io_solve2 = nullptr;                        //   host pipeline: slab s on s % 3 of the three)
  std::vector<cudaEvent_t> io_events;  // 5 per slab + 1
  // device-resident pipeline of lrd_denoise: x-slabs whose Gram, solve and
  // reconstruction overlap on the plan's streams (1 = one pass per phase);
  // the enqueue of a call holds the mutex (the streams and events are shared)
  int dev_slabs = 1;
  mutable std::mutex pipe_mu;
  // measurement hook: a ring of per-call phase events
  bool profiling = false;
  int prof_calls = 0;
  std::vector<cudaEvent_t> prof_events;  // kProfRing * (LRD_NUM_PHASES + 1)
  // slab of a sharded volume: local plane 0 is global plane slab_x0; planes
  // [0, slab_hin) continue the lower slab's sums, planes [slab_own_hi, nx) are
  // handed to the upper slab
  bool is_slab = false;
  int slab_x0 = 0, slab_hin = 0, slab_own_hi = 0, slab_ci_lo = 0, slab_ci_hi = 0, slab = 0, n_slabs = 1;
};

namespace {
constexpr int kProfRing = 256;
constexpr int kIoSlabs = 16;     // event capacity of the host-buffer pipeline
// x-slabs the host-buffer pipeline uses (about 3.5 MiB of input each, at most
// this many). Measured e2e at 96x96x48x48 / 11^3 / stride 3 on B200 (ms), one
// reconstruction stream: 4 slabs 4.73, 6 4.74, 8 4.62, 10 4.55, 12 4.62, 16
// 5.05; with the current kernels 8 3.61, 10 3.60, 12 3.62; two alternating
// reconstruction streams: 8 3.61, 10 3.51, 12 3.48; and two / three / four
// solve streams: 12 slabs 3.48 / 3.48 / 3.60, 16 3.49 / 3.38 / 3.53, 20
// 3.63 / 3.45 / 3.65, 24 3.90 / 3.60 / 3.73. At 48x48x24x48 (10 MiB), three
// solve streams: 1 slab 0.83, 2 0.73, 3 0.70, 4 0.72, 5 0.73.
constexpr int kIoSlabsUsed = 16;
constexpr long long kIoSlabBytes = 7ll << 19;
}

namespace {

// Voxel-row split of the column Gram. Measured on B200 (96x96x48xT, 11^3,
// stride 3, before short last waves were cut into window ranges): T = 48
// runs 0.80 ms with 2 threads per block (160-thread CTAs)
// against 0.96 ms unsplit and 1.27 ms with 4; T = 32, 64 and 96 are fastest
// unsplit (0.58 / 1.44 / 1.21 ms, the split costing 30-60%).
int gramz_split(int T) { return (T > 40 && T <= 56) ? 2 : 1; }

void* gramtc_kernel_ptr(bool bf16) {
  return bf16 ? (void*)lrd::gram_tc_kernel<true> : (void*)lrd::gram_tc_kernel<false>;
}

void* gramz_kernel_ptr(int ks) {
  switch (ks) {
    case 2: return (void*)lrd::gram_z_kernel<2>;
    case 4: return (void*)lrd::gram_z_kernel<4>;
    default: return (void*)lrd::gram_z_kernel<1>;
  }
}

// Reconstruction thread layout for T frames: two threads per voxel up to
// T = 48, four above (a thread's frame slices, accumulators and projections
// live in registers: 3 x T/split of them). Measured on B200, reconstruction
// ms, brick 3x3x3, split 2 -> 4: T = 64 at 11^3 / stride 1 181 -> 82,
// 11^3 / stride 2 27 -> 16, 5^3 / stride 1 13.5 -> 7.9; T = 96 at 7^3 /
// stride 1 30 -> 27; T = 48 at 11^3 / stride 3 1.32 -> 1.53 (keeps 2); one
// thread per voxel needs ~220 registers at T = 48 and measured 3.4x slower.
// The forms that accumulate in float64 (accurate, tensor) take four threads
// at every T: their accumulators double the registers (T = 48 headline:
// 3.62 -> 1.68 ms).
// The frames are cut into four chunks of Q = round4(ceil(T/4)) and a thread
// owns 4/split consecutive chunks (TPT = Q * 4 / split), so every split sums
// y_k in the same tree.
void pick_recon_layout(int T, int want_split, bool acc64, int& split, int& tpt) {
  split = (T <= 48 && !acc64) ? 2 : 4;
  if (want_split == 1 || want_split == 2 || want_split == 4) split = want_split;
  if (T > 48 && split < 2) split = 2;  // one thread per voxel is built up to T = 48
  if (T > 96 && split < 4) split = 4;  // two up to T = 96
  const int q = (((T + 3) / 4) + 3) & ~3;
  tpt = q * 4 / split;
}

// Brick choice for the reconstruction: minimise the thread-slots the CTAs spend
// on (voxel, touching patch) pairs, per axis sum_b touch(b) * b, with 64..512
// threads per CTA.
struct BrickAxis {
  long long slots;
  int nblocks;
};

BrickAxis brick_axis_cost(int size, int patch, const std::vector<int32_t>& corners, int bsz) {
  BrickAxis r{0, (size + bsz - 1) / bsz};
  for (int b = 0; b < r.nblocks; ++b) {
    const int lo = b * bsz, hi = std::min(size, lo + bsz) - 1;
    int touch = 0;
    for (int32_t c : corners)
      if (c <= hi && c + patch - 1 >= lo) ++touch;
    r.slots += (long long)touch * bsz;
  }
  return r;
}

// Largest number of patches touching one brick (the recon kernel stages their
// ranks and weights in shared memory).
int max_touch(const std::vector<int32_t> brick[3]) {
  int best = 0;
  for (size_t a = 0; a < brick[0].size() / 2; ++a)
    for (size_t b = 0; b < brick[1].size() / 2; ++b)
      for (size_t c = 0; c < brick[2].size() / 2; ++c) {
        const int n = std::max(0, brick[0][2 * a + 1] - brick[0][2 * a] + 1) *
                      std::max(0, brick[1][2 * b + 1] - brick[1][2 * b] + 1) *
                      std::max(0, brick[2][2 * c + 1] - brick[2][2 * c] + 1);
        best = std::max(best, n);
      }
  return best;
}

// Default reconstruction brick: 27..128 threads per CTA (small CTAs keep
// several resident per SM), fewest (voxel, touching patch) thread slots -
// counting the idle lanes of a partial last warp - plus a small per-(brick,
// patch) staging cost.
void choose_brick(const int dims[3], const int pat[3], const std::vector<int32_t> corners[3], int split,
                  int best[3]) {
  double best_cost = 1e300;
  for (int bx = 1; bx <= 16; ++bx)
    for (int by = 1; by <= 16; ++by)
      for (int bz = 1; bz <= 32; ++bz) {
        const int threads = bx * by * bz * split;
        if (threads < 27 || threads > 128) continue;
        if ((bx > dims[0] && bx > 1) || (by > dims[1] && by > 1) || (bz > dims[2] && bz > 1)) continue;
        const BrickAxis ax = brick_axis_cost(dims[0], pat[0], corners[0], bx);
        const BrickAxis ay = brick_axis_cost(dims[1], pat[1], corners[1], by);
        const BrickAxis az = brick_axis_cost(dims[2], pat[2], corners[2], bz);
        const double pad = (double)((threads + 31) / 32 * 32) / threads;
        const double touch = (double)ax.slots / bx * ay.slots / by * az.slots / bz;
        const double cost = (double)ax.slots * ay.slots * az.slots * pad + 4.0 * touch;
        if (cost < best_cost) {
          best_cost = cost;
          best[0] = bx;
          best[1] = by;
          best[2] = bz;
        }
      }
}

// Float32 eigensolver kernel, its threads and shared-memory floats for frame
// count T: one warp per matrix (register-resident rows) up to T = 64, one
// CTA of TMAX threads per matrix (TMAX = 64, 96, 128) above or when asked.
bool eigh_use_cta(int T, int eigh_block) { return eigh_block == 2 || (eigh_block == 0 && T > 64); }
size_t eigh_smem_for(int T, bool cta) {
  if (cta) {
    if (T <= 64) return lrd::eigh_cta_smem_floats<64>();
    if (T <= 96) return lrd::eigh_cta_smem_floats<96>();
    return lrd::eigh_cta_smem_floats<128>();
  }
  if (T <= 32) return lrd::eigh_reg_smem_floats<32>();
  if (T <= 48) return lrd::eigh_reg_smem_floats<48>();
  return lrd::eigh_reg_smem_floats<64>();
}
const void* eigh_kernel_for(int T, bool cta, unsigned* threads = nullptr) {
  if (threads) *threads = cta ? (T <= 64 ? 64u : (T <= 96 ? 96u : 128u)) : 32u;
  if (cta) {
    if (T <= 64) return (const void*)lrd::eigh_cta_kernel<64>;
    if (T <= 96) return (const void*)lrd::eigh_cta_kernel<96>;
    return (const void*)lrd::eigh_cta_kernel<128>;
  }
  if (T <= 32) return (const void*)lrd::eigh_reg_kernel<32>;
  if (T <= 48) return (const void*)lrd::eigh_reg_kernel<48>;
  return (const void*)lrd::eigh_reg_kernel<64>;
}

template <int TPT, int SPLIT>
void* recon_fn(bool accurate) {
  return accurate ? (void*)lrd::recon_kernel<TPT, SPLIT, true> : (void*)lrd::recon_kernel<TPT, SPLIT, false>;
}

void* recon_kernel_ptr(int tpt, int split, bool accurate) {
  if (split == 1) {
    switch (tpt) {
      case 16: return recon_fn<16, 1>(accurate);
      case 32: return recon_fn<32, 1>(accurate);
      case 48: return recon_fn<48, 1>(accurate);
    }
  } else if (split == 2) {
    switch (tpt) {
      case 8: return recon_fn<8, 2>(accurate);
      case 16: return recon_fn<16, 2>(accurate);
      case 24: return accurate ? recon_fn<24, 2>(true) : (void*)lrd::recon_kernel_t24s2;
      case 32: return recon_fn<32, 2>(accurate);
      case 40: return recon_fn<40, 2>(accurate);
      case 48: return recon_fn<48, 2>(accurate);
    }
  } else if (split == 4) {
    switch (tpt) {
      case 4: return recon_fn<4, 4>(accurate);
      case 8: return recon_fn<8, 4>(accurate);
      case 12: return recon_fn<12, 4>(accurate);
      case 16: return recon_fn<16, 4>(accurate);
      case 20: return recon_fn<20, 4>(accurate);
      case 24: return recon_fn<24, 4>(accurate);
      case 28: return recon_fn<28, 4>(accurate);
      case 32: return recon_fn<32, 4>(accurate);
    }
  }
  return nullptr;
}

void* recon_warp_ptr(int T, bool accurate) {
  switch (T) {
    case 32: return accurate ? (void*)lrd::recon_warp_kernel<8, true> : (void*)lrd::recon_warp_kernel<8, false>;
    case 48: return accurate ? (void*)lrd::recon_warp_kernel<12, true> : (void*)lrd::recon_warp_kernel<12, false>;
    case 64: return accurate ? (void*)lrd::recon_warp_kernel<16, true> : (void*)lrd::recon_warp_kernel<16, false>;
    case 96: return accurate ? (void*)lrd::recon_warp_kernel<24, true> : (void*)lrd::recon_warp_kernel<24, false>;
  }
  return nullptr;
}

void* recon_tc_ptr(int T) {
  switch (lrd::recon_tc_tn(T)) {
    case 16: return (void*)lrd::recon_tc_kernel<16>;
    case 32: return (void*)lrd::recon_tc_kernel<32>;
    case 48: return (void*)lrd::recon_tc_kernel<48>;
    default: return (void*)lrd::recon_tc_kernel<64>;
  }
}

// The dynamic shared-memory limit is a property of the kernel, shared by
// every plan in the process: only ever raise it (per device and kernel), so a
// plan created later with a smaller need cannot shrink an earlier plan's.
std::mutex g_smem_mu;
std::map<std::pair<int, const void*>, size_t> g_smem_set;

int set_smem(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return LRD_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_smem_mu);
  size_t& cur = g_smem_set[{dev, fn}];
  if (bytes <= cur) return LRD_OK;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(max dynamic smem)");
  cur = bytes;
  return LRD_OK;
}

int launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  return LRD_OK;
}

// Centre voxel rows [v0, v0 + nv).
int run_center(const lrd_plan* P, const float* d_vol, char* ws, cudaStream_t st, long long v0 = 0,
               long long nv = -1) {
  if (nv < 0) nv = P->nvox - v0;
  if (nv <= 0) return LRD_OK;
  float* mean = reinterpret_cast<float*>(ws + P->off_mean);
  float* xc = reinterpret_cast<float*>(ws + P->off_xc);
  const int T = P->g.nt;
  const long long per_block = 32LL * P->center_warps;
  const long long blocks = (nv + per_block - 1) / per_block;
  lrd::center_kernel<<<(unsigned)blocks, 32 * P->center_warps, P->smem_center, st>>>(
      d_vol + v0 * T, xc + v0 * T, mean + v0, nv, T);
  return launch_check("center_kernel launch");
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// 4D tensor map over the centred volume (t, z, y, x), box (T, 1, py, px): one
// z-plane of one patch column per TMA load.
int encode_plane_map(const lrd_plan* P, const float* xc, CUtensorMap* map) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(LRD_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const lrd::Geom& g = P->g;
  const cuuint64_t dims[4] = {(cuuint64_t)g.nt, (cuuint64_t)g.nz, (cuuint64_t)g.ny, (cuuint64_t)g.nx};
  const cuuint64_t strides[3] = {(cuuint64_t)g.nt * 4, (cuuint64_t)g.nz * g.nt * 4,
                                 (cuuint64_t)g.ny * g.nz * g.nt * 4};
  const cuuint32_t box[4] = {(cuuint32_t)g.nt, 1, (cuuint32_t)g.py, (cuuint32_t)g.px};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(xc), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(LRD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return LRD_OK;
}

// Gram matrices of the patch columns [col_lo, col_hi) (x-major column index
// ci * ncy + cj; -1 = all), i.e. of patches [col_lo * ncz, col_hi * ncz).
// ``spread``: a launch of fewer columns than the device holds at once has all
// of them cut into window ranges (more, shorter CTAs: lower latency for more
// plane reads, for a Gram on the critical path of an otherwise idle device).
int run_gram(const lrd_plan* P, char* ws, float* d_gram, cudaStream_t st, long long col_lo = 0,
             long long col_hi = -1, bool spread = false) {
  const float* xc = reinterpret_cast<const float*>(ws + P->off_xc);
  const long long ncol = (long long)P->g.ncx * P->g.ncy;
  if (col_hi < 0) col_hi = ncol;
  if (col_hi <= col_lo) return LRD_OK;
  const long long TT = (long long)P->g.nt * P->g.nt;
  if (P->use_gramz || P->use_gramtc) {
    CUtensorMap map;
    int rc = encode_plane_map(P, xc, &map);
    if (rc) return rc;
    int* status = reinterpret_cast<int*>(ws + P->off_status);
    const long long cols = P->prob.batch > 0 ? std::max<long long>(1, P->prob.batch / P->g.ncz) : ncol;
    for (long long c0 = col_lo; c0 < col_hi; c0 += cols) {
      const long long nc = std::min(cols, col_hi - c0);
      // A last wave of a few whole columns would leave most SMs idle while
      // they finish: cut those columns into window ranges instead.
      const long long slots = P->use_gramtc ? P->gramtc_slots : P->gramz_slots;
      long long nfull = nc;
      int nsplit = 1;
      const long long rem = slots > 0 ? nc % slots : 0;
      if (spread && slots > 0 && nc < slots && P->g.ncz > 1) {
        nsplit = (int)std::min<long long>(P->g.ncz, std::max<long long>(1, slots / nc));
        if (nsplit > 1) nfull = 0;
        else nsplit = 1;
      } else if (slots > 0 && nc > slots && rem > 0 && 2 * rem <= slots && P->g.ncz > 1) {
        nsplit = (int)std::min<long long>(P->g.ncz, slots / rem);
        if (nsplit > 1) nfull = nc - rem;
        else nsplit = 1;
      }
      const long long grid = nfull + (nc - nfull) * nsplit;
      if (P->use_gramtc) {
        if (P->gramtc_bf16)
          lrd::gram_tc_kernel<true><<<(unsigned)grid, lrd::kGramTcThreads, P->smem_gramtc, st>>>(
              map, d_gram + c0 * P->g.ncz * TT, P->g, P->tab, c0, P->gramz_ring, (int)nfull, nsplit, status);
        else
          lrd::gram_tc_kernel<false><<<(unsigned)grid, lrd::kGramTcThreads, P->smem_gramtc, st>>>(
              map, d_gram + c0 * P->g.ncz * TT, P->g, P->tab, c0, P->gramz_ring, (int)nfull, nsplit, status);
        rc = launch_check("gram_tc_kernel launch");
      } else {
        void* fn = gramz_kernel_ptr(P->gramz_ks);
        float* gout = d_gram + c0 * P->g.ncz * TT;
        lrd::Geom gg = P->g;
        lrd::AxisTables tt = P->tab;
        int ring = P->gramz_ring, nf = (int)nfull;
        void* args[] = {(void*)&map, (void*)&gout, (void*)&gg, (void*)&tt, (void*)&c0, (void*)&ring,
                        (void*)&nf, (void*)&nsplit, (void*)&status};
        cudaError_t le = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(lrd::gramz_threads(P->g.nt, P->gramz_ks)),
                                          args, P->smem_gramz, st);
        if (le != cudaSuccess) return cuda_fail(le, "gram_z_kernel launch");
        rc = launch_check("gram_z_kernel launch");
      }
      if (rc) return rc;
    }
    return LRD_OK;
  }
  const long long p_lo = col_lo * P->g.ncz, p_hi = col_hi * P->g.ncz;
  const long long batch = P->prob.batch > 0 ? P->prob.batch : (p_hi - p_lo);
  for (long long p0 = p_lo; p0 < p_hi; p0 += batch) {
    const long long nb = std::min(batch, p_hi - p0);
    lrd::gram_kernel<<<(unsigned)nb, P->gram_threads, P->smem_gram, st>>>(xc, d_gram + p0 * TT, P->g,
                                                                         P->tab, p0);
    int rc = launch_check("gram_kernel launch");
    if (rc) return rc;
  }
  return LRD_OK;
}

// Float32 eigensolver over patches [p_lo, p_hi) (-1 = all), then the float64
// pass over the near-tie patches it queued (the queue lives in the workspace:
// [count, refined, 62 unused, ids...]; the centred volume there is the one
// the Gram was formed from). ``reset`` clears the queue first.
int run_eigh(const lrd_plan* P, char* ws, const float* d_gram, float* d_vecs, float* d_lam, int32_t* d_rank,
             float* d_wgt, cudaStream_t st, long long p_lo = 0, long long p_hi = -1, bool reset = true,
             const float* d_vol = nullptr, int queue = -1) {
  const long long npatch = P->g.npatch;
  if (p_hi < 0) p_hi = npatch;
  const long long batch = P->prob.batch > 0 ? P->prob.batch : npatch;
  const int T = P->g.nt;
  const long long TT = (long long)T * T;
  int* rcount = reinterpret_cast<int*>(ws + P->off_refine);
  int* rids = rcount + 64;
  if (queue >= 0) {
    // a private near-tie queue for patches [p_lo, p_hi): its counters at header
    // ints 2 + 2q, 3 + 2q (zeroed by the caller), its ids where those patches'
    // would go, so solves of different patch ranges can run at the same time
    rcount += 2 + 2 * queue;
    rids += p_lo;
  }
  float* sig2 = reinterpret_cast<float*>(ws + P->off_sig2);
  if (reset) LRD_CUDA(cudaMemsetAsync(rcount, 0, 2 * sizeof(int), st));
  for (long long p0 = p_lo; p0 < p_hi; p0 += batch) {
    const long long nb = std::min(batch, p_hi - p0);
    const float* gin = d_gram + p0 * TT;
    float* vout = d_vecs + p0 * TT;
    float* lout = d_lam ? d_lam + p0 * T : nullptr;
    int32_t* r = d_rank + p0;
    float* w = d_wgt + p0;
    float* s2 = sig2 + p0;
    const int nv = P->g.nvox_patch;
    unsigned eth = 32;
    const void* efn = eigh_kernel_for(T, P->eigh_cta, &eth);
    long long p0v = p0;
    int tv = T, nvv = nv;
    void* eargs[] = {(void*)&gin, (void*)&vout, (void*)&lout, (void*)&r,      (void*)&w,   (void*)&s2,
                     (void*)&tv,  (void*)&nvv,  (void*)&p0v,  (void*)&rcount, (void*)&rids};
    cudaError_t le = cudaLaunchKernel(efn, dim3((unsigned)nb), dim3(eth), eargs, P->smem_eigh, st);
    if (le != cudaSuccess) return cuda_fail(le, "eigh kernel launch");
    int rc = launch_check("eigh kernel launch");
    if (rc) return rc;
  }
  const float* xc = reinterpret_cast<const float*>(ws + P->off_xc);
  lrd::eigh_refine_kernel<<<P->refine_blocks, 128, P->smem_refine, st>>>(d_vol, xc, d_vecs, d_lam, d_rank, d_wgt,
                                                                        sig2,
                                                                        P->g, P->tab, rcount, rids);
  int rc = launch_check("eigh_refine_kernel launch");
  if (rc) return rc;
  lrd::refine_advance_kernel<<<1, 1, 0, st>>>(rcount);
  return launch_check("refine_advance_kernel launch");
}

// Reconstruction of bricks [b_lo, b_hi) (x-major brick index; -1 = all).
// ``io`` restricts the voxels to an x-range and routes slab halos (slab
// sharding); nullptr = every voxel, normalised into ``d_out``.
int run_recon(const lrd_plan* P, char* ws, float* d_out, cudaStream_t st, long long b_lo = 0, long long b_hi = -1,
              const lrd::SlabIO* io = nullptr) {
  const float* xc = reinterpret_cast<const float*>(ws + P->off_xc);
  const float* mean = reinterpret_cast<const float*>(ws + P->off_mean);
  const float* gv = reinterpret_cast<const float*>(ws + P->off_gv);
  const int32_t* rank = reinterpret_cast<const int32_t*>(ws + P->off_rank);
  const float* wgt = reinterpret_cast<const float*>(ws + P->off_wgt);
  const bool acc = P->prob.form != LRD_FORM_PLAIN;
  const long long nbricks = (long long)P->g.nbx * P->g.nby * P->g.nbz;
  if (b_hi < 0) b_hi = nbricks;
  if (b_hi <= b_lo) return LRD_OK;
  const unsigned threads = P->recon_tc     ? (unsigned)lrd::kRtcThreads
                           : P->recon_warp ? 32u * lrd::kReconWarps
                                           : (unsigned)(P->g.bx * P->g.by * P->g.bz * P->split);
  void* fn = P->recon_tc     ? recon_tc_ptr(P->g.nt)
             : P->recon_warp ? recon_warp_ptr(P->g.nt, acc)
                             : recon_kernel_ptr(P->tpt, P->split, acc);
  const size_t smem = P->recon_tc ? P->smem_recon_tc : (P->recon_warp ? 0 : P->smem_recon);
  lrd::Geom g = P->g;
  lrd::AxisTables tab = P->tab;
  int brick0 = (int)b_lo;
  lrd::SlabIO sio{0, g.nx, 0, nullptr, g.nx, nullptr};
  if (io) sio = *io;
  int* status = reinterpret_cast<int*>(ws + P->off_status);
  void* args[] = {(void*)&xc, (void*)&mean, (void*)&gv,  (void*)&rank,   (void*)&wgt,   (void*)&d_out,
                  (void*)&g,  (void*)&tab,  (void*)&brick0, (void*)&sio, (void*)&status};
  cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)(b_hi - b_lo)), dim3(threads), args, smem, st);
  if (e != cudaSuccess) return cuda_fail(e, "recon_kernel launch");
  return LRD_OK;
}

int check_plan(const lrd_plan* P) {
  if (!P) return fail(LRD_ERR_INVALID, "plan is NULL");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != P->device)
    return fail(LRD_ERR_INVALID, "plan was created on device %d but device %d is current", P->device, dev);
  return LRD_OK;
}

// Checks of a problem shared by every entry point that takes one.
int validate_problem(const lrd_problem* pr) {
  const int dims[3] = {pr->nx, pr->ny, pr->nz};
  const int pat[3] = {pr->px, pr->py, pr->pz};
  for (int a = 0; a < 3; ++a) {
    if (dims[a] < 1) return fail(LRD_ERR_INVALID, "volume axis %d has size %d", a, dims[a]);
    if (pat[a] < 1 || pat[a] > dims[a])
      return fail(LRD_ERR_INVALID, "patch side %d (axis %d) must be in [1, %d]", pat[a], a, dims[a]);
  }
  if (pr->nt < 2) return fail(LRD_ERR_INVALID, "need at least 2 frames, got %d", pr->nt);
  if (pr->nt > lrd::kMaxT) return fail(LRD_ERR_UNSUPPORTED, "nt=%d exceeds the compiled limit %d", pr->nt, lrd::kMaxT);
  if (pr->stride < 1) return fail(LRD_ERR_INVALID, "stride must be >= 1, got %d", pr->stride);
  if (pr->form != LRD_FORM_PLAIN && pr->form != LRD_FORM_ACCURATE && pr->form != LRD_FORM_TENSOR &&
      pr->form != LRD_FORM_TENSOR_BF16)
    return fail(LRD_ERR_INVALID, "unknown form %d", pr->form);
  if (pr->batch < 0) return fail(LRD_ERR_INVALID, "batch must be >= 0, got %d", pr->batch);
  if (pr->recon_split != 0 && pr->recon_split != 1 && pr->recon_split != 2 && pr->recon_split != 4)
    return fail(LRD_ERR_INVALID, "recon_split must be 0, 1, 2 or 4, got %d", pr->recon_split);
  if (pr->gram_split != 0 && pr->gram_split != 1 && pr->gram_split != 2 && pr->gram_split != 4)
    return fail(LRD_ERR_INVALID, "gram_split must be 0, 1, 2 or 4, got %d", pr->gram_split);
  if (pr->eigh_block < 0 || pr->eigh_block > 2)
    return fail(LRD_ERR_INVALID, "eigh_block must be 0 (plan), 1 (warp) or 2 (CTA), got %d", pr->eigh_block);
  if (pr->eigh_block == 1 && pr->nt > 64)
    return fail(LRD_ERR_INVALID, "eigh_block 1 (one warp per matrix) needs T <= 64, got T = %d", pr->nt);
  const long long nvox = (long long)pr->nx * pr->ny * pr->nz;
  if (nvox * pr->nt >= (1LL << 40)) return fail(LRD_ERR_UNSUPPORTED, "volume too large");
  const long long nvp = (long long)pr->px * pr->py * pr->pz;
  if (nvp > (1 << 30)) return fail(LRD_ERR_UNSUPPORTED, "patch too large");
  if (nvp < pr->nt)
    return fail(LRD_ERR_UNSUPPORTED,
                "patch has %lld voxels < %d frames: the Gram route needs N >= T", nvp, pr->nt);
  return LRD_OK;
}

// Reconstruction layout of a problem: threads per voxel, frames per thread
// and the brick - the cost model's choice, or the problem's recon_split and
// brick when set (a brick must fit the reconstruction kernel's threads per
// CTA). Without either, frame counts the warp kernel is built for take it
// (``warp``; brick 2 x 2 x recon_warp_bz(), four lanes per voxel).
// Measured on B200, reconstruction ms, 96x96x48x48 / 11^3 / stride 3:
// brick kernel (3x3x3, 2 threads per voxel) 1.22 -> warp kernel (see DESIGN).
int pick_layout(const lrd_problem* pr, const int dims[3], const int pat[3], const std::vector<int32_t> corners[3],
                int& rsplit, int& rtpt, int best[3], bool* warp = nullptr, bool* tc = nullptr) {
  if (warp) *warp = false;
  if (tc) *tc = false;
  const char* tc_env = getenv("LRD_RECON_TC");  // "0": the tensor forms keep the warp kernel
  // the largest patch box a 4 x 4 x 8 brick touches (per axis: corners whose
  // patch meets the brick's range), which the tensor-core kernel keeps in
  // shared memory
  auto box_side = [&](int a, int bs) {
    long long most = 0;
    for (int lo = 0; lo < dims[a]; lo += bs) {
      const int hi = std::min(dims[a], lo + bs) - 1;
      long long cnt = 0;
      for (int c : corners[a]) cnt += (c <= hi && c + pat[a] - 1 >= lo);
      most = std::max(most, cnt);
    }
    return most;
  };
  if (tc && (pr->form == LRD_FORM_TENSOR || pr->form == LRD_FORM_TENSOR_BF16) && pr->recon_split == 0 &&
      pr->brick_x == 0 && pr->brick_y == 0 && pr->brick_z == 0 && lrd::recon_tc_supported(pr->nt) &&
      !(tc_env && tc_env[0] == '0') &&
      box_side(0, lrd::kRtcBX) * box_side(1, lrd::kRtcBY) * box_side(2, lrd::kRtcBZ) <= lrd::kRtcMaxBoxPatches) {
    *tc = true;
    rsplit = 1;
    rtpt = pr->nt;
    best[0] = lrd::kRtcBX;
    best[1] = lrd::kRtcBY;
    best[2] = lrd::kRtcBZ;
    return LRD_OK;
  }
  if (warp && pr->recon_split == 0 && pr->brick_x == 0 && pr->brick_y == 0 && pr->brick_z == 0 &&
      lrd::recon_warp_supported(pr->nt)) {
    *warp = true;
    rsplit = 4;
    rtpt = pr->nt / 4;
    best[0] = 2;
    best[1] = 2;
    best[2] = lrd::recon_warp_bz();
    return LRD_OK;
  }
  pick_recon_layout(pr->nt, pr->recon_split, pr->form != LRD_FORM_PLAIN, rsplit, rtpt);
  choose_brick(dims, pat, corners, rsplit, best);
  if (pr->brick_x > 0 || pr->brick_y > 0 || pr->brick_z > 0) {
    if (pr->brick_x < 1 || pr->brick_y < 1 || pr->brick_z < 1 ||
        (long long)pr->brick_x * pr->brick_y * pr->brick_z * rsplit > 1024)
      return fail(LRD_ERR_INVALID, "brick %dx%dx%d: each side >= 1 and at most 256 voxels", pr->brick_x,
                  pr->brick_y, pr->brick_z);
    best[0] = pr->brick_x;
    best[1] = pr->brick_y;
    best[2] = pr->brick_z;
    // the CTA must also fit the reconstruction kernel's registers
    cudaFuncAttributes fa{};
    for (bool acc : {false, true}) {
      cudaError_t fe = cudaFuncGetAttributes(&fa, recon_kernel_ptr(rtpt, rsplit, acc));
      if (fe != cudaSuccess) return cuda_fail(fe, "cudaFuncGetAttributes(recon_kernel)");
      if ((long long)pr->brick_x * pr->brick_y * pr->brick_z * rsplit > fa.maxThreadsPerBlock)
        return fail(LRD_ERR_INVALID, "brick %dx%dx%d x %d threads per voxel exceeds the reconstruction kernel's %d "
                    "threads per CTA", pr->brick_x, pr->brick_y, pr->brick_z, rsplit, fa.maxThreadsPerBlock);
    }
  }
  return LRD_OK;
}

// Plan for ``pr``; ``x_corners`` (nullable) replaces the x-axis corner list
// (a slab of a larger volume), which must be sorted, start >= 0 and end
// with a patch inside the volume.
int create_plan(const lrd_problem* pr, const std::vector<int32_t>* x_corners, lrd_plan** out) {
  g_last_error.clear();
  if (!pr || !out) return fail(LRD_ERR_INVALID, "problem or plan pointer is NULL");
  *out = nullptr;
  if (int vrc = validate_problem(pr)) return vrc;
  const int dims[3] = {pr->nx, pr->ny, pr->nz};
  const int pat[3] = {pr->px, pr->py, pr->pz};
  const long long nvox = (long long)pr->nx * pr->ny * pr->nz;
  const long long nvp = (long long)pr->px * pr->py * pr->pz;

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(LRD_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));

  std::vector<int32_t> corners[3], cover[3], brick[3];
  for (int a = 0; a < 3; ++a) {
    corners[a] = (a == 0 && x_corners) ? *x_corners : axis_corners(dims[a], pat[a], pr->stride);
    cover[a].resize(2 * (size_t)dims[a]);
    for (int x = 0; x < dims[a]; ++x) {
      int lo = -1, hi = -2;
      for (int i = 0; i < (int)corners[a].size(); ++i) {
        const int c = corners[a][i];
        if (c <= x && x <= c + pat[a] - 1) {
          if (lo < 0) lo = i;
          hi = i;
        }
      }
      cover[a][2 * x] = lo;
      cover[a][2 * x + 1] = hi;
    }
  }
  // brick shape
  int best[3] = {1, 1, 1};
  int rsplit = 1, rtpt = 4;
  bool warp_recon = false, tc_recon = false;
  if (int lrc = pick_layout(pr, dims, pat, corners, rsplit, rtpt, best, &warp_recon, &tc_recon)) return lrc;
  const int bsz[3] = {best[0], best[1], best[2]};
  for (int a = 0; a < 3; ++a) {
    const int nb = (dims[a] + bsz[a] - 1) / bsz[a];
    brick[a].resize(2 * (size_t)nb);
    for (int b = 0; b < nb; ++b) {
      const int lo = b * bsz[a], hi = std::min(dims[a], lo + bsz[a]) - 1;
      int ilo = -1, ihi = -2;
      for (int i = 0; i < (int)corners[a].size(); ++i) {
        const int c = corners[a][i];
        if (c <= hi && c + pat[a] - 1 >= lo) {
          if (ilo < 0) ilo = i;
          ihi = i;
        }
      }
      brick[a][2 * b] = ilo;
      brick[a][2 * b + 1] = ihi;
    }
  }

  lrd_plan* P = new lrd_plan();
  P->prob = *pr;
  P->device = dev;
  P->nvox = nvox;
  lrd::Geom& g = P->g;
  g.nx = pr->nx; g.ny = pr->ny; g.nz = pr->nz; g.nt = pr->nt;
  g.px = pr->px; g.py = pr->py; g.pz = pr->pz;
  g.ncx = (int)corners[0].size(); g.ncy = (int)corners[1].size(); g.ncz = (int)corners[2].size();
  g.npatch = (long long)g.ncx * g.ncy * g.ncz;
  g.nvox_patch = (int)nvp;
  g.bx = bsz[0]; g.by = bsz[1]; g.bz = bsz[2];
  g.nbx = (int)brick[0].size() / 2; g.nby = (int)brick[1].size() / 2; g.nbz = (int)brick[2].size() / 2;

  // device tables
  size_t total = 0;
  size_t offs[9];
  const std::vector<int32_t>* tabs[9] = {&corners[0], &corners[1], &corners[2], &cover[0], &cover[1],
                                         &cover[2],   &brick[0],   &brick[1],   &brick[2]};
  for (int i = 0; i < 9; ++i) {
    offs[i] = total;
    total += align256(tabs[i]->size() * sizeof(int32_t));
  }
  std::vector<char> host(total, 0);
  for (int i = 0; i < 9; ++i) memcpy(host.data() + offs[i], tabs[i]->data(), tabs[i]->size() * sizeof(int32_t));
  e = cudaMalloc(&P->d_tables, total);
  if (e != cudaSuccess) {
    delete P;
    return fail(LRD_ERR_NOMEM, "cudaMalloc(%zu) for plan tables: %s", total, cudaGetErrorString(e));
  }
  e = cudaMemcpy(P->d_tables, host.data(), total, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(P->d_tables);
    delete P;
    return cuda_fail(e, "cudaMemcpy plan tables");
  }
  char* base = static_cast<char*>(P->d_tables);
  for (int a = 0; a < 3; ++a) {
    P->tab.corners[a] = reinterpret_cast<const int32_t*>(base + offs[a]);
    P->tab.cover[a] = reinterpret_cast<const int32_t*>(base + offs[3 + a]);
    P->tab.brick[a] = reinterpret_cast<const int32_t*>(base + offs[6 + a]);
  }

  const int T = pr->nt;
  P->tpt = rtpt;
  P->split = rsplit;
  P->recon_warp = warp_recon;
  P->recon_tc = tc_recon;
  if (tc_recon) {
    // the largest patch box of a brick (its touching patches, one group per x corner)
    int qx = 1, qy = 1, qz = 1;
    for (size_t b = 0; b + 1 < brick[0].size(); b += 2) qx = std::max(qx, brick[0][b + 1] - brick[0][b] + 1);
    for (size_t b = 0; b + 1 < brick[1].size(); b += 2) qy = std::max(qy, brick[1][b + 1] - brick[1][b] + 1);
    for (size_t b = 0; b + 1 < brick[2].size(); b += 2) qz = std::max(qz, brick[2][b + 1] - brick[2][b] + 1);
    P->smem_recon_tc = lrd::recon_tc_smem_bytes(T, qx * qy * qz, qx);
  }
  const int nb4 = (T + 3) / 4;
  P->gram_threads = nb4 * (nb4 + 1) / 2;
  P->center_warps = 4;
  P->smem_center = sizeof(float) * (size_t)P->center_warps * (32 * (T + 1) + 32);
  P->smem_gram = sizeof(float) * (size_t)pr->py * pr->pz * (4 * nb4);
  P->eigh_cta = eigh_use_cta(T, pr->eigh_block);
  P->smem_eigh = sizeof(float) * eigh_smem_for(T, P->eigh_cta);
  P->smem_recon = lrd::recon_smem_bytes(T, max_touch(brick));
  {
    int ring = 1;
    for (int z = 0; z < pr->nz; ++z) ring = std::max(ring, cover[2][2 * z + 1] - cover[2][2 * z] + 1);
    P->gramz_ring = ring;
    P->gramz_ks = pr->gram_split > 0 ? pr->gram_split : gramz_split(T);
    P->smem_gramz = lrd::gramz_smem_bytes(pr->px * pr->py, T, ring, P->gram_threads);
    P->use_gramz = (T % 4 == 0) && P->smem_gramz <= 200 * 1024 && tensor_map_encoder() != nullptr &&
                   pr->px <= 256 && pr->py <= 256;
    P->gramtc_bf16 = pr->form == LRD_FORM_TENSOR_BF16;
    P->smem_gramtc = lrd::gramtc_smem_bytes(pr->px * pr->py, T, ring, P->gramtc_bf16);
    P->use_gramtc = (pr->form == LRD_FORM_TENSOR || pr->form == LRD_FORM_TENSOR_BF16) && T <= 64 && (T % 4 == 0) && pr->px * pr->py <= 128 &&
                    P->smem_gramtc <= 200 * 1024 && tensor_map_encoder() != nullptr;
  }
  int rc = set_smem((const void*)lrd::center_kernel, P->smem_center);
  if (!rc) rc = set_smem((const void*)lrd::gram_kernel, P->smem_gram);
  if (!rc && P->use_gramz) rc = set_smem(gramz_kernel_ptr(P->gramz_ks), P->smem_gramz);
  if (!rc && P->use_gramtc) rc = set_smem(gramtc_kernel_ptr(P->gramtc_bf16), P->smem_gramtc);
  P->smem_refine = lrd::eigh_refine_smem_bytes(T, pr->pz);
  if (!rc) rc = set_smem((const void*)lrd::eigh_refine_kernel, P->smem_refine);
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    P->refine_blocks = std::max(1, std::min<int>(2 * sms, (int)std::min<long long>(g.npatch, 1 << 20)));
    P->sms = sms;
    int per_sm = 0;
    if (!rc && P->use_gramz) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gramz_kernel_ptr(P->gramz_ks),
                                                        lrd::gramz_threads(T, P->gramz_ks),
                                                        P->smem_gramz) == cudaSuccess)
        P->gramz_slots = per_sm * sms;
      else
        (void)cudaGetLastError();  // no cut columns; the launches report their own errors
    }
    if (!rc && P->use_gramtc) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gramtc_kernel_ptr(P->gramtc_bf16), lrd::kGramTcThreads,
                                                        P->smem_gramtc) == cudaSuccess)
        P->gramtc_slots = per_sm * sms;
      else
        (void)cudaGetLastError();
    }
  }
  if (!rc) rc = set_smem(eigh_kernel_for(T, P->eigh_cta), P->smem_eigh);
  if (!rc && !P->recon_tc) rc = set_smem(recon_kernel_ptr(P->tpt, P->split, false), P->smem_recon);
  if (!rc && !P->recon_tc) rc = set_smem(recon_kernel_ptr(P->tpt, P->split, true), P->smem_recon);
  if (!rc && P->recon_tc) rc = set_smem(recon_tc_ptr(T), P->smem_recon_tc);
  if (rc) {
    cudaFree(P->d_tables);
    delete P;
    return rc;
  }
  if (P->smem_gram > 227 * 1024 || P->smem_eigh > 227 * 1024 || (!P->recon_tc && P->smem_recon > 227 * 1024) ||
      P->smem_refine > 227 * 1024 || P->smem_recon_tc > 227 * 1024) {
    cudaFree(P->d_tables);
    delete P;
    return fail(LRD_ERR_UNSUPPORTED, "patch plane or T too large for shared memory");
  }

  // host-buffer pipeline: x-axis tables, copy streams, slab events
  P->h_corner_x = corners[0];
  P->h_brick_x = brick[0];
  {
    cudaError_t e1 = cudaStreamCreateWithFlags(&P->io_in, cudaStreamNonBlocking);
    cudaError_t e2 = cudaStreamCreateWithFlags(&P->io_out, cudaStreamNonBlocking);
    for (cudaStream_t* ps : {&P->io_prep[0], &P->io_prep[1], &P->io_prep[2], &P->io_solve, &P->io_solve2}) {
      cudaError_t e4 = cudaStreamCreateWithFlags(ps, cudaStreamNonBlocking);
      if (e4 != cudaSuccess) {
        *ps = nullptr;
        if (e1 == cudaSuccess) e1 = e4;
      }
    }
    // the reconstruction streams at the highest priority: a slab's bricks are
    // reconstructed (and copied out) as soon as its solve ends, ahead of the
    // next slabs' Grams (e2e 3.51 -> 3.50 ms at the headline; the solves at the
    // highest priority instead measured slower)
    int prio_lo = 0, prio_hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess) prio_hi = 0;
    for (cudaStream_t* ps : {&P->io_recon, &P->io_recon2}) {
      cudaError_t e4 = cudaStreamCreateWithPriority(ps, cudaStreamNonBlocking, prio_hi);
      if (e4 != cudaSuccess) {
        *ps = nullptr;
        if (e1 == cudaSuccess) e1 = e4;
      }
    }
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
      lrd_plan_destroy(P);
      return cuda_fail(e1 != cudaSuccess ? e1 : e2, "cudaStreamCreateWithFlags");
    }
    P->io_events.resize(5 * kIoSlabs + 1);
    for (auto& ev : P->io_events) {
      cudaError_t e3 = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e3 != cudaSuccess) {
        ev = nullptr;
        lrd_plan_destroy(P);
        return cuda_fail(e3, "cudaEventCreateWithFlags");
      }
    }
  }

  // device-resident pipeline: off by default (LRD_DEVICE_SLABS = S > 1 turns it
  // on). Measured on B200, device ms per denoise at 96x96x48x48 / 11^3 /
  // stride 3, plain, S = 1 / 2 / 3 / 4 / 6 / 8 / 12: 2.86 / 2.94 / 2.94 / 2.93 /
  // 2.95 / 3.19 / 3.42 (accurate 3.13 -> 3.21 .. 3.57): a slab's eigensolve
  // takes one matrix's latency (~0.2 ms) however few matrices it has, and
  // the eigensolver's CTAs leave little room on the SMs for the neighbouring
  // slabs' Gram and reconstruction, so the phases do not overlap enough to
  // pay for the extra launches.
  {
    long long sl = 1;
    if (const char* env = getenv("LRD_DEVICE_SLABS")) sl = std::max(1, atoi(env));
    P->dev_slabs = (int)std::min<long long>({sl, (long long)g.ncx, (long long)kIoSlabs});
  }

  // workspace layout
  size_t off = 0;
  P->off_mean = off; off += align256(sizeof(float) * (size_t)nvox);
  P->off_xc = off; off += align256(sizeof(float) * (size_t)nvox * T);
  P->off_gv = off; off += align256(sizeof(float) * (size_t)g.npatch * T * T);
  P->off_rank = off; off += align256(sizeof(int32_t) * (size_t)g.npatch);
  P->off_wgt = off; off += align256(sizeof(float) * (size_t)g.npatch);
  P->off_sig2 = off; off += align256(sizeof(float) * (size_t)g.npatch);
  P->off_status = off; off += align256(sizeof(int32_t));
  P->off_refine = off; off += align256(sizeof(int32_t) * (64 + (size_t)g.npatch));
  P->ws_bytes = off;
  *out = P;
  return LRD_OK;
}

// Cut of the x-corner list into n contiguous slabs: per slab {first corner,
// end corner, first plane read, end plane read}. Slab r owns output planes
// [x0(r), x0(r + 1)); the planes [x0(r + 1), x1(r)) are touched by both.
int slab_partition(const lrd_problem* pr, int n, std::vector<int32_t>& b) {
  if (!pr) return fail(LRD_ERR_INVALID, "problem is NULL");
  if (pr->nx < 1 || pr->px < 1 || pr->px > pr->nx || pr->stride < 1)
    return fail(LRD_ERR_INVALID, "bad x axis (nx %d, px %d, stride %d)", pr->nx, pr->px, pr->stride);
  const std::vector<int32_t> cx = axis_corners(pr->nx, pr->px, pr->stride);
  const int nc = (int)cx.size();
  if (n < 1 || n > nc) return fail(LRD_ERR_INVALID, "n_slabs=%d must be in [1, %d] (x-corners)", n, nc);
  b.assign(4 * (size_t)n, 0);
  for (int r = 0; r < n; ++r) {
    b[4 * r] = (int32_t)((long long)r * nc / n);
    b[4 * r + 1] = (int32_t)((long long)(r + 1) * nc / n);
    b[4 * r + 2] = r == 0 ? 0 : cx[b[4 * r]];
  }
  for (int r = 0; r < n; ++r)
    b[4 * r + 3] = r == n - 1 ? pr->nx : std::max(cx[b[4 * r + 1] - 1] + pr->px, b[4 * (r + 1) + 2]);
  for (int r = 0; r + 2 < n; ++r)
    if (b[4 * r + 3] > b[4 * (r + 2) + 2])
      return fail(LRD_ERR_UNSUPPORTED,
                  "%d slabs: planes [%d, %d) would be touched by three slabs; use fewer slabs", n,
                  b[4 * (r + 2) + 2], b[4 * r + 3]);
  return LRD_OK;
}

}  // namespace

extern "C" {

int lrd_version(void) { return LRD_VERSION; }

const char* lrd_last_error_string(void) { return g_last_error.c_str(); }

int lrd_plan_create(const lrd_problem* pr, lrd_plan** out) { return create_plan(pr, nullptr, out); }

int lrd_plan_set_profiling(lrd_plan* P, int enable) {
  if (!P) return fail(LRD_ERR_INVALID, "plan is NULL");
  if (enable && P->prof_events.empty()) {
    P->prof_events.resize((size_t)kProfRing * (LRD_NUM_PHASES + 1));
    for (auto& e : P->prof_events) LRD_CUDA(cudaEventCreate(&e));
  }
  P->profiling = enable != 0;
  P->prof_calls = 0;
  return LRD_OK;
}

int lrd_plan_phase_ms(lrd_plan* P, float* ms, int32_t* n_calls) {
  if (!P || !ms) return fail(LRD_ERR_INVALID, "NULL argument");
  for (int k = 0; k < LRD_NUM_PHASES; ++k) ms[k] = 0.f;
  const int n = P->prof_calls;
  if (n > 0) {
    const cudaEvent_t* ev = P->prof_events.data();
    LRD_CUDA(cudaEventSynchronize(ev[(size_t)(n - 1) * (LRD_NUM_PHASES + 1) + LRD_NUM_PHASES]));
    for (int c = 0; c < n; ++c)
      for (int k = 0; k < LRD_NUM_PHASES; ++k) {
        float t = 0.f;
        LRD_CUDA(cudaEventElapsedTime(&t, ev[(size_t)c * (LRD_NUM_PHASES + 1) + k],
                                      ev[(size_t)c * (LRD_NUM_PHASES + 1) + k + 1]));
        ms[k] += t;
      }
  }
  if (n_calls) *n_calls = n;
  P->prof_calls = 0;
  return LRD_OK;
}

int lrd_plan_destroy(lrd_plan* P) {
  if (!P) return LRD_OK;
  for (auto& e : P->prof_events) cudaEventDestroy(e);
  for (auto& e : P->io_events)
    if (e) cudaEventDestroy(e);
  if (P->io_in) cudaStreamDestroy(P->io_in);
  if (P->io_out) cudaStreamDestroy(P->io_out);
  for (auto ps : P->io_prep)
    if (ps) cudaStreamDestroy(ps);
  if (P->io_recon) cudaStreamDestroy(P->io_recon);
  if (P->io_recon2) cudaStreamDestroy(P->io_recon2);
  if (P->io_solve) cudaStreamDestroy(P->io_solve);
  if (P->io_solve2) cudaStreamDestroy(P->io_solve2);
  if (P->d_tables) cudaFree(P->d_tables);
  delete P;
  return LRD_OK;
}

int lrd_plan_num_patches(const lrd_plan* P, int64_t* n) {
  if (!P || !n) return fail(LRD_ERR_INVALID, "NULL argument");
  *n = P->g.npatch;
  return LRD_OK;
}

int lrd_workspace_size(const lrd_plan* P, size_t* bytes) {
  if (!P || !bytes) return fail(LRD_ERR_INVALID, "NULL argument");
  *bytes = P->ws_bytes;
  return LRD_OK;
}

// lrd_denoise over x-slabs of patch corners whose phases overlap: slab s is
// centred and its columns' Grams formed on a plan stream (io_prep[s % 3], after
// the previous slab's centring, whose planes its columns share), its patches
// solved and refined on ``st`` once its Grams are in, and the bricks whose
// touching patches are then all final reconstructed on io_recon - so one
// slab's latency-bound eigensolve shares the SMs with the next slab's Gram
// and the previous slab's reconstruction. Every patch and voxel computes
// exactly what the one-pass call computes (same kernels, same order per
// voxel). All side streams join ``st`` again.
int run_pipelined(const lrd_plan* P, const float* d_vol, float* d_out, char* ws, cudaStream_t st) {
  const lrd::Geom& g = P->g;
  const long long plane_vox = (long long)g.ny * g.nz;
  float* gv = reinterpret_cast<float*>(ws + P->off_gv);
  int32_t* rank = reinterpret_cast<int32_t*>(ws + P->off_rank);
  float* wgt = reinterpret_cast<float*>(ws + P->off_wgt);
  // k: 1 centred, 2 Gram, 3 reconstructed, 4 solved
  auto ev = [&](int s, int k) { return P->io_events[5 * s + k]; };
  cudaEvent_t start = P->io_events[5 * kIoSlabs];
  int rc;
  LRD_CUDA(cudaMemsetAsync(ws + P->off_status, 0, sizeof(int32_t), st));
  LRD_CUDA(cudaMemsetAsync(ws + P->off_refine, 0, 64 * sizeof(int32_t), st));  // every slab's queue
  LRD_CUDA(cudaEventRecord(start, st));
  for (auto ps : P->io_prep) LRD_CUDA(cudaStreamWaitEvent(ps, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_recon, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_solve, start, 0));
  const int S = P->dev_slabs;
  int planes_in = 0, ci_done = 0, bx_done = 0;
  const long long colz = (long long)g.ncy, patz = (long long)g.ncy * g.ncz, brz = (long long)g.nby * g.nbz;
  for (int s = 0; s < S; ++s) {
    const int ci_end = (int)((long long)(s + 1) * g.ncx / S);
    const bool lastslab = s == S - 1;
    const int x_need = lastslab ? g.nx : std::min(g.nx, P->h_corner_x[ci_end - 1] + g.px);
    cudaStream_t prep = P->io_prep[s % 3];
    if (s > 0) LRD_CUDA(cudaStreamWaitEvent(prep, ev(s - 1, 1), 0));
    if (x_need > planes_in &&
        (rc = run_center(P, d_vol, ws, prep, planes_in * plane_vox, (long long)(x_need - planes_in) * plane_vox)))
      return rc;
    LRD_CUDA(cudaEventRecord(ev(s, 1), prep));
    planes_in = std::max(planes_in, x_need);
    if ((rc = run_gram(P, ws, gv, prep, ci_done * colz, ci_end * colz))) return rc;
    LRD_CUDA(cudaEventRecord(ev(s, 2), prep));
    // successive slabs' solves on two streams: one slab's solve takes a matrix's
    // latency however few matrices it has, so two run side by side
    cudaStream_t solve = (s & 1) ? P->io_solve : st;
    LRD_CUDA(cudaStreamWaitEvent(solve, ev(s, 2), 0));
    if ((rc = run_eigh(P, ws, gv, gv, nullptr, rank, wgt, solve, ci_done * patz, ci_end * patz, false, d_vol, s)))
      return rc;
    ci_done = ci_end;
    int bx_end = bx_done;
    while (bx_end < g.nbx && (lastslab || P->h_brick_x[2 * bx_end + 1] < ci_end)) ++bx_end;
    LRD_CUDA(cudaEventRecord(ev(s, 4), solve));
    LRD_CUDA(cudaStreamWaitEvent(P->io_recon, ev(s, 4), 0));
    if ((rc = run_recon(P, ws, d_out, P->io_recon, bx_done * brz, bx_end * brz))) return rc;
    LRD_CUDA(cudaEventRecord(ev(s, 3), P->io_recon));
    bx_done = bx_end;
  }
  // the side streams join the caller's stream: the last reconstruction follows
  // every solve (each reconstruction waited for its slab's) and every Gram
  LRD_CUDA(cudaStreamWaitEvent(st, ev(S - 1, 3), 0));
  for (int s = 0; s < S && s < 3; ++s) LRD_CUDA(cudaStreamWaitEvent(st, ev(S - 1 - s, 2), 0));
  return LRD_OK;
}

int lrd_denoise(const lrd_plan* P, const float* d_vol, float* d_out, int32_t* d_ranks, void* d_ws,
                void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!d_vol || !d_out || !d_ws) return fail(LRD_ERR_INVALID, "NULL device buffer");
  if (reinterpret_cast<uintptr_t>(d_ws) % 256) return fail(LRD_ERR_INVALID, "workspace not 256-byte aligned");
  const size_t vbytes = sizeof(float) * (size_t)P->nvox * P->g.nt;
  const char* a = reinterpret_cast<const char*>(d_vol);
  const char* b = reinterpret_cast<const char*>(d_out);
  if (a < b + vbytes && b < a + vbytes) return fail(LRD_ERR_INVALID, "d_vol and d_out overlap");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_ws);
  float* gv = reinterpret_cast<float*>(ws + P->off_gv);
  int32_t* rank = reinterpret_cast<int32_t*>(ws + P->off_rank);
  float* wgt = reinterpret_cast<float*>(ws + P->off_wgt);
  cudaEvent_t* ev = nullptr;
  if (P->profiling && P->prof_calls < kProfRing) {
    ev = const_cast<cudaEvent_t*>(P->prof_events.data()) + (size_t)P->prof_calls * (LRD_NUM_PHASES + 1);
    ++const_cast<lrd_plan*>(P)->prof_calls;
  }
  if (!ev && P->dev_slabs > 1 && !P->is_slab) {
    std::lock_guard<std::mutex> lk(P->pipe_mu);
    if ((rc = run_pipelined(P, d_vol, d_out, ws, st))) return rc;
    if (d_ranks) LRD_CUDA(cudaMemcpyAsync(d_ranks, rank, sizeof(int32_t) * P->g.npatch, cudaMemcpyDeviceToDevice, st));
    return LRD_OK;
  }
  if (ev) LRD_CUDA(cudaEventRecord(ev[0], st));
  LRD_CUDA(cudaMemsetAsync(ws + P->off_status, 0, sizeof(int32_t), st));
  if ((rc = run_center(P, d_vol, ws, st))) return rc;
  if (ev) LRD_CUDA(cudaEventRecord(ev[1], st));
  if ((rc = run_gram(P, ws, gv, st))) return rc;
  if (ev) LRD_CUDA(cudaEventRecord(ev[2], st));
  if ((rc = run_eigh(P, ws, gv, gv, nullptr, rank, wgt, st, 0, -1, true, d_vol))) return rc;
  if (ev) LRD_CUDA(cudaEventRecord(ev[3], st));
  if ((rc = run_recon(P, ws, d_out, st))) return rc;
  if (ev) LRD_CUDA(cudaEventRecord(ev[4], st));
  if (d_ranks) LRD_CUDA(cudaMemcpyAsync(d_ranks, rank, sizeof(int32_t) * P->g.npatch, cudaMemcpyDeviceToDevice, st));
  return LRD_OK;
}

// End corner index of host-pipeline slab s of S over nc x-corners: the first
// and the last slab get one corner each (the first copy-in and the last
// copy-out are the pipeline's exposed ends), the others an equal share.
static int slab_end(int s, int S, int nc) {
  if (s == S - 1) return nc;
  if (S < 4 || nc < S) return (int)((long long)(s + 1) * nc / S);
  if (s == 0) return 1;
  return 1 + (int)((long long)s * (nc - 2) / (S - 2));
}

int lrd_denoise_host(const lrd_plan* P, const float* h_vol, float* h_out, int32_t* h_ranks, float* d_in,
                     float* d_out, int32_t* d_ranks, void* d_ws, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!h_vol || !h_out || !d_in || !d_out || !d_ws) return fail(LRD_ERR_INVALID, "NULL buffer");
  if (h_ranks && !d_ranks) return fail(LRD_ERR_INVALID, "h_ranks needs d_ranks");
  if (reinterpret_cast<uintptr_t>(d_ws) % 256) return fail(LRD_ERR_INVALID, "workspace not 256-byte aligned");
  // Pipeline over x-slabs of patch corners. Slab s: copy in the x-planes its
  // patch columns need (copy-in stream); centre them and form those columns'
  // Gram matrices on io_prep[s % 3] (a slab's Gram launch is a fraction of a
  // wave, so three slabs' Grams run side by side); solve the slab's patches
  // and refine their near-ties on one of three solve streams (the caller's
  // ``stream``, io_solve, io_solve2: s % 3); reconstruct the bricks whose
  // touching patches are now all final on one of two reconstruction streams
  // (alternating, so one slab's reconstruction fills the tail of the
  // previous one's, and both overlap the next slabs' solves); copy those
  // bricks' output planes back (copy-out stream). Events order: copy-in(s)
  // -> centre(s) (after centre(s - 1), whose planes the slab's columns
  // share) -> Gram(s) -> solve(s) -> reconstruct(s) (also after solve(s - 1))
  // -> copy-out(s).
  std::lock_guard<std::mutex> lk(P->pipe_mu);  // the plan's streams and events
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_ws);
  const lrd::Geom& g = P->g;
  const long long plane = (long long)g.ny * g.nz * g.nt;  // floats per x-plane
  const long long plane_vox = (long long)g.ny * g.nz;
  float* gv = reinterpret_cast<float*>(ws + P->off_gv);
  int32_t* rank = reinterpret_cast<int32_t*>(ws + P->off_rank);
  float* wgt = reinterpret_cast<float*>(ws + P->off_wgt);
  // k: 0 copied in, 1 centred, 2 Gram, 3 reconstructed, 4 solved
  auto ev = [&](int s, int k) { return P->io_events[5 * s + k]; };
  cudaEvent_t start = P->io_events[5 * kIoSlabs];
  LRD_CUDA(cudaMemsetAsync(ws + P->off_status, 0, sizeof(int32_t), st));
  LRD_CUDA(cudaMemsetAsync(ws + P->off_refine, 0, 64 * sizeof(int32_t), st));  // every slab's queue
  LRD_CUDA(cudaEventRecord(start, st));
  LRD_CUDA(cudaStreamWaitEvent(P->io_in, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_out, start, 0));
  for (auto ps : P->io_prep) LRD_CUDA(cudaStreamWaitEvent(ps, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_recon, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_recon2, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_solve, start, 0));
  LRD_CUDA(cudaStreamWaitEvent(P->io_solve2, start, 0));
  // about kIoSlabBytes of input per slab, at most kIoSlabsUsed slabs: a small
  // volume's slabs would be launch- and event-bound
  const long long vbytes = (long long)sizeof(float) * P->nvox * g.nt;
  const int S = std::max(1, std::min<int>({kIoSlabsUsed, g.ncx, (int)((vbytes + kIoSlabBytes - 1) / kIoSlabBytes)}));
  int planes_in = 0, ci_done = 0, bx_done = 0;
  const long long colz = (long long)g.ncy, patz = (long long)g.ncy * g.ncz, brz = (long long)g.nby * g.nbz;
  for (int s = 0; s < S; ++s) {
    const int ci_end = slab_end(s, S, g.ncx);
    const bool lastslab = s == S - 1;
    const int x_need = lastslab ? g.nx : std::min(g.nx, P->h_corner_x[ci_end - 1] + g.px);
    cudaStream_t prep = P->io_prep[s % 3];
    if (x_need > planes_in)
      LRD_CUDA(cudaMemcpyAsync(d_in + planes_in * plane, h_vol + planes_in * plane,
                               sizeof(float) * (size_t)(x_need - planes_in) * plane, cudaMemcpyHostToDevice,
                               P->io_in));
    LRD_CUDA(cudaEventRecord(ev(s, 0), P->io_in));
    LRD_CUDA(cudaStreamWaitEvent(prep, ev(s, 0), 0));
    if (s > 0) LRD_CUDA(cudaStreamWaitEvent(prep, ev(s - 1, 1), 0));
    if ((rc = run_center(P, d_in, ws, prep, planes_in * plane_vox, (long long)(x_need - planes_in) * plane_vox)))
      return rc;
    LRD_CUDA(cudaEventRecord(ev(s, 1), prep));
    planes_in = std::max(planes_in, x_need);
    if ((rc = run_gram(P, ws, gv, prep, ci_done * colz, ci_end * colz, s == 0))) return rc;
    LRD_CUDA(cudaEventRecord(ev(s, 2), prep));
    // successive slabs' solves on three streams, each slab with its own
    // near-tie queue: a slab's solve takes a matrix's latency however few it
    // holds, so up to three run side by side
    cudaStream_t solve = (s % 3 == 0) ? st : (s % 3 == 1 ? P->io_solve : P->io_solve2);
    LRD_CUDA(cudaStreamWaitEvent(solve, ev(s, 2), 0));
    if ((rc = run_eigh(P, ws, gv, gv, nullptr, rank, wgt, solve, ci_done * patz, ci_end * patz, false, d_in, s)))
      return rc;
    ci_done = ci_end;
    int bx_end = bx_done;
    while (bx_end < g.nbx && (lastslab || P->h_brick_x[2 * bx_end + 1] < ci_end)) ++bx_end;
    LRD_CUDA(cudaEventRecord(ev(s, 4), solve));
    // slab s's bricks touch patches of slab s, s - 1 and possibly earlier
    // slabs (a brick's patches span four corners): s and s - 1 are waited for
    // here, the earlier ones through the previous reconstruction on the same
    // stream (slab s - 2's, which waited for s - 2 and s - 3)
    cudaStream_t recon = (s & 1) ? P->io_recon2 : P->io_recon;
    LRD_CUDA(cudaStreamWaitEvent(recon, ev(s, 4), 0));
    if (s > 0) LRD_CUDA(cudaStreamWaitEvent(recon, ev(s - 1, 4), 0));
    if ((rc = run_recon(P, ws, d_out, recon, bx_done * brz, bx_end * brz))) return rc;
    LRD_CUDA(cudaEventRecord(ev(s, 3), recon));
    if (bx_end > bx_done) {
      const long long x0 = (long long)bx_done * g.bx, x1 = std::min<long long>((long long)bx_end * g.bx, g.nx);
      LRD_CUDA(cudaStreamWaitEvent(P->io_out, ev(s, 3), 0));
      LRD_CUDA(cudaMemcpyAsync(h_out + x0 * plane, d_out + x0 * plane, sizeof(float) * (size_t)(x1 - x0) * plane,
                               cudaMemcpyDeviceToHost, P->io_out));
    }
    bx_done = bx_end;
  }
  // the last two reconstructions join the caller's stream (each followed
  // every solve before it)
  LRD_CUDA(cudaStreamWaitEvent(st, ev(S - 1, 3), 0));
  if (S >= 2) LRD_CUDA(cudaStreamWaitEvent(st, ev(S - 2, 3), 0));
  if (d_ranks) LRD_CUDA(cudaMemcpyAsync(d_ranks, rank, sizeof(int32_t) * g.npatch, cudaMemcpyDeviceToDevice, st));
  if (h_ranks) {
    LRD_CUDA(cudaEventRecord(ev(S - 1, 4), st));
    LRD_CUDA(cudaStreamWaitEvent(P->io_out, ev(S - 1, 4), 0));
    LRD_CUDA(cudaMemcpyAsync(h_ranks, d_ranks, sizeof(int32_t) * g.npatch, cudaMemcpyDeviceToHost, P->io_out));
  }
  LRD_CUDA(cudaStreamSynchronize(P->io_out));
  LRD_CUDA(cudaStreamSynchronize(st));
  int32_t status = 0;
  if ((rc = lrd_workspace_status(P, d_ws, &status, stream))) return rc;
  if (status) return fail(LRD_ERR_TIMEOUT, "a device wait gave up (status 0x%x): the result is invalid", status);
  return LRD_OK;
}

int lrd_slab_partition(const lrd_problem* pr, int32_t n, int32_t* bounds) {
  g_last_error.clear();
  if (!bounds) return fail(LRD_ERR_INVALID, "bounds is NULL");
  std::vector<int32_t> b;
  int rc = slab_partition(pr, n, b);
  if (rc) return rc;
  memcpy(bounds, b.data(), b.size() * sizeof(int32_t));
  return LRD_OK;
}

int lrd_slab_plan_create(const lrd_problem* pr, int32_t n, int32_t slab, lrd_plan** out) {
  g_last_error.clear();
  if (!out) return fail(LRD_ERR_INVALID, "plan pointer is NULL");
  *out = nullptr;
  std::vector<int32_t> b;
  int rc = slab_partition(pr, n, b);
  if (rc) return rc;
  if (slab < 0 || slab >= n) return fail(LRD_ERR_INVALID, "slab %d not in [0, %d)", slab, n);
  const int ci_lo = b[4 * slab], ci_hi = b[4 * slab + 1], x0 = b[4 * slab + 2], x1 = b[4 * slab + 3];
  const std::vector<int32_t> cx = axis_corners(pr->nx, pr->px, pr->stride);
  std::vector<int32_t> local(cx.begin() + ci_lo, cx.begin() + ci_hi);
  for (auto& c : local) c -= x0;
  lrd_problem lp = *pr;
  lp.nx = x1 - x0;
  lrd_plan* P = nullptr;
  if ((rc = create_plan(&lp, &local, &P))) return rc;
  P->is_slab = true;
  P->slab = slab;
  P->n_slabs = n;
  P->slab_x0 = x0;
  P->slab_ci_lo = ci_lo;
  P->slab_ci_hi = ci_hi;
  P->slab_hin = slab == 0 ? 0 : b[4 * (slab - 1) + 3] - x0;
  P->slab_own_hi = slab == n - 1 ? lp.nx : b[4 * (slab + 1) + 2] - x0;
  *out = P;
  return LRD_OK;
}

int lrd_slab_info(const lrd_plan* P, int32_t* info) {
  if (!P || !info) return fail(LRD_ERR_INVALID, "NULL argument");
  if (!P->is_slab) return fail(LRD_ERR_INVALID, "not a slab plan");
  const int32_t v[8] = {P->slab_x0, P->g.nx, P->slab_hin, P->slab_own_hi,
                        P->slab_ci_lo, P->slab_ci_hi, P->slab, P->n_slabs};
  memcpy(info, v, sizeof(v));
  return LRD_OK;
}

int lrd_slab_prepare(const lrd_plan* P, const float* d_vol, int32_t* d_ranks, void* d_ws, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!P->is_slab) return fail(LRD_ERR_INVALID, "not a slab plan");
  if (!d_vol || !d_ws) return fail(LRD_ERR_INVALID, "NULL device buffer");
  if (reinterpret_cast<uintptr_t>(d_ws) % 256) return fail(LRD_ERR_INVALID, "workspace not 256-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_ws);
  float* gv = reinterpret_cast<float*>(ws + P->off_gv);
  int32_t* rank = reinterpret_cast<int32_t*>(ws + P->off_rank);
  float* wgt = reinterpret_cast<float*>(ws + P->off_wgt);
  LRD_CUDA(cudaMemsetAsync(ws + P->off_status, 0, sizeof(int32_t), st));
  if ((rc = run_center(P, d_vol, ws, st))) return rc;
  if ((rc = run_gram(P, ws, gv, st))) return rc;
  if ((rc = run_eigh(P, ws, gv, gv, nullptr, rank, wgt, st, 0, -1, true, d_vol))) return rc;
  if (d_ranks) LRD_CUDA(cudaMemcpyAsync(d_ranks, rank, sizeof(int32_t) * P->g.npatch, cudaMemcpyDeviceToDevice, st));
  return LRD_OK;
}

int lrd_slab_recon(const lrd_plan* P, float* d_out, void* d_ws, int32_t part, const double* d_halo_in,
                   double* d_halo_out, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!P->is_slab) return fail(LRD_ERR_INVALID, "not a slab plan");
  if (!d_ws) return fail(LRD_ERR_INVALID, "NULL workspace");
  lrd::SlabIO io{0, 0, P->slab_hin, nullptr, P->slab_own_hi, nullptr};
  if (part == LRD_SLAB_HALO_OUT) {
    io.x_lo = P->slab_own_hi;
    io.x_hi = P->g.nx;
    io.halo_out = d_halo_out;
    if (io.x_lo < io.x_hi && !d_halo_out) return fail(LRD_ERR_INVALID, "d_halo_out is NULL");
  } else if (part == LRD_SLAB_INTERIOR) {
    io.x_lo = P->slab_hin;
    io.x_hi = P->slab_own_hi;
  } else if (part == LRD_SLAB_HALO_IN) {
    io.x_lo = 0;
    io.x_hi = P->slab_hin;
    io.halo_in = d_halo_in;
    if (io.x_lo < io.x_hi && !d_halo_in) return fail(LRD_ERR_INVALID, "d_halo_in is NULL");
  } else {
    return fail(LRD_ERR_INVALID, "unknown slab part %d", part);
  }
  if (io.x_lo >= io.x_hi) return LRD_OK;
  if (part != LRD_SLAB_HALO_OUT && !d_out) return fail(LRD_ERR_INVALID, "d_out is NULL");
  const long long brz = (long long)P->g.nby * P->g.nbz;
  const long long b_lo = (long long)(io.x_lo / P->g.bx) * brz;
  const long long b_hi = (long long)((io.x_hi + P->g.bx - 1) / P->g.bx) * brz;
  return run_recon(P, static_cast<char*>(d_ws), d_out, static_cast<cudaStream_t>(stream), b_lo, b_hi, &io);
}

int lrd_noise_map(const lrd_plan* P, const void* d_ws, float* d_sigma2, float* d_noise, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!d_ws) return fail(LRD_ERR_INVALID, "NULL workspace");
  if (d_noise && P->is_slab)
    return fail(LRD_ERR_UNSUPPORTED, "the voxel noise map of a slab needs its neighbours' patches; "
                "take the per-patch estimates (d_sigma2) instead");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const char* ws = static_cast<const char*>(d_ws);
  const float* sig2 = reinterpret_cast<const float*>(ws + P->off_sig2);
  const float* wgt = reinterpret_cast<const float*>(ws + P->off_wgt);
  if (d_sigma2)
    LRD_CUDA(cudaMemcpyAsync(d_sigma2, sig2, sizeof(float) * P->g.npatch, cudaMemcpyDeviceToDevice, st));
  if (d_noise) {
    const unsigned blocks = (unsigned)((P->nvox + 255) / 256);
    lrd::noise_map_kernel<<<blocks, 256, 0, st>>>(sig2, wgt, d_noise, P->g, P->tab);
    return launch_check("noise_map_kernel launch");
  }
  return LRD_OK;
}

int lrd_workspace_status(const lrd_plan* P, const void* d_ws, int32_t* status, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!d_ws || !status) return fail(LRD_ERR_INVALID, "NULL argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  LRD_CUDA(cudaMemcpyAsync(status, static_cast<const char*>(d_ws) + P->off_status, sizeof(int32_t),
                           cudaMemcpyDeviceToHost, st));
  LRD_CUDA(cudaStreamSynchronize(st));
  return LRD_OK;
}

int lrd_selftest_wait_timeout(int64_t limit_ns, int32_t* d_status, void* stream) {
  g_last_error.clear();
  if (!d_status) return fail(LRD_ERR_INVALID, "d_status is NULL");
  if (limit_ns < 1000 || limit_ns > 10000000000ll)
    return fail(LRD_ERR_INVALID, "limit_ns=%lld not in [1e3, 1e10]", (long long)limit_ns);
  lrd::wait_timeout_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      d_status, (unsigned long long)limit_ns, lrd::kStatusTmaTimeout);
  return launch_check("wait_timeout_selftest_kernel launch");
}

int lrd_stage_gram(const lrd_plan* P, const float* d_vol, float* d_gram, void* d_ws, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!d_vol || !d_gram || !d_ws) return fail(LRD_ERR_INVALID, "NULL device buffer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_ws);
  LRD_CUDA(cudaMemsetAsync(ws + P->off_status, 0, sizeof(int32_t), st));
  if ((rc = run_center(P, d_vol, ws, st))) return rc;
  return run_gram(P, ws, d_gram, st);
}

int lrd_stage_eigh(const lrd_plan* P, const float* d_gram, float* d_lam, float* d_vecs, int32_t* d_ranks,
                   void* d_ws, void* stream) {
  int rc = check_plan(P);
  if (rc) return rc;
  if (!d_gram || !d_vecs || !d_ranks || !d_ws) return fail(LRD_ERR_INVALID, "NULL device buffer");
  if (d_gram == d_vecs) return fail(LRD_ERR_INVALID, "d_gram and d_vecs must differ");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_ws);
  float* wgt = reinterpret_cast<float*>(ws + P->off_wgt);
  return run_eigh(P, ws, d_gram, d_vecs, d_lam, d_ranks, wgt, st);
}

}  // extern "C"

#include "lrd_static.inc"
#include "lrd_batch.inc"
