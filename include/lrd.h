/*
 * lrd.h - C ABI of the B200 patch-wise MP-PCA denoiser (U-free Gram route).
 *
 * The ladder's drop-in call is the Python function ``denoise(vol_np) ->
 * np.ndarray`` (step8_tuned.py:116-146, called by common.run, common.py:103,
 * 130, 138) with patch shape, stride and batch taken from module globals
 * (common.py:28-29, step8_tuned.py:21). This header is the native boundary
 * under that call: plain pointers and sizes, device buffers owned by the
 * caller, work enqueued on the caller's CUDA stream (passed as ``void*``), no
 * host synchronisation inside ``lrd_denoise``.
 *
 * Conventions
 *   - every function returns an int status: LRD_OK (0) or a negative LRD_ERR_*;
 *     lrd_last_error_string() gives a message for the calling thread's last
 *     failure;
 *   - a volume is float32, C order (x, y, z, t), t contiguous;
 *   - a plan's problem, tables and launch shapes do not change after creation,
 *     and lrd_denoise, the stage entry points and lrd_noise_map may be called
 *     on one plan from several threads at once (each call on its own
 *     workspace) while its profiling is off. Two parts of a plan are mutable:
 *     with profiling on (lrd_plan_set_profiling) every lrd_denoise records
 *     into the plan's event ring, so profiled calls must come from one thread;
 *     lrd_denoise_host drives the plan's own copy and compute streams and
 *     events, so it runs one call at a time per plan. One stream must not run
 *     two calls on the same workspace at once.
 */
#ifndef LRD_H
#define LRD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LRD_VERSION 1

enum lrd_status {
  LRD_OK = 0,
  LRD_ERR_INVALID = -1,     /* bad argument, shape or null pointer          */
  LRD_ERR_NOMEM = -2,       /* device allocation for the plan's tables failed */
  LRD_ERR_CUDA = -3,        /* a CUDA call or launch failed                  */
  LRD_ERR_UNSUPPORTED = -4, /* shape outside the compiled kernels' limits    */
  LRD_ERR_NODEVICE = -5,    /* no CUDA device / driver                       */
  LRD_ERR_TIMEOUT = -6      /* a bounded device-side wait gave up            */
};

/* Bits of the device status word (lrd_workspace_status). */
#define LRD_STATUS_TMA_TIMEOUT 1 /* a TMA completion wait exceeded its deadline */
#define LRD_STATUS_MMA_TIMEOUT 2 /* a tensor-core completion wait exceeded its deadline */

/* Arithmetic forms of the path. */
enum lrd_form {
  /* FP32 throughout; the weighted overlap accumulation runs per voxel in the
   * ladder's patch order (x-major corners) with float32 rounding at every
   * step, as step0_numpy_loop.py:36-39 does - deterministic. */
  LRD_FORM_PLAIN = 0,
  /* Same contractions; the accumulation keeps the temporal mean out of the
   * running sums (out = m + sum w (x-m)P / sum w, float64 weight sums): error
   * against a float64 run of the algorithm at the float32 output floor. */
  LRD_FORM_ACCURATE = 1,
  /* Precision form: both contractions on the tcgen05 tensor cores in TF32
   * with 3xTF32 split products (x = hi + lo; hi.hi + hi.lo + lo.hi). The
   * Gram accumulates in tensor memory per plane (T <= 64, px*py <= 128;
   * otherwise the FP32 Gram); the reconstruction (T % 4 == 0, T <= 64) is two
   * chained GEMMs per 4 x 4 x 8 voxel brick with one accumulator per 8
   * columns, the mean kept out of the sums as in the accurate form.
   * Near-tie MP decisions are redone in FP64. The tensor-core Gram's
   * eigenvalues are about 1e-6 of the largest one from float64 (FP32 FFMA:
   * about 1e-8), so a patch that close to an MP tie may take a different
   * count than step 0. */
  LRD_FORM_TENSOR = 2,
  /* Precision form with BF16 Gram operands: as LRD_FORM_TENSOR, the Gram on
   * tcgen05 in kind::f16 with each float32 value split into three BF16 terms
   * (x = b0 + b1 + b2) and the six products of combined order <= 2 summed in
   * FP32 in tensor memory per plane. */
  LRD_FORM_TENSOR_BF16 = 3
};

/* One problem: volume (nx, ny, nz, nt), patch (px, py, pz), one stride for the
 * three spatial axes (common.py:28-29, 37-44), the form, ``batch`` = patches
 * per Gram/eigensolver launch (step8_tuned.py:21; 0 = all in one launch), and
 * the reconstruction brick (voxels per CTA along x, y, z) and threads per
 * voxel (recon_split: 1, 2 or 4); 0 = chosen by the plan's cost model (the
 * autotuner fills them in). These change speed only: every voxel's arithmetic
 * and accumulation order are the same for any brick and split.
 * ``gram_split``: threads sharing a 4x4 block of the column Gram (1, 2 or 4,
 * each summing every n-th voxel row); ``eigh_block``: 1 = one warp per
 * matrix (T <= 64), 2 = one CTA of 64 / 96 / 128 threads per matrix; 0 = the
 * plan's choice for both. These two change the float32 rounding of the Gram
 * and the eigenvalues (ranks stay the same: near-ties are decided in FP64
 * from the input). */
typedef struct lrd_problem {
  int32_t nx, ny, nz, nt;
  int32_t px, py, pz;
  int32_t stride;
  int32_t form;
  int32_t batch;
  int32_t brick_x, brick_y, brick_z;
  int32_t recon_split;
  int32_t gram_split;
  int32_t eigh_block;
} lrd_problem;

typedef struct lrd_plan lrd_plan;

/* Validate the problem, build the patch-index tables (common.py:37-44) on the
 * current device, pick launch shapes. Replaces the per-call host work of
 * step8_tuned.py:121-126 (allocation + patch_bases). */
int lrd_plan_create(const lrd_problem* problem, lrd_plan** plan);
int lrd_plan_destroy(lrd_plan* plan);

/* Number of patches (common.py:37-44 product of the per-axis corner lists). */
int lrd_plan_num_patches(const lrd_plan* plan, int64_t* n_patches);

/* Bytes of device workspace ``lrd_denoise`` needs (temporal means, centred
 * volume, per-patch Gram/eigenvector blocks, ranks, weights). Replaces the
 * per-batch ``gram`` allocation of step8_tuned.py:130. */
int lrd_workspace_size(const lrd_plan* plan, size_t* bytes);

/* Denoise one volume, all on ``stream`` (a cudaStream_t; NULL = legacy
 * default stream). ``d_vol`` and ``d_out`` are device arrays of
 * nx*ny*nz*nt float32 and must not overlap; ``d_ranks`` (nullable) receives
 * the MP rank chosen for every patch (int32, x-major patch order);
 * ``d_workspace`` has ``lrd_workspace_size`` bytes, 256-byte aligned.
 * Replaces step8_tuned.py:116-146 minus its host<->device copies: gather +
 * Gram (gram_kernel, step8:32-56), eigh + MP rank + projector + weight
 * (step8:134-137, mp_keep step8:96-113), reconstruction + weighted overlap
 * add (recon_scatter_kernel, step8:59-86) and the normalisation (step8:145). */
int lrd_denoise(const lrd_plan* plan, const float* d_vol, float* d_out, int32_t* d_ranks,
                void* d_workspace, void* stream);

/* Host-buffer form of lrd_denoise: copies ``h_vol`` (pinned or pageable host
 * memory) to ``d_in``, denoises into ``d_out``, copies the result to
 * ``h_out`` and waits. ``d_in``/``d_out`` are caller-owned device buffers of
 * the volume's size. This is the whole host->host call of step8_tuned.py:
 * 116-146 (from_numpy().cuda() ... host.copy_(...)), pipelined: the volume
 * moves in x-slabs on the plan's copy streams, each slab's centring and Gram
 * run on the plan's side streams as soon as its planes are in, its solve on
 * ``stream``, its reconstruction on another plan stream, and finished output
 * planes copy out while later slabs compute (pinned host buffers make the
 * copies asynchronous). Results are identical to lrd_denoise's. The plan's
 * streams and events make this one call at a time per plan. */
int lrd_denoise_host(const lrd_plan* plan, const float* h_vol, float* h_out, int32_t* h_ranks,
                     float* d_in, float* d_out, int32_t* d_ranks, void* d_workspace,
                     void* stream);

/* Device status word of the last call that used ``d_workspace`` on
 * ``stream``: 0, or LRD_STATUS_* bits set by kernels whose bounded waits gave
 * up (the output of that call is then invalid). Synchronises ``stream``.
 * lrd_denoise_host checks it itself and returns LRD_ERR_TIMEOUT. No
 * counterpart in the reference (its kernels have no device-side waits). */
int lrd_workspace_status(const lrd_plan* plan, const void* d_workspace, int32_t* status, void* stream);

/* Self-test of the failure path above, without a GPU fault: a one-thread
 * kernel waits on a device barrier that nothing completes, gives up after
 * ``limit_ns`` nanoseconds (1 us .. 10 s) and or-s LRD_STATUS_TMA_TIMEOUT into
 * the int32 at ``d_status`` (device memory), on ``stream``; the context stays
 * usable. The kernels' own waits use the same routine with a 2 s limit. No
 * counterpart in the reference. */
int lrd_selftest_wait_timeout(int64_t limit_ns, int32_t* d_status, void* stream);

/* Stage entry points, for per-stage parity checks against step 4's unfused
 * route (step4_gram_eigh.py:60-67).
 *   lrd_stage_gram: G = Xc^T Xc for every patch -> d_gram (n_patches, nt, nt).
 *   lrd_stage_eigh: from d_gram, ascending eigenvalues -> d_lam (n_patches, nt)
 *     (nullable), the top-p eigenvectors in descending eigenvalue order as the
 *     rows of a compact p x nt block at the start of each patch's nt*nt slot
 *     of d_vecs, MP ranks -> d_ranks. d_gram is left unchanged. */
int lrd_stage_gram(const lrd_plan* plan, const float* d_vol, float* d_gram, void* d_workspace,
                   void* stream);
int lrd_stage_eigh(const lrd_plan* plan, const float* d_gram, float* d_lam, float* d_vecs,
                   int32_t* d_ranks, void* d_workspace, void* stream);

/* Measurement hook (no counterpart in the reference): with profiling on,
 * every lrd_denoise call records CUDA events between its phases on its
 * stream; lrd_plan_phase_ms waits for the last recorded call and returns, per
 * phase, the summed milliseconds and the number of calls recorded since the
 * previous read (then clears them). Phases: 0 centring, 1 Gram, 2 eigensolver
 * + MP rank, 3 reconstruction + accumulation. Profiling state is per plan and
 * not thread-safe. */
#define LRD_NUM_PHASES 4
int lrd_plan_set_profiling(lrd_plan* plan, int enable);
int lrd_plan_phase_ms(lrd_plan* plan, float* ms /* LRD_NUM_PHASES */, int32_t* n_calls);

/* Denoise with no device allocation at all. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc (code running where the CUDA
 * allocator is off limits, or a host framework that owns every device
 * allocation): lrd_denoise needs a plan (whose index tables are
 * cudaMalloc'd) and a caller-allocated workspace; this entry point needs
 * neither. The caller passes only the problem, the input and output volumes
 * and the optional rank array, all as for lrd_denoise. Every scratch buffer
 * (patch-index tables, temporal means, centred volume, Gram/eigenvector
 * blocks, ranks, weights) lives in one file-scope static device array of
 * LRD_STATIC_SCRATCH_BYTES, which every GPU that loads the library holds
 * until the process exits. Problems needing more scratch than that (about
 * 21 MiB for a 48x48x24x48 volume with 11^3 patches at stride 3; the
 * 96x96x48x48 headline needs about 203 MiB) are rejected with
 * LRD_ERR_UNSUPPORTED and a message giving the size needed.
 *
 * The problem's fields mean what they mean for lrd_plan_create (brick and
 * recon_split included); d_vol and d_out must not overlap. Every form runs
 * its Gram on the per-patch FP32 kernel here (the tensor form's tcgen05 Gram
 * and the column Gram are not used), so the tensor form gives the accurate
 * form's result; the patch-index tables are written into the array by a
 * kernel on ``stream``.
 *
 * The first call on a device looks up the array's device address (with that
 * device current) and caches it; make that first call before any stream
 * capture. All calls share the one array and it keeps the last call's
 * contents (nothing in it needs to start at zero): calls whose work overlaps
 * on the GPU - on different streams, or from different threads - race on it
 * and must be serialised by the caller. */
#define LRD_STATIC_SCRATCH_BYTES (32u << 20)
int lrd_denoise_static(const lrd_problem* problem, const float* d_vol, float* d_out, int32_t* d_ranks,
                       void* stream);

/* Batched form: many volumes of different shapes (frame counts, patch sizes,
 * strides) in one call. Replaces a Python loop of the ladder's ``denoise``
 * over volumes (step8_tuned.py:116-146 per volume).
 *
 * lrd_batch_plan_create builds one plan per problem (the problems' brick and
 * split fields may carry autotuned values) and groups the volumes' kernels
 * into packed launches: per phase, one grid covers every volume of a kernel
 * class (centring: all volumes; column Gram: per frame count; eigensolver:
 * per solver class T <= 32 / 48 / 64 / 96 / 128; near-tie pass: all;
 * reconstruction: per frame count and form), each block finding its volume
 * in a device table of per-volume descriptors. Volumes whose Gram or
 * reconstruction runs on another kernel (T % 4 != 0, the tcgen05 Gram of the
 * tensor form, an explicit brick) get per-volume launches in that phase.
 * Every volume's result is bit-identical to lrd_denoise's. ``n_streams`` is
 * accepted for compatibility and unused: the launches run in order on
 * ``stream``.
 *
 * lrd_batch_denoise runs the batch; d_vols, d_outs and d_ranks are host
 * arrays of n device pointers (d_ranks and its entries may be NULL); the
 * workspace is one allocation of lrd_batch_workspace_size bytes. Without
 * ``use_graph`` the call copies the descriptor table from pinned staging
 * memory (stream-ordered) and launches; with ``use_graph`` the launches are
 * captured once into a CUDA graph with its own device table and later calls
 * with the same pointers replay it as a single graph launch (different
 * pointers re-capture). No host synchronisation on the replay path. One call
 * at a time per batch plan. lrd_batch_num_launches gives the kernel launches
 * of one call (17 for the 24 mixed-shape volumes of the batched benchmark,
 * against 6 per volume one by one). */
typedef struct lrd_batch_plan lrd_batch_plan;
int lrd_batch_plan_create(const lrd_problem* problems, int32_t n, int32_t n_streams, lrd_batch_plan** plan);
int lrd_batch_plan_destroy(lrd_batch_plan* plan);
int lrd_batch_workspace_size(const lrd_batch_plan* plan, size_t* bytes);
int lrd_batch_num_launches(const lrd_batch_plan* plan, int32_t* launches);
int lrd_batch_denoise(lrd_batch_plan* plan, const float* const* d_vols, float* const* d_outs,
                      int32_t* const* d_ranks, void* d_workspace, void* stream, int32_t use_graph);

/* Slab sharding: one volume over several GPUs (one process per GPU), cut by
 * x-corner. Replaces, for a volume too large or too slow for one GPU, the
 * ladder's single ``denoise`` call (step0_numpy_loop.py:28-39; corners from
 * common.py:40-43).
 *
 * The x-corner list is cut into n_slabs contiguous runs of about equal
 * length. Slab r reads global x-planes [x0, x1): from its first corner to the
 * last plane its patches touch (the last slab to the volume's end), and owns
 * the output planes [x0, x0 of slab r+1). Its top planes [x0 of slab r+1, x1)
 * are also touched by slab r+1's patches: slab r hands its unnormalised sums
 * (sum of w * xd per frame, then sum of w, float64) for those planes to slab
 * r+1, which continues them with its own patches. A voxel's patches are
 * therefore added in the single-GPU (x-major) order and every slab's owned
 * planes equal the single-GPU output bit for bit. No voxel may be touched by
 * three slabs (LRD_ERR_UNSUPPORTED otherwise: use fewer slabs).
 *
 * lrd_slab_partition fills bounds[4*r .. 4*r+3] = {first corner index, end
 * corner index, x0, x1} for each slab r. lrd_slab_plan_create makes the plan
 * of slab ``slab`` (its local volume is planes [x0, x1) of the global one;
 * workspace and buffers sized by the plan as for lrd_plan_create).
 * lrd_slab_info gives info[0..7] = {x0, local planes nx, halo-in planes hin,
 * owned planes own_hi, first corner, end corner, slab, n_slabs}; the halo a
 * slab receives is hin x ny x nz x (nt + 1) doubles, the one it sends
 * (nx - own_hi) x ny x nz x (nt + 1).
 *
 * lrd_slab_prepare runs centring, Gram, eigensolve and MP rank for the slab's
 * patches (ranks -> d_ranks, nullable). lrd_slab_recon then reconstructs one
 * part of the local planes: LRD_SLAB_HALO_OUT (planes [own_hi, nx), sums ->
 * d_halo_out), LRD_SLAB_INTERIOR (planes [hin, own_hi) -> d_out) or
 * LRD_SLAB_HALO_IN (planes [0, hin), continuing from d_halo_in -> d_out).
 * d_out has the local volume's shape; only the owned planes are written. The
 * halo pointers are ignored by the parts that do not use them. */
#define LRD_SLAB_HALO_OUT 0
#define LRD_SLAB_INTERIOR 1
#define LRD_SLAB_HALO_IN 2
int lrd_slab_partition(const lrd_problem* problem, int32_t n_slabs, int32_t* bounds);
int lrd_slab_plan_create(const lrd_problem* problem, int32_t n_slabs, int32_t slab, lrd_plan** plan);
int lrd_slab_info(const lrd_plan* plan, int32_t* info);
int lrd_slab_prepare(const lrd_plan* plan, const float* d_vol, int32_t* d_ranks, void* d_workspace,
                     void* stream);
int lrd_slab_recon(const lrd_plan* plan, float* d_out, void* d_workspace, int32_t part,
                   const double* d_halo_in, double* d_halo_out, void* stream);

/* Per-patch outputs of the last lrd_denoise / lrd_denoise_host /
 * lrd_slab_prepare on ``d_workspace`` (the ladder returns only the volume,
 * step0_numpy_loop.py:28-39; the ranks come out of every denoise call):
 * d_sigma2 (n_patches floats, nullable) receives each patch's MP noise
 * variance estimate, the mean of its t - p noise eigenvalues
 * (eigs = lambda / N as in step0_numpy_loop.py:18, t = nt - 1, p the MP
 * rank; 0 when p = t); d_noise (nx*ny*nz floats, nullable) receives the
 * voxel noise map, the patches' estimates averaged with the denoiser's
 * weights w = 1/(2+p) in its patch order (0 where no patch covers). Slab
 * plans give d_sigma2 only. Enqueued on ``stream``. */
int lrd_noise_map(const lrd_plan* plan, const void* d_workspace, float* d_sigma2, float* d_noise, void* stream);

/* Message of the calling thread's last failure ("" if none). */
const char* lrd_last_error_string(void);
int lrd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LRD_H */
