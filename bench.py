"""Benchmark of the MP-PCA denoiser hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form plain|accurate] [--workload headline|config1]

A step is one denoise of one synthetic volume already resident in HBM: the
headline workload is 96x96x48x48 (x, y, z, t) with 11^3 patches at stride 3
(12600 patches of 1331 x 48), rank-4 signal in [0, 1] plus N(0, 0.05^2) noise.
``value`` is whole-job patches/s from CUDA events around each step (L2 flushed
by a 256 MiB write between steps, outside the events); ``e2e`` is the same
metric through the C ABI's host-buffer call (pinned host in/out, both copies
inside the timed region). Under torchrun (N GPUs) the workload's volume is
repeated N times along x and cut into N x-slabs of patch corners, one per
rank, with one NCCL halo send/recv between neighbours per step (weak scaling:
about the single-GPU work per rank); ``--parallel replica`` gives every rank
an independent volume instead. The step time is the max over ranks.

The headline line also states the accuracy of the timed output (relative L2
against the reference's step 0 in float32 and float64 on a seeded sample of
the volume, ranks against both), the ``accurate`` form's times and errors
(the form at the float64 bar), the reference's own step-8 GPU path timed on
the same GPU in the same run, and ``torch.linalg.eigh`` on the same Gram
blocks beside the library's eigensolver phase.

``--impl reference`` times the reference algorithm's CPU implementation (the
reference's own step-0 NumPy loop from ``baseline/_ref`` when it is
installed there, else its restatement in oracle/; all host cores through a
spawn pool) on a bounded sample of the same workload's patches.

``python bench.py --install-reference <checkout>`` installs the reference
into ``baseline/_ref`` (its pip package, which holds only ``micro/``, plus
the ladder's top-level modules, unmodified).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "headline": dict(shape=(96, 96, 48, 48), patch=(11, 11, 11), stride=3,
                     desc="96x96x48x48 volume, 11^3 patches, stride 3 (12600 patches of 1331x48)"),
    "config1": dict(shape=(48, 48, 24, 48), patch=(11, 11, 11), stride=3,
                    desc="48x48x24x48 volume, 11^3 patches, stride 3 (1176 patches of 1331x48)"),
}
PUBLISHED_STEP8_MS = 66.5  # reference step 8, host->host best of 5, 12600 patches (README.md:48)
REF_DIR = os.path.join(ROOT, "baseline", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")
# golden fixture holding the reference's step-0 output (float32 and float64 runs) on the
# workload's benchmark phantom with seed 0 and on the ladder's own phantom
GOLDEN_FOR = {"headline": ("headline_lowrank.npz", "headline_ref.npz"),
              "config1": ("config1_lowrank.npz", "config1_ref.npz")}


def bench_config(wl, world=1):
    """The ``config`` object both arms print (same keys and values)."""
    return dict(workload=wl["desc"], shape=list(wl["shape"]), patch=list(wl["patch"]), stride=wl["stride"],
                phantom="rank-4 [0,1] + N(0,0.05^2), seed 0",
                l2="flushed by a 256 MiB write between timed GPU steps (outside the events)",
                parallelism=f"replica x{world}" if world > 1 else "single GPU")


def golden_accuracy(out, ranks, fixture):
    """Errors of a volume ``out`` (numpy, the workload's shape) and per-patch
    ``ranks`` against a golden fixture of the reference's step 0: relative L2
    on the fixture's seeded 20000-element sample against the float32 step-0
    output and the float64 run of the same code, and rank mismatches against
    both runs' ranks."""
    import numpy as _np

    d = _np.load(os.path.join(GOLDEN, fixture))
    idx = d["sample_idx"]
    o = _np.asarray(out, dtype=_np.float64).reshape(-1)[idx]
    ref32 = d["out_sample"].astype(_np.float64)
    ref64 = d["out64_sample"]
    res = dict(rel_err_vs_fp64=float(_np.linalg.norm(o - ref64) / _np.linalg.norm(ref64)),
               rel_err_vs_step0=float(_np.linalg.norm(o - ref32) / _np.linalg.norm(ref32)),
               step0_vs_fp64=float(_np.linalg.norm(ref32 - ref64) / _np.linalg.norm(ref64)),
               sample=f"{len(idx)}-element seeded sample of the output ({fixture})")
    if ranks is not None:
        r = _np.asarray(ranks).astype(_np.int32)
        res.update(rank_mismatch_vs_step0=int((r != d["ranks"]).sum()),
                   rank_mismatch_vs_fp64=int((r != d["ranks64"]).sum()), n_patches=int(len(r)))
    return res


def install_reference(src):
    """Install the reference into ``baseline/_ref``: ``pip install --target``
    of the reference's package from a copy of the checkout (the package holds
    only ``micro/``: its pyproject builds no modules), then the ladder's
    top-level modules (``common.py``, ``stepN_*.py``) copied unmodified beside
    it, so the ladder's own entry points (and ``micro/``'s ``from common
    import ...``) import from there."""
    import shutil

    src = os.path.abspath(src)
    tmp = tempfile.mkdtemp(prefix="lrd_refsrc_")
    copy = os.path.join(tmp, "ref")
    shutil.copytree(src, copy, ignore=shutil.ignore_patterns(".git", "results", "__pycache__"))
    os.makedirs(REF_DIR, exist_ok=True)
    cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation", "--no-deps",
           "--find-links", "/opt/wheelhouse", "--target", REF_DIR, "--upgrade", copy]
    rc = subprocess.run(cmd).returncode
    for f in sorted(os.listdir(src)):
        if f.endswith(".py"):
            shutil.copy(os.path.join(src, f), REF_DIR)
    shutil.rmtree(tmp, ignore_errors=True)
    print(json.dumps(dict(pip_rc=rc, target=REF_DIR,
                          modules=sorted(f for f in os.listdir(REF_DIR) if f.endswith(".py")))))


def reference_step0():
    """The reference's own ``step0_numpy_loop`` module from ``baseline/_ref``
    (None when it is not installed there)."""
    if not os.path.exists(os.path.join(REF_DIR, "step0_numpy_loop.py")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import step0_numpy_loop

    return step0_numpy_loop


def phase_kernel(phase, T, form):
    """Kernel that a plan phase launches for T frames (the eigensolve phase
    also runs the refine kernel and its cursor, both under 0.5% of it)."""
    if phase == "gram":
        return "gram_tc_kernel" if (form in ("tensor", "tensor_bf16") and T <= 64) else "gram_z_kernel"
    if phase == "eigh_mp":
        return "eigh_reg_kernel" if T <= 64 else "eigh_cta_kernel"
    if phase == "recon" and form in ("tensor", "tensor_bf16") and T % 4 == 0 and 8 <= T <= 64:
        return "recon_tc_kernel"  # tcgen05, 4x4x8 voxel bricks
    if phase == "recon" and T in (32, 48, 64, 96):
        return "recon_warp_kernel"  # one warp per 2x2x2 voxel block (the plan's default layout)
    if phase == "recon" and form == "plain" and 45 <= T <= 48:
        return "recon_kernel_t24s2"  # 24 frames x 2 threads, built with 112 registers
    return {"center": "center_kernel", "recon": "recon_kernel"}[phase]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["plain", "accurate", "tensor", "tensor_bf16"], default="plain")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched", "serving"], default="headline")
    ap.add_argument("--volumes", type=int, default=24, help="batched: number of volumes")
    ap.add_argument("--requests", type=int, default=48, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=40.0, help="serving: Poisson arrival rate (req/s)")
    ap.add_argument("--duration", type=float, default=0.0,
                    help="serving: arrivals for this many seconds instead of --requests (config: 60)")
    ap.add_argument("--serving-requests", type=int, default=12,
                    help="headline line: requests of the bounded serving sample (0 = none)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-step8", action="store_true", help="skip the reference's step-8 GPU timing")
    ap.add_argument("--step8-repeats", type=int, default=3, help="step 8: timed host->host calls (best of)")
    ap.add_argument("--single-form", action="store_true",
                    help="time only --form (no accurate/plain companion, no ladder-phantom lines)")
    ap.add_argument("--install-reference", metavar="CHECKOUT", default=None,
                    help="install the reference checkout into baseline/_ref and exit")
    ap.add_argument("--cpu-sample", type=int, default=0, help="patches in the CPU sample (0 = auto)")
    ap.add_argument("--brick", default=None, help="recon brick bx,by,bz (default: the plan's choice)")
    ap.add_argument("--split", type=int, default=0, help="recon threads per voxel (0 = the plan's choice)")
    ap.add_argument("--parallel", choices=["shard", "replica"], default="shard",
                    help="N>1: one (96N)-plane volume cut in N x-slabs with a halo exchange (shard), "
                         "or one volume per GPU (replica)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ----------------------------------------------------------------------------- CPU side
def cpu_step0_rate(vol, patch, stride, n_patches_sample, processes):
    """Patches/s of the step-0 loop over a sample of the corner list, spread
    over ``processes`` spawn workers with one BLAS thread each. The per-patch
    routine is the reference's own ``step0_numpy_loop.mppca_patch``
    (step0_numpy_loop.py:8-25) when ``baseline/_ref`` has it, else its
    restatement in oracle/; returns (rate, seconds, workers, kind).

    Each worker receives the volume once (pool initializer) and runs the
    step-0 per-patch work - gather, centre, SVD, MP rank, reconstruct, weighted
    accumulate into its own ``out``/``wsum`` (step0_numpy_loop.py:32-38) - over
    its share of the sample; the wall time of that loop across the pool is the
    measurement.
    """
    import multiprocessing as mp

    from lowrank_gpu_fastest_b200.problem import patch_corners

    corners = patch_corners(vol.shape, patch, stride)
    sample = corners[np.linspace(0, len(corners) - 1, n_patches_sample).astype(int)]
    chunks = [c for c in np.array_split(sample, processes) if len(c)]
    for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    use_ref = os.path.exists(os.path.join(REF_DIR, "step0_numpy_loop.py"))
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(chunks), initializer=_cpu_init, initargs=(vol, patch, use_ref)) as pool:
        pool.map(_cpu_worker, [c[:1] for c in chunks])  # warm (imports, first SVD)
        t0 = time.perf_counter()
        pool.map(_cpu_worker, chunks)
        dt = time.perf_counter() - t0
    return len(sample) / dt, dt, len(chunks), ("reference" if use_ref else "port")


_CPU = {}


def _cpu_init(vol, patch, use_ref):
    _CPU["vol"] = vol
    _CPU["patch"] = patch
    _CPU["out"] = np.zeros_like(vol)
    _CPU["wsum"] = np.zeros(vol.shape[:3] + (1,), dtype=vol.dtype)
    if use_ref:
        _CPU["mppca_patch"] = reference_step0().mppca_patch
    else:
        from oracle import mppca as orc

        _CPU["mppca_patch"] = orc.mppca_patch


def _cpu_worker(corners):
    vol, (px, py, pz) = _CPU["vol"], _CPU["patch"]
    out, wsum, mppca_patch = _CPU["out"], _CPU["wsum"], _CPU["mppca_patch"]
    for i, j, k in corners:
        sl = np.s_[i:i + px, j:j + py, k:k + pz]
        xd, p = mppca_patch(vol[sl].reshape(-1, vol.shape[-1]))
        w = 1.0 / (2.0 + p)
        out[sl] += w * xd.reshape(px, py, pz, -1)
        wsum[sl] += w
    return len(corners)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, wl):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    vol, _ = make_phantom_lowrank(wl["shape"], seed=0)
    cores = host_cores()
    per_step = args.cpu_sample or max(64, 256 * cores)  # ~1 s of all cores per step
    for _ in range(args.warmup):
        cpu_step0_rate(vol, wl["patch"], wl["stride"], min(per_step, cores * 4), cores)
    rates = []
    for _ in range(args.steps):
        r, _, used, kind = cpu_step0_rate(vol, wl["patch"], wl["stride"], per_step, cores)
        rates.append(r)
    from lowrank_gpu_fastest_b200.problem import n_patches

    P = n_patches(wl["shape"], wl["patch"], wl["stride"])
    value = float(statistics.mean(rates))
    who = ("the reference's own step0_numpy_loop.mppca_patch from baseline/_ref" if kind == "reference"
           else "the step-0 loop restated in oracle/ (baseline/_ref not installed)")
    line = dict(
        impl="reference", metric="patches_per_s", value=value, unit="patches/s", n_gpus=args.gpus,
        steps=args.steps, warmup=args.warmup, ms_per_step=1e3 * per_step / value,
        ms_per_volume=1e3 * P / value, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f32", data="synthetic",
        config=bench_config(wl, args.gpus),
        cpu_baseline=dict(value=value, unit="patches/s", cores=used, kind=kind,
                          sample=f"{per_step} patches per step, evenly spaced over the {P}-patch corner "
                                 f"list; {who} (SVD + MP rank) with the loop's weighted accumulate, one "
                                 f"BLAS thread per spawn worker"),
        e2e=dict(value=value, unit="patches/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
    )
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU side
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return dict(sm_mhz=statistics.median(sms) if sms else None, sm_max_mhz=mx,
                    reasons=sorted(reasons), samples=len(sms),
                    power_w_max=max(power) if power else None)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return dict(hbm_gbs=d["hbm_gbs"], bf16_tflops=d["bf16_tflops"],
                    bf16_tflops_sustained=d.get("bf16_tflops_sustained"), source="of measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, bf16_tflops_sustained=1400.0, source="of fallback")


def fp32_simt_peak_tflops(torch, tf32=False):
    """FP32 CUDA-core GEMM throughput (cuBLAS SGEMM, TF32 off) as the FFMA
    reference point for the float32 kernels; with ``tf32`` the same GEMM on
    the tensor cores in TF32 (the reference point of the tensor form's Gram)."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = bool(tf32)
    try:
        n = 8192
        a = torch.randn(n, n, device="cuda")
        b = torch.randn(n, n, device="cuda")
        c = torch.empty(n, n, device="cuda")
        for _ in range(2):
            torch.matmul(a, b, out=c)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b, out=c)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b, c
        return 2 * n**3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def ncu_traffic():
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def time_form(torch, dist, args, wl, form, vol, rank, world, local, *, clocks=False, golden=None):
    """Time one form on one resident volume: ``args.steps`` device-timed
    denoises (CUDA events per step on the launching stream, L2 flushed
    between steps outside the events; max over ranks), the library's phase
    events, then the same number of host->host calls through
    ``lrd_denoise_host`` (pinned host in/out, both copies inside the timed
    region; max over ranks). With ``golden`` (a fixture name) the output and
    ranks of the last timed step are checked against it."""
    from lowrank_gpu_fastest_b200 import api

    shape, patch, stride = wl["shape"], wl["patch"], wl["stride"]
    dev = torch.device("cuda", local)
    d_vol = torch.from_numpy(vol).to(dev)
    d_out = torch.empty_like(d_vol)
    brick = tuple(int(v) for v in args.brick.split(",")) if args.brick else None
    plan = api.get_plan(shape, patch, stride, form=form, device=local, brick=brick, split=args.split)
    ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device=dev)
    d_ranks = torch.empty(plan.n_patches, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sid = stream.cuda_stream
    P = plan.n_patches

    def step():
        plan.denoise(d_vol.data_ptr(), d_out.data_ptr(), d_ranks.data_ptr(), ws.data_ptr(), sid)

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    sampler = None
    if clocks:
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for s, e in evs:
        flush.zero_()
        s.record(stream)
        step()
        e.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    wall = time.perf_counter() - t_wall
    clk = sampler.stop() if sampler else None
    status = plan.status(ws.data_ptr(), sid)
    # phase times from separate profiled calls (a profiled call runs its phases one after
    # another; the timed calls above overlap the phases of successive x-slabs)
    plan.set_profiling(True)
    for _ in range(min(args.steps, 5)):
        flush.zero_()
        step()
    phases, ncalls = plan.phase_ms()
    plan.set_profiling(False)
    torch.cuda.synchronize()
    t = torch.tensor([sum(s.elapsed_time(e) for s, e in evs)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps
    out_np = d_out.cpu().numpy()
    ranks_np = d_ranks.cpu().numpy()

    # e2e: host buffers through the C ABI (pinned in/out), copies inside the timed region
    h_in = torch.from_numpy(vol).pin_memory()
    h_out = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    h_ranks = torch.empty(P, dtype=torch.int32, pin_memory=True)
    d_in = torch.empty_like(d_vol)

    def e2e_step():
        plan.denoise_host(h_in.data_ptr(), h_out.data_ptr(), h_ranks.data_ptr(), d_in.data_ptr(),
                          d_out.data_ptr(), d_ranks.data_ptr(), ws.data_ptr(), sid)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if world > 1:
        dist.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()  # returns after the D2H copies completed
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    t = torch.tensor([statistics.mean(e2e_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms_step = float(t.item())
    e2e_same = bool(np.array_equal(h_out.numpy(), out_np) and np.array_equal(h_ranks.numpy(), ranks_np))
    res = dict(form=form, P=P, ms_per_step=ms_per_step, value=world * P / (ms_per_step * 1e-3),
               phases_sum_ms=None,
               e2e_ms=e2e_ms_step, e2e_value=world * P / (e2e_ms_step * 1e-3), wall=wall, clocks=clk,
               phases={k: v / max(ncalls, 1) for k, v in phases.items()}, status=status,
               e2e_output_identical=e2e_same, out=out_np, ranks=ranks_np, plan=plan)
    res["phases_sum_ms"] = sum(res["phases"].values())
    if golden is not None:
        res["accuracy"] = golden_accuracy(out_np, ranks_np, golden)
    del d_vol, d_out, ws, flush, d_in, h_in, h_out
    return res


def library_eigh(torch, wl, vol, local, batch=2048):
    """``torch.linalg.eigh`` (the eigensolver of the reference's step 8,
    step8_tuned.py:134) on the same Gram blocks the library's eigensolver
    phase solves: Grams from ``lrd_stage_gram`` on the resident volume, solved
    in batches of ``batch`` (step 8's BATCH) and timed with CUDA events, beside
    ``lrd_stage_eigh`` (eigenvalues, MP ranks, top-p eigenvectors) on the
    same blocks. The backend is named from the kernels the profiler lists for
    one batched call."""
    from lowrank_gpu_fastest_b200 import api

    shape, patch, stride = wl["shape"], wl["patch"], wl["stride"]
    T = shape[3]
    dev = torch.device("cuda", local)
    plan = api.get_plan(shape, patch, stride, form="plain", device=local)
    P = plan.n_patches
    d_vol = torch.from_numpy(vol).to(dev)
    ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device=dev)
    g = torch.empty((P, T, T), dtype=torch.float32, device=dev)
    sid = torch.cuda.current_stream(dev).cuda_stream
    plan.stage_gram(d_vol.data_ptr(), g.data_ptr(), ws.data_ptr(), sid)
    lam = torch.empty((P, T), dtype=torch.float32, device=dev)
    vecs = torch.empty_like(g)
    rk = torch.empty(P, dtype=torch.int32, device=dev)

    def ours():
        plan.stage_eigh(g.data_ptr(), lam.data_ptr(), vecs.data_ptr(), rk.data_ptr(), ws.data_ptr(), sid)

    def lib():
        for b0 in range(0, P, batch):
            torch.linalg.eigh(g[b0:b0 + batch])

    def timed(fn, reps):
        best = 1e30
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        return best

    torch.linalg.eigh(g[:batch])  # warm (handles, workspaces)
    ours()
    torch.cuda.synchronize()
    res = dict(matrices=P, T=T, batch=batch, ours_ms=timed(ours, 5))
    res["torch_linalg_eigh_ms"] = timed(lib, 2)
    res["speedup"] = res["torch_linalg_eigh_ms"] / res["ours_ms"]
    try:
        from torch.profiler import ProfilerActivity, profile

        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            torch.linalg.eigh(g[:256])
            torch.cuda.synchronize()
        ks = []
        for ev in prof.key_averages():
            tt = getattr(ev, "device_time_total", None)
            if tt is None:
                tt = getattr(ev, "cuda_time_total", 0)
            if tt and tt > 0:
                ks.append((tt, ev.key))
        ks.sort(reverse=True)
        names = [k for _, k in ks[:5]]
        low = " ".join(names).lower()
        backend = ("cuSOLVER syevj (Jacobi), batched" if "syevj" in low else
                   "cuSOLVER syevd" if ("syevd" in low or "stedc" in low or "sytrd" in low) else
                   "cuSOLVER (kernel names: see eigh_kernels)")
        res.update(backend=backend, eigh_kernels=names)
    except Exception as exc:  # the profiler is optional: the timing above stands without it
        res.update(backend=f"unnamed ({type(exc).__name__}: {exc})")
    res["torch"] = torch.__version__
    del g, vecs, ws, d_vol
    return res


def reference_step8(torch, wl, vols, repeats=3, budget_s=60.0):
    """The reference's step-8 GPU path (``step8_tuned.denoise``,
    step8_tuned.py:116-146), unmodified, imported from ``baseline/_ref``,
    on this GPU.

    ``vols``: {name: (volume, golden fixture)}. Per volume: one warm-up call
    (Triton JIT), then the ladder's own protocol (common.py:129-143: wall
    clock host->host around the call plus a synchronize, best of up to
    ``repeats`` calls within ``budget_s``), the device span of one call
    (CUDA events on the current stream around it: its pageable H2D, the
    kernels and library calls, the pinned D2H), the call's two copies timed
    alone the same way, and the device time without them; errors of the
    output against the golden fixture's step-0 float32 and float64 samples.
    """
    if not os.path.exists(os.path.join(REF_DIR, "step8_tuned.py")):
        return dict(unavailable="baseline/_ref has no step8_tuned.py (python bench.py --install-reference "
                                "<checkout> installs it)")
    if tuple(wl["patch"]) != (11, 11, 11):
        return dict(unavailable="the ladder's patch is fixed at 11^3 (common.py:28)")
    os.environ["VOL"] = ",".join(str(s) for s in wl["shape"])
    os.environ["STEP"] = str(wl["stride"])
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    try:
        import importlib

        import triton

        common = importlib.import_module("common")
        if tuple(common.VOL_SHAPE) != tuple(wl["shape"]) or common.STEP != wl["stride"]:
            return dict(unavailable=f"the ladder's common was imported with VOL={common.VOL_SHAPE}, "
                                    f"STEP={common.STEP}")
        s8 = importlib.import_module("step8_tuned")
    except Exception as exc:
        return dict(unavailable=f"import of the reference's step 8 failed: {type(exc).__name__}: {exc}")
    res = dict(source="baseline/_ref/step8_tuned.py (unmodified)", torch=torch.__version__,
               triton=triton.__version__, batch=s8.BATCH, gram_cfg=s8.GRAM_CFG, recon_cfg=s8.RECON_CFG)
    try:
        for name, (vol, fixture) in vols.items():
            t0 = time.perf_counter()
            out = s8.denoise(vol)
            torch.cuda.synchronize()
            first = time.perf_counter() - t0
            host = []
            deadline = time.perf_counter() + budget_s
            for _ in range(repeats):
                t0 = time.perf_counter()
                out = s8.denoise(vol)
                torch.cuda.synchronize()
                host.append(time.perf_counter() - t0)
                if time.perf_counter() > deadline:
                    break
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s.record()
            s8.denoise(vol)
            e.record()
            torch.cuda.synchronize()
            call_ms = s.elapsed_time(e)
            # the call's copies alone: pageable H2D as torch.from_numpy(vol).cuda() does (step8:118),
            # D2H into pinned memory as step8:144-146 does
            s.record()
            dv = torch.from_numpy(vol).cuda()
            e.record()
            torch.cuda.synchronize()
            h2d = s.elapsed_time(e)
            hb = torch.empty(dv.shape, pin_memory=True)
            s.record()
            hb.copy_(dv)
            e.record()
            torch.cuda.synchronize()
            d2h = s.elapsed_time(e)
            del dv, hb
            r = dict(host_ms=1e3 * min(host), host_ms_runs=[1e3 * h for h in host], first_call_ms=1e3 * first,
                     call_device_ms=call_ms, h2d_ms=h2d, d2h_ms=d2h, device_ms=call_ms - h2d - d2h)
            if fixture:
                r["accuracy"] = golden_accuracy(out, None, fixture)
            res[name] = r
    except Exception as exc:
        res["error"] = f"{type(exc).__name__}: {exc}"
    return res


def run_ours(args, wl):
    import torch
    import torch.distributed as dist

    from lowrank_gpu_fastest_b200.harness import make_phantom, make_phantom_lowrank

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    shape, patch, stride = wl["shape"], wl["patch"], wl["stride"]
    wl_name = next((k for k, v in WORKLOADS.items() if v is wl), None)
    fixtures = GOLDEN_FOR.get(wl_name, (None, None))

    # CPU baseline first (spawn pool before any heavy GPU work), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        vol0, _ = make_phantom_lowrank(shape, seed=0)
        cores = host_cores()
        n = args.cpu_sample or max(64, 256 * cores)  # ~10-15 s of CPU work
        rate, dt, used, kind = cpu_step0_rate(vol0, patch, stride, n, cores)
        who = ("the reference's own step0_numpy_loop.mppca_patch (baseline/_ref)" if kind == "reference"
               else "the step-0 loop restated in oracle/")
        cpu = dict(value=rate, unit="patches/s", cores=used, kind=kind,
                   sample=f"{n} patches evenly spaced over the corner list, {who} with the loop's "
                          f"weighted accumulate, {used} spawn workers x 1 BLAS thread, {dt:.1f} s wall")

    vol, _ = make_phantom_lowrank(shape, seed=rank)
    golden = fixtures[0] if (rank == 0 and fixtures[0]) else None
    main = time_form(torch, dist, args, wl, args.form, vol, rank, world, local, clocks=True, golden=golden)

    extra = {}
    if world == 1 and not args.single_form:
        # the other forms beside the timed one: accurate and the tensor-core forms
        # meet the float64 bar
        for f in ("plain", "accurate", "tensor", "tensor_bf16"):
            if f != args.form:
                r = time_form(torch, dist, args, wl, f, vol, rank, world, local, golden=golden)
                extra[f] = r
    ladder = {}
    if world == 1 and fixtures[1] and patch == (11, 11, 11) and not args.single_form:
        # the ladder's own phantom (common.make_phantom: rank 5 on a ~1000 baseline, sigma 4)
        vref, _ = make_phantom(shape)
        for f in ("plain", "accurate"):
            ladder[f] = time_form(torch, dist, args, wl, f, vref, rank, world, local, golden=fixtures[1])
    step8, libeigh = None, None
    if world == 1 and rank == 0 and not args.no_step8 and fixtures[0]:
        vref = make_phantom(shape)[0] if fixtures[1] else None
        vols = {"lowrank": (vol, fixtures[0])}
        if vref is not None:
            vols["ladder_phantom"] = (vref, fixtures[1])
        libeigh = library_eigh(torch, wl, vol, local)
        step8 = reference_step8(torch, wl, vols, repeats=args.step8_repeats)
    serving = None
    if world == 1 and rank == 0 and args.serving_requests > 0 and not args.single_form:
        try:
            serving = serving_run(args.serving_requests, args.rate, args.seed)
            serving["note"] = ("bounded sample of the serving stream; the full one is "
                               "bench.py --workload serving --duration 60")
        except Exception as exc:  # the headline numbers stand without it
            serving = dict(error=f"{type(exc).__name__}: {exc}")

    if rank == 0:
        P = main["P"]
        ph = main["phases"]
        roof = roofline(ph, shape, patch, P, args.form, main["ranks"])
        N = int(np.prod(patch))
        T = shape[3]
        vbytes = int(np.prod(shape)) * 4
        fp32_peak = fp32_simt_peak_tflops(torch)
        tf32_peak = fp32_simt_peak_tflops(torch, tf32=True)
        total_flops = 4 * N * T * T * P

        def summary(r):
            d = dict(ms_per_volume=r["ms_per_step"], patches_per_s=r["value"], e2e_ms=r["e2e_ms"],
                     e2e_patches_per_s=r["e2e_value"], phases_ms=r["phases"], device_status=r["status"],
                     e2e_output_identical=r["e2e_output_identical"])
            if "accuracy" in r:
                d["accuracy"] = r["accuracy"]
            return d

        line = dict(
            metric="patches_per_s", value=main["value"], unit="patches/s", n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=main["ms_per_step"], ms_per_volume=main["ms_per_step"],
            higher_is_better=True, scaling="weak",
            vs_baseline=main["e2e_value"] / (12600 / (PUBLISHED_STEP8_MS * 1e-3)) if wl_name == "headline" else None,
            vs_baseline_basis="e2e host->host patches/s / published step-8 (66.5 ms host->host, "
                              "12600 patches, unstated GPU)",
            dtype="f32", data="synthetic", form=args.form,
            config=bench_config(wl, world),
            e2e=dict(value=main["e2e_value"], unit="patches/s", ms_per_step=main["e2e_ms"],
                     h2d_bytes_per_step=vbytes, d2h_bytes_per_step=vbytes + 4 * P,
                     path="lrd_denoise_host (pinned host in/out, H2D + denoise + D2H + sync)",
                     output_identical_to_device_call=main["e2e_output_identical"]),
            phases_ms=ph,
            device_status=main["status"],
            roofline=roof,
            fp32_simt=dict(peak_tflops_sgemm=fp32_peak, peak_tflops_tf32_gemm=tf32_peak,
                           algorithmic_tflops_gram_recon=total_flops / ((ph["gram"] + ph["recon"]) * 1e-3) / 1e12,
                           **executed_fp32(ph, shape, patch, stride, main["ranks"], fp32_peak, args.form)),
            cpu_baseline=cpu,
            clocks=main["clocks"],
            gpu_launches=6 * args.steps,
            gpu_launches_note="per step: center, gram (column TMA or tensor), eigh, eigh_refine, "
                              "refine_advance, recon (plus two status memsets)",
            wall_s_timed_region=main["wall"],
        )
        if "accuracy" in main:
            line["accuracy"] = main["accuracy"]
        if extra:
            line["forms"] = {f: summary(r) for f, r in extra.items()}
        if ladder:
            line["ladder_phantom"] = {f: summary(r) for f, r in ladder.items()}
        if libeigh is not None:
            line["eigh_vs_library"] = libeigh
        if serving is not None:
            line["serving"] = serving
        if step8 is not None:
            line["reference_step8"] = step8
            lr = step8.get("lowrank")
            if lr:
                allf = dict(extra, **{args.form: main})
                line["vs_step8"] = {
                    f"device_{f}": lr["device_ms"] / r["ms_per_step"] for f, r in allf.items()}
                line["vs_step8"].update({f"e2e_{f}": lr["host_ms"] / r["e2e_ms"] for f, r in allf.items()})
                line["vs_step8"]["basis"] = ("device: step 8's call on the device less its two copies / our "
                                             "device-timed denoise; e2e: step 8 host->host best-of / our "
                                             "lrd_denoise_host; both on the benchmark phantom")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def executed_fp32(ph, shape, patch, stride, ranks, fp32_peak, form):
    """FP32 work the Gram and reconstruction kernels execute (not the 2 N T^2
    per patch of the full-square algorithmic count), over their phase times,
    as a fraction of the measured SGEMM rate: the column Gram forms each
    z-plane's Gram once per (x, y) column on the upper triangle in 4x4 blocks
    and adds it into the windows; the reconstruction does y = (x - m) V_p^T
    and y V_p (4 p T flops) for every covered voxel-patch pair."""
    from lowrank_gpu_fastest_b200.problem import axis_corners

    X, Y, Z, T = shape
    px, py, pz = patch
    ncx = len(axis_corners(X, px, stride))
    ncy = len(axis_corners(Y, py, stride))
    nb = (T + 3) // 4
    gram_fl = 2.0 * ncx * ncy * Z * px * py * 16 * nb * (nb + 1) / 2
    N = px * py * pz
    recon_fl = float(4 * T * N * np.asarray(ranks, dtype=np.float64).sum())
    out = dict(executed_gflop_gram=gram_fl / 1e9, executed_gflop_recon=recon_fl / 1e9,
               mean_rank=float(np.mean(ranks)))
    if form not in ("tensor", "tensor_bf16") or T > 64:
        out["executed_tflops_gram"] = gram_fl / (ph["gram"] * 1e-3) / 1e12
        out["gram_frac_of_sgemm"] = out["executed_tflops_gram"] / fp32_peak
    if phase_kernel("recon", T, form) != "recon_tc_kernel":
        out["executed_tflops_recon"] = recon_fl / (ph["recon"] * 1e-3) / 1e12
        out["recon_frac_of_sgemm"] = out["executed_tflops_recon"] / fp32_peak
    return out


def roofline(ph, shape, patch, P, form, ranks=None):
    """``roofline`` object for the dominant phase of one denoise (phase ms
    ``ph``): algorithmic FLOPs (Gram, reconstruction: 2 N T^2 per patch) or
    bytes (centre: volume in/out + means; eigensolve: Gram block in and
    eigenvector block out, 2 T^2 x 4 per patch) per launch over the phase's
    event time, against the measured peaks; DRAM traffic per launch from the
    committed ncu summary. For the reconstruction the executed FP32 rate
    (4 p T flops per covered voxel-patch pair, p the patch's rank) is given
    beside it."""
    peaks = measured_peaks()
    dom = max(ph, key=ph.get)
    N = int(np.prod(patch))
    T = shape[3]
    vbytes = int(np.prod(shape)) * 4
    flops_unit = {"gram": 2 * N * T * T, "recon": 2 * N * T * T}
    kname = phase_kernel(dom, T, form)
    traffic = ncu_traffic().get(kname)
    if dom in flops_unit:
        achieved = flops_unit[dom] * P / (ph[dom] * 1e-3) / 1e12
        note = None
        if not (dom == "gram" and kname == "gram_tc_kernel"):
            note = ("FFMA on the CUDA cores (float32 products and sums); the fraction is of the bf16 "
                    "tensor peak, fp32_simt compares the executed work with the measured SGEMM peak")
        r = dict(kernel=kname, bound="tensor", achieved=achieved, peak=peaks["bf16_tflops"], unit="TFLOP/s",
                 frac=achieved / peaks["bf16_tflops"], traffic=traffic,
                 peak_source=f"bf16 dense burst {peaks['source']}",
                 algorithmic=f"2*N*T^2 = {flops_unit[dom]} flop/patch x {P} patches per launch", note=note)
        if dom == "recon" and ranks is not None:
            ex = 4.0 * T * N * float(np.asarray(ranks, dtype=np.float64).sum())
            r["executed_tflops"] = ex / (ph[dom] * 1e-3) / 1e12
            r["executed"] = "4*p*T flop per covered voxel-patch pair (rank-p projection)"
        return r
    byts = {"center": 2 * vbytes + vbytes // T, "eigh_mp": 2 * P * T * T * 4}[dom]
    achieved = byts / (ph[dom] * 1e-3) / 1e9
    return dict(kernel=kname, bound="hbm", achieved=achieved, peak=peaks["hbm_gbs"], unit="GB/s",
                frac=achieved / peaks["hbm_gbs"], traffic=traffic, peak_source=f"HBM copy {peaks['source']}",
                algorithmic=f"{byts / P:.0f} B/patch x {P} patches per launch",
                note="the eigensolver is latency-bound (Householder and Sturm recurrences), not HBM-bound"
                if dom == "eigh_mp" else None)


def run_sharded(args, wl):
    """N GPUs, one volume: the workload's volume repeated N times along x
    ((X*N, Y, Z, T)), its x-corners cut in N slabs (one per rank), one NCCL
    halo exchange between neighbours per step. Per-GPU work is about the
    single-GPU workload's (weak scaling)."""
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank
    from lowrank_gpu_fastest_b200.problem import n_patches
    from lowrank_gpu_fastest_b200.shard import CudaSlab, run_slab, slab_partition

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    X, Y, Z, T = wl["shape"]
    gshape = (X * world, Y, Z, T)
    patch, stride = wl["patch"], wl["stride"]
    parts = slab_partition(gshape, patch, stride, world)
    me = parts[rank]
    base, _ = make_phantom_lowrank(wl["shape"], seed=0)
    planes = np.ascontiguousarray(np.take(base, np.arange(me["x0"], me["x1"]) % X, axis=0))
    slab = CudaSlab(gshape, rank, world, patch, stride, args.form, device=local)
    h_in = torch.from_numpy(planes).pin_memory()
    own = slab.own[1] - slab.own[0]
    h_out = torch.empty((own, Y, Z, T), dtype=torch.float32, pin_memory=True)
    slab.load(h_in)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    P_total = n_patches(gshape, patch, stride)
    # this rank's kernels per step: centre, Gram, eigensolve, refine, refine cursor, and one
    # reconstruction per non-empty part (halo out, interior, halo in)
    launches = 5 + int(slab.halo_out.numel() > 0) + int(slab.own[1] - slab.own[0] > slab.plan.hin) + \
        int(slab.plan.hin > 0)

    def step():
        run_slab(slab, rank, world)

    dist.barrier()  # brings the communicator up before the first send/recv
    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    dist.barrier()
    torch.cuda.synchronize()
    for s, e in evs:
        flush.zero_()
        s.record(stream)
        step()
        e.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    t = torch.tensor([sum(s.elapsed_time(e) for s, e in evs)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps
    value = P_total / (ms_per_step * 1e-3)

    # e2e: the slab's planes from pinned host memory, the step, the owned planes back
    def e2e_step():
        slab.vol.copy_(h_in, non_blocking=True)
        run_slab(slab, rank, world)
        h_out.copy_(slab.owned(), non_blocking=True)
        torch.cuda.synchronize()

    for _ in range(max(1, args.warmup)):
        e2e_step()
    dist.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    t = torch.tensor([statistics.mean(e2e_ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms_step = float(t.item())
    halo_bytes = slab.halo_out.numel() * 8
    roof = None
    if rank == 0:  # the per-GPU kernels' roofline: phase events of the single-GPU workload's plan
        from lowrank_gpu_fastest_b200 import api

        plan = api.get_plan(wl["shape"], patch, stride, form=args.form, device=local)
        d_vol = torch.from_numpy(base).to(dev)
        d_out = torch.empty_like(d_vol)
        ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device=dev)
        for _ in range(2):
            plan.denoise(d_vol.data_ptr(), d_out.data_ptr(), None, ws.data_ptr(), stream.cuda_stream)
        plan.set_profiling(True)
        for _ in range(3):
            plan.denoise(d_vol.data_ptr(), d_out.data_ptr(), None, ws.data_ptr(), stream.cuda_stream)
        phases, ncalls = plan.phase_ms()
        plan.set_profiling(False)
        roof = roofline({k: v / max(ncalls, 1) for k, v in phases.items()}, wl["shape"], patch,
                        plan.n_patches, args.form)
        del d_vol, d_out, ws
    if rank == 0:
        line = dict(
            metric="patches_per_s", value=value, unit="patches/s", n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=ms_per_step, ms_per_volume=ms_per_step,
            higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
            config=dict(workload=f"{wl['desc']} repeated {world}x along x, cut in {world} x-slabs",
                        shape=list(gshape), patch=list(patch), stride=stride, form=args.form,
                        phantom="rank-4 [0,1] + N(0,0.05^2) seed 0, tiled along x",
                        l2="flushed by a 256 MiB write between timed steps (outside the events)",
                        parallelism=f"x-slab shard x{world}, NCCL send/recv halo "
                                    f"({halo_bytes / 1e6:.1f} MB per boundary)",
                        patches=P_total),
            e2e=dict(value=P_total / (e2e_ms_step * 1e-3), unit="patches/s", ms_per_step=e2e_ms_step,
                     h2d_bytes_per_step=int(h_in.numel() * 4), d2h_bytes_per_step=int(h_out.numel() * 4),
                     path="per rank: H2D of its slab planes, slab step with halo exchange, D2H of owned "
                          "planes (rank 0's bytes; max time over ranks)"),
            clocks=clocks,
            roofline=roof,
            cpu_baseline=None,
            gpu_launches=launches * args.steps,
            gpu_launches_note="rank 0's own kernels (NCCL's send/recv kernels not counted)",
        )
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def run_batched(args):
    """Batched uneven form: ``--volumes`` seeded volumes of mixed shapes, the
    whole batch one CUDA-graph launch of packed kernels per step
    (device-timed), against the same volumes denoised one by one (the sum of
    their single-volume device times)."""
    import torch

    from lowrank_gpu_fastest_b200 import api
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank
    from lowrank_gpu_fastest_b200.problem import n_patches
    from lowrank_gpu_fastest_b200.serve import draw_request_shapes

    shapes = draw_request_shapes(args.volumes, seed=args.seed, big_fraction=0.0)
    vols = [torch.from_numpy(make_phantom_lowrank(r["shape"], seed=i, sigma=r["sigma"])[0]).cuda()
            for i, r in enumerate(shapes)]
    patches = [r["patch"] for r in shapes]
    strides = [r["stride"] for r in shapes]
    P = sum(n_patches(r["shape"], r["patch"], r["stride"]) for r in shapes)

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            out.append(s.elapsed_time(e))
        return out

    for _ in range(args.warmup):
        api.denoise_batch(vols, patches, strides, use_graph=True)
    torch.cuda.synchronize()
    times = timed(lambda: api.denoise_batch(vols, patches, strides, use_graph=True), args.steps)
    ms = statistics.mean(times)
    launches = next(iter(api._batch_plans.values())).launches
    api._batch_plans.clear()  # frees the batch's workspace (tens of GB for the stride-1 volumes)
    torch.cuda.empty_cache()
    # the same volumes one by one: lrd_denoise each on one shared workspace, warm plans
    from lowrank_gpu_fastest_b200 import _native

    plans = [_native.Plan(tuple(v.shape), pt, st) for v, pt, st in zip(vols, patches, strides)]
    ws = torch.empty(max(p.workspace_bytes for p in plans), dtype=torch.uint8, device="cuda")
    out = torch.empty(max(v.numel() for v in vols), dtype=torch.float32, device="cuda")
    sid = torch.cuda.current_stream().cuda_stream
    single = []
    for v, plan in zip(vols, plans):
        def one():
            plan.denoise(v.data_ptr(), out.data_ptr(), None, ws.data_ptr(), sid)

        one()
        torch.cuda.synchronize()
        single.append(min(timed(one, 2)))
    N = [int(np.prod(r["patch"])) for r in shapes]
    flops = sum(4 * n * r["shape"][3] ** 2 * n_patches(r["shape"], r["patch"], r["stride"]) for n, r in zip(N, shapes))
    print(json.dumps(dict(
        metric="patches_per_s", workload="batched", value=P / (ms * 1e-3), unit="patches/s", n_gpus=1,
        steps=args.steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True, dtype="f32", data="synthetic",
        single_volume_ms_sum=sum(single), vs_single_volumes=sum(single) / ms,
        gpu_launches=launches * args.steps, launches_per_batch=launches,
        launches_one_by_one=6 * len(shapes),
        config=dict(volumes=args.volumes, seed=args.seed, patches=P, algorithmic_tflop=flops / 1e12,
                    shapes=[[list(r["shape"]), r["patch"][0], r["stride"]] for r in shapes],
                    note="one lrd_batch_denoise CUDA-graph launch per step: packed kernels, one grid per phase and "
                         "kernel class across the volumes"),
        achieved_tflops=flops / (ms * 1e-3) / 1e12)), flush=True)


def serving_run(requests, rate, seed=0, duration=None, distinct=24, slots=4):
    """Serving form: Poisson arrivals at ``rate`` req/s (``requests`` of them,
    or as many as arrive within ``duration`` s) of the serving mix (x, y in
    64..128, z in 32..64, T in {32, 48, 64, 96}, patch 5^3 / 7^3 / 11^3,
    stride 1..3; 10% 128x128x64x96 / 11^3 / stride 2), submitted to a
    ``Server`` as they arrive; p50 / p99 latency (submit to result) and
    patches/s. The requests cycle through ``distinct`` seeded volumes of the
    mix (a pool, so a long stream needs no volume generation on the clock);
    the baseline is the same request list solved one after another host ->
    host through ``denoise`` (each distinct volume timed once, warm)."""
    import torch

    from lowrank_gpu_fastest_b200 import api
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank
    from lowrank_gpu_fastest_b200.problem import n_patches
    from lowrank_gpu_fastest_b200.serve import Server, draw_request_shapes, poisson_arrivals

    arr = poisson_arrivals(rate, duration if duration else float("inf"), seed=seed,
                           max_count=None if duration else requests)
    k = max(1, min(distinct, len(arr)))
    shapes = draw_request_shapes(k, seed=seed, big_fraction=0.1)
    vols = [make_phantom_lowrank(r["shape"], seed=i, sigma=r["sigma"])[0] for i, r in enumerate(shapes)]
    seq = []
    for v, r in zip(vols, shapes):  # warm plans, then one host -> host solve each
        api.denoise(torch.from_numpy(v).cuda(), r["patch"], r["stride"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        api.denoise(v, r["patch"], r["stride"])
        seq.append(time.perf_counter() - t0)
    idx = [i % k for i in range(len(arr))]
    P = sum(n_patches(vols[i].shape, shapes[i]["patch"], shapes[i]["stride"]) for i in idx)
    seq_s = sum(seq[i] for i in idx)
    import collections

    with Server(n_slots=slots) as srv:
        start = time.perf_counter()
        pending = collections.deque()  # results are dropped as they arrive (host memory stays bounded)
        for t, i in zip(arr, idx):
            now = time.perf_counter() - start
            if t > now:
                time.sleep(t - now)
            pending.append(srv.submit(vols[i], shapes[i]["patch"], shapes[i]["stride"]))
            while pending and pending[0].done():
                pending.popleft().result()
        while pending:
            pending.popleft().result()
        st = srv.stats()
    return dict(value=st["patches_per_s"], unit="patches/s", p50_ms=st["p50_ms"], p99_ms=st["p99_ms"],
                mean_ms=st["mean_ms"], requests=st["n"], requests_per_s=st["requests_per_s"],
                offered_rate_per_s=rate, duration_s=duration, span_s=st["span_s"],
                sequential_patches_per_s=P / seq_s, vs_sequential=st["patches_per_s"] / (P / seq_s),
                sequential_ms_per_request=1e3 * seq_s / max(1, len(idx)),
                config=dict(requests=len(arr), rate_per_s=rate, seed=seed, slots=slots, distinct_volumes=k,
                            mix="x,y 64..128, z 32..64, T {32,48,64,96}, patch {5,7,11}^3, stride {1,2,3}; "
                                "10% 128x128x64x96 / 11^3 / stride 2"))


def run_serving(args):
    """``--workload serving``: ``--requests`` requests at ``--rate`` req/s, or
    with ``--duration`` the stream of that many seconds (the serving
    configuration: 40 req/s for 60 s)."""
    r = serving_run(args.requests, args.rate, args.seed, duration=args.duration or None)
    print(json.dumps(dict(metric="patches_per_s", workload="serving", n_gpus=1, higher_is_better=True, dtype="f32",
                          data="synthetic", **r)), flush=True)


def main():
    args = parse()
    if args.install_reference:
        return install_reference(args.install_reference)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "serving":
        return run_serving(args)
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl)
    elif dist_env()[1] > 1 and args.parallel == "shard":
        run_sharded(args, wl)
    else:
        run_ours(args, wl)


if __name__ == "__main__":
    main()
