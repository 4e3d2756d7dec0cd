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

``--impl reference`` times the reference algorithm's CPU implementation (the
step-0 NumPy loop restated in oracle/, all host cores through a spawn pool)
on a bounded sample of the same workload's patches.
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
def phase_kernel(phase, T, form):
    """Kernel that a plan phase launches for T frames (the eigensolve phase
    also runs the refine kernel and its cursor, both under 0.5% of it)."""
    if phase == "gram":
        return "gram_tc_kernel" if (form == "tensor" and T <= 64) else "gram_z_kernel"
    if phase == "eigh_mp":
        return "eigh_reg_kernel" if T <= 64 else "eigh_cta_kernel"
    if phase == "recon" and form == "plain" and 45 <= T <= 48:
        return "recon_kernel_t24s2"  # 24 frames x 2 threads, built with 112 registers
    return {"center": "center_kernel", "recon": "recon_kernel"}[phase]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["plain", "accurate", "tensor"], default="plain")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched", "serving"], default="headline")
    ap.add_argument("--volumes", type=int, default=24, help="batched: number of volumes")
    ap.add_argument("--requests", type=int, default=48, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=40.0, help="serving: Poisson arrival rate (req/s)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    """Patches/s of the step-0 loop (oracle port) over a sample of the corner
    list, spread over ``processes`` spawn workers with one BLAS thread each.

    Each worker receives the volume once (pool initializer) and runs the
    step-0 per-patch work - gather, centre, SVD, MP rank, reconstruct, weighted
    accumulate into its own ``out``/``wsum`` - over its share of the sample;
    the wall time of that loop across the pool is the measurement.
    """
    import multiprocessing as mp

    from oracle import mppca as orc

    corners = orc.patch_corners(vol.shape, patch, stride)
    sample = corners[np.linspace(0, len(corners) - 1, n_patches_sample).astype(int)]
    chunks = [c for c in np.array_split(sample, processes) if len(c)]
    for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(chunks), initializer=_cpu_init, initargs=(vol, patch)) as pool:
        pool.map(_cpu_worker, [c[:1] for c in chunks])  # warm (imports, first SVD)
        t0 = time.perf_counter()
        pool.map(_cpu_worker, chunks)
        dt = time.perf_counter() - t0
    return len(sample) / dt, dt, len(chunks)


_CPU = {}


def _cpu_init(vol, patch):
    _CPU["vol"] = vol
    _CPU["patch"] = patch
    _CPU["out"] = np.zeros_like(vol)
    _CPU["wsum"] = np.zeros(vol.shape[:3] + (1,), dtype=vol.dtype)


def _cpu_worker(corners):
    from oracle import mppca as orc

    vol, (px, py, pz) = _CPU["vol"], _CPU["patch"]
    out, wsum = _CPU["out"], _CPU["wsum"]
    for i, j, k in corners:
        sl = np.s_[i:i + px, j:j + py, k:k + pz]
        xd, p = orc.mppca_patch(vol[sl].reshape(-1, vol.shape[-1]))
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
        r, _, used = cpu_step0_rate(vol, wl["patch"], wl["stride"], per_step, cores)
        rates.append(r)
    from lowrank_gpu_fastest_b200.problem import n_patches

    P = n_patches(wl["shape"], wl["patch"], wl["stride"])
    value = float(statistics.mean(rates))
    line = dict(
        impl="reference", metric="patches_per_s", value=value, unit="patches/s", n_gpus=args.gpus,
        steps=args.steps, warmup=args.warmup, ms_per_step=1e3 * per_step / value,
        ms_per_volume=1e3 * P / value, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f32", data="synthetic",
        config=dict(workload=wl["desc"], shape=list(wl["shape"]), patch=list(wl["patch"]),
                    stride=wl["stride"], phantom="rank-4 [0,1] + N(0,0.05^2), seed 0"),
        cpu_baseline=dict(value=value, unit="patches/s", cores=used, kind="port",
                          sample=f"{per_step} patches per step, evenly spaced over the {P}-patch corner "
                                 f"list; step-0 NumPy loop (SVD + MP rank + weighted accumulate), one BLAS "
                                 f"thread per spawn worker"),
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


def run_ours(args, wl):
    import torch
    import torch.distributed as dist

    from lowrank_gpu_fastest_b200 import api
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    shape, patch, stride = wl["shape"], wl["patch"], wl["stride"]

    # CPU baseline first (spawn pool before any heavy GPU work), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        vol0, _ = make_phantom_lowrank(shape, seed=0)
        cores = host_cores()
        n = args.cpu_sample or max(64, 256 * cores)  # ~10-15 s of CPU work
        rate, dt, used = cpu_step0_rate(vol0, patch, stride, n, cores)
        cpu = dict(value=rate, unit="patches/s", cores=used, kind="port",
                   sample=f"{n} patches evenly spaced over the corner list, step-0 NumPy loop "
                          f"(SVD + MP rank + weighted accumulate), {used} spawn workers x 1 BLAS "
                          f"thread, {dt:.1f} s wall")

    vol, _ = make_phantom_lowrank(shape, seed=rank)
    dev = torch.device("cuda", local)
    d_vol = torch.from_numpy(vol).to(dev)
    d_out = torch.empty_like(d_vol)
    brick = tuple(int(v) for v in args.brick.split(",")) if args.brick else None
    plan = api.get_plan(shape, patch, stride, form=args.form, device=local, brick=brick, split=args.split)
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

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    plan.set_profiling(True)
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
    clocks = sampler.stop()
    phases, ncalls = plan.phase_ms()
    plan.set_profiling(False)
    ms_total = sum(s.elapsed_time(e) for s, e in evs)
    t = torch.tensor([ms_total], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps
    value = world * P / (ms_per_step * 1e-3)

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

    if rank == 0:
        ph = {k: v / max(ncalls, 1) for k, v in phases.items()}
        roof = roofline(ph, shape, patch, P, args.form)
        N = int(np.prod(patch))
        T = shape[3]
        vbytes = int(np.prod(shape)) * 4
        fp32_peak = fp32_simt_peak_tflops(torch)
        tf32_peak = fp32_simt_peak_tflops(torch, tf32=True)
        total_flops = 4 * N * T * T * P
        line = dict(
            metric="patches_per_s", value=value, unit="patches/s", n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=ms_per_step, ms_per_volume=ms_per_step,
            higher_is_better=True, scaling="weak",
            vs_baseline=(world * P / (e2e_ms_step * 1e-3)) / (12600 / (PUBLISHED_STEP8_MS * 1e-3))
            if wl is WORKLOADS["headline"] else None,
            vs_baseline_basis="e2e host->host patches/s / published step-8 (66.5 ms host->host, "
                              "12600 patches, unstated GPU)",
            dtype="f32", data="synthetic",
            config=dict(workload=wl["desc"], shape=list(shape), patch=list(patch), stride=stride,
                        form=args.form, phantom="rank-4 [0,1] + N(0,0.05^2), seed = rank",
                        l2="flushed by a 256 MiB write between timed steps (outside the events)",
                        parallelism=f"replica x{world}" if world > 1 else "single GPU"),
            e2e=dict(value=world * P / (e2e_ms_step * 1e-3), unit="patches/s",
                     ms_per_step=e2e_ms_step, h2d_bytes_per_step=vbytes,
                     d2h_bytes_per_step=vbytes + 4 * P,
                     path="lrd_denoise_host (pinned host in/out, H2D + denoise + D2H + sync)"),
            phases_ms=ph,
            roofline=roof,
            fp32_simt=dict(peak_tflops_sgemm=fp32_peak, peak_tflops_tf32_gemm=tf32_peak,
                           achieved_tflops_gram_recon=total_flops / ((ph["gram"] + ph["recon"]) * 1e-3) / 1e12),
            cpu_baseline=cpu,
            clocks=clocks,
            gpu_launches=6 * args.steps,
            gpu_launches_note="per step: center, gram (column TMA or tensor), eigh, eigh_refine, "
                              "refine_advance, recon (plus two status memsets)",
            wall_s_timed_region=wall,
        )
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def roofline(ph, shape, patch, P, form):
    """``roofline`` object for the dominant phase of one denoise (phase ms
    ``ph``): algorithmic FLOPs (Gram, reconstruction: 2 N T^2 per patch) or
    bytes (centre: volume in/out + means; eigensolve: Gram block in and
    eigenvector block out, 2 T^2 x 4 per patch) per launch over the phase's
    event time, against the measured peaks; DRAM traffic per launch from the
    committed ncu summary."""
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
                    "tensor peak, fp32_simt compares the contractions with the measured SGEMM peak")
        return dict(kernel=kname, bound="tensor", achieved=achieved, peak=peaks["bf16_tflops"], unit="TFLOP/s",
                    frac=achieved / peaks["bf16_tflops"], traffic=traffic,
                    peak_source=f"bf16 dense burst {peaks['source']}",
                    algorithmic=f"2*N*T^2 = {flops_unit[dom]} flop/patch x {P} patches per launch", note=note)
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
    """Batched uneven form: ``--volumes`` seeded volumes of mixed shapes in one
    CUDA-graph launch per step (device-timed)."""
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
    for _ in range(args.warmup):
        api.denoise_batch(vols, patches, strides, use_graph=True)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        api.denoise_batch(vols, patches, strides, use_graph=True)
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    ms = statistics.mean(times)
    N = [int(np.prod(r["patch"])) for r in shapes]
    flops = sum(4 * n * r["shape"][3] ** 2 * n_patches(r["shape"], r["patch"], r["stride"]) for n, r in zip(N, shapes))
    print(json.dumps(dict(
        metric="patches_per_s", workload="batched", value=P / (ms * 1e-3), unit="patches/s", n_gpus=1,
        steps=args.steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True, dtype="f32", data="synthetic",
        config=dict(volumes=args.volumes, seed=args.seed, patches=P, algorithmic_tflop=flops / 1e12,
                    shapes=[[list(r["shape"]), r["patch"][0], r["stride"]] for r in shapes],
                    note="one lrd_batch_denoise CUDA-graph launch per step, volumes on 4 internal streams"),
        achieved_tflops=flops / (ms * 1e-3) / 1e12)), flush=True)


def run_serving(args):
    """Serving form: ``--requests`` seeded requests arriving as a Poisson
    stream at ``--rate`` req/s (10% 128x128x64x96 / 11^3 / stride 2), served
    with continuous batching; compared with solving the same requests one
    after another."""
    import torch

    from lowrank_gpu_fastest_b200 import api
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank
    from lowrank_gpu_fastest_b200.serve import Server, draw_request_shapes, poisson_arrivals

    shapes = draw_request_shapes(args.requests, seed=args.seed, big_fraction=0.1)
    arr = poisson_arrivals(args.rate, float("inf"), seed=args.seed, max_count=args.requests)
    vols = [make_phantom_lowrank(r["shape"], seed=i, sigma=r["sigma"])[0] for i, r in enumerate(shapes)]
    # warm: plans and one solve per distinct problem
    seen = set()
    for v, r in zip(vols, shapes):
        k = (v.shape, r["patch"], r["stride"])
        if k not in seen:
            seen.add(k)
            api.denoise(torch.from_numpy(v).cuda(), r["patch"], r["stride"])
    torch.cuda.synchronize()
    # sequential plain-form solves (host -> host each)
    t0 = time.perf_counter()
    for v, r in zip(vols, shapes):
        api.denoise(v, r["patch"], r["stride"])
    seq_s = time.perf_counter() - t0
    from lowrank_gpu_fastest_b200.problem import n_patches

    P = sum(n_patches(v.shape, r["patch"], r["stride"]) for v, r in zip(vols, shapes))
    with Server(n_slots=4) as srv:
        start = time.perf_counter()
        futs = []
        for t, v, r in zip(arr, vols, shapes):
            now = time.perf_counter() - start
            if t > now:
                time.sleep(t - now)
            futs.append(srv.submit(v, r["patch"], r["stride"]))
        for f in futs:
            f.result()
        st = srv.stats()
    print(json.dumps(dict(
        metric="patches_per_s", workload="serving", value=st["patches_per_s"], unit="patches/s", n_gpus=1,
        higher_is_better=True, dtype="f32", data="synthetic",
        p50_ms=st["p50_ms"], p99_ms=st["p99_ms"], mean_ms=st["mean_ms"], requests=st["n"],
        requests_per_s=st["requests_per_s"], sequential_patches_per_s=P / seq_s,
        vs_sequential=st["patches_per_s"] / (P / seq_s),
        config=dict(requests=args.requests, rate_per_s=args.rate, seed=args.seed, slots=4,
                    mix="x,y 64..128, z 32..64, T {32,48,64,96}, patch {5,7,11}^3, stride {1,2,3}; "
                        "10% 128x128x64x96 / 11^3 / stride 2"))), flush=True)


def main():
    args = parse()
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
