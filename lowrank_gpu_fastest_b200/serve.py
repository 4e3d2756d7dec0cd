"""Serving loop: continuous batching of denoise requests on one GPU.

Requests (a host volume plus its patch shape and stride) are submitted from
any thread and return a ``concurrent.futures.Future``. One scheduler thread
owns the device:

* admission - a pending request is started as soon as a slot (a CUDA stream)
  is free and its device footprint (input, output, rank array, plan
  workspace) fits in the HBM that ``cudaMemGetInfo`` reports free minus a
  reserve; requests that do not fit wait, in arrival order, while others run;
* each admitted request runs on its slot's stream: host->device copy from a
  pinned staging buffer (filled at admission, so only admitted requests hold
  pinned host memory and a long backlog holds no more than the callers'
  arrays), ``lrd_denoise``, device->host copy into pinned memory, an event;
  requests on different slots overlap on the device;
* completion - the scheduler polls the events without blocking, resolves the
  future with the denoised volume (and ranks), frees the slot, returns the
  request's device buffers to a pool (reused by later requests of the same
  size class, so a steady stream allocates no device memory after warm-up)
  and admits the next requests.

Because every kernel is deterministic and a request's arithmetic does not
depend on what runs beside it, a request's result is bit-identical alone and
in the mix. ``stats()`` reports per-request latency percentiles (submit to
result) and throughput.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np


@dataclass
class _Req:
    vol: np.ndarray
    h_in: object
    patch: tuple
    stride: int
    form: str
    t_submit: float
    future: Future
    n_patches: int = 0
    need: int = 0
    slot: int = -1
    bufs: dict = field(default_factory=dict)
    event: object = None
    t_start: float = 0.0


class _Pool:
    """Buffers kept for reuse across requests, by kind and size class: a
    request takes the smallest free buffer of its kind that is large enough
    (sizes rounded up to 2 MiB classes) and gives it back when it completes,
    so a steady stream allocates nothing after warm-up."""

    CLASS = 2 << 20

    def __init__(self, alloc):
        self.alloc = alloc  # (kind, nbytes) -> uint8 tensor of nbytes
        self.free: dict = collections.defaultdict(list)
        self.free_bytes = 0

    def take(self, kind, nbytes):
        nb = max(self.CLASS, -(-int(nbytes) // self.CLASS) * self.CLASS)
        lst = self.free[kind]
        best = None
        for i, t in enumerate(lst):
            if t.numel() >= nb and (best is None or t.numel() < lst[best].numel()):
                best = i
        if best is not None:
            t = lst.pop(best)
            self.free_bytes -= t.numel()
            return t
        return self.alloc(kind, nb)

    def give(self, kind, t):
        self.free[kind].append(t)
        self.free_bytes += t.numel()

    def trim(self):
        """Drop every free buffer (the device memory returns to the allocator)."""
        self.free.clear()
        self.free_bytes = 0


class Server:
    """Continuous-batching denoise server on one CUDA device."""

    def __init__(self, device=0, n_slots=4, hbm_reserve_bytes=2 << 30, hbm_budget_bytes=None,
                 autotune=False, poll_s=0.0002):
        import torch

        self.torch = torch
        self.device = device
        self.n_slots = int(n_slots)
        self.reserve = int(hbm_reserve_bytes)
        self.budget = hbm_budget_bytes  # optional cap on this server's device bytes in flight
        self.autotune = autotune
        self.poll_s = poll_s
        self._pending: collections.deque = collections.deque()
        self._running: dict = {}
        self._lock = threading.Condition()
        self._stop = False
        self._thread = None
        self._done: list = []  # (t_submit, t_start, t_done, n_patches, shape)
        self._in_flight_bytes = 0
        with torch.cuda.device(device):
            self._streams = [torch.cuda.Stream(device=device) for _ in range(self.n_slots)]
        self._free_slots = list(range(self.n_slots))

        def alloc(kind, nbytes):
            return torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{device}")

        self._pool = _Pool(alloc)

    # -- public --------------------------------------------------------------
    def start(self):
        self._stop = False
        self._thread = threading.Thread(target=self._loop, name="lrd-serve", daemon=True)
        self._thread.start()
        return self

    def stop(self, wait=True):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        if wait and self._thread is not None:
            self._thread.join()

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def submit(self, vol, patch=(11, 11, 11), stride=3, form="plain") -> Future:
        from .problem import n_patches

        t_submit = time.perf_counter()
        fut: Future = Future()
        try:
            vol = np.ascontiguousarray(vol, dtype=np.float32)
            if vol.ndim != 4:
                raise ValueError("volume must be 4D (x, y, z, t)")
            npatch = n_patches(vol.shape, tuple(int(p) for p in patch), int(stride))
        except Exception as e:  # a bad request fails its own future only
            fut.set_exception(e)
            return fut
        # staged into pinned memory at admission: a backlog of waiting requests
        # holds only the callers' arrays
        r = _Req(vol, None, tuple(int(p) for p in patch), int(stride), form, t_submit, fut)
        r.n_patches = npatch
        with self._lock:
            self._pending.append(r)
            self._lock.notify_all()
        return fut

    def stats(self):
        with self._lock:
            done = list(self._done)
        if not done:
            return dict(n=0)
        lat = np.array([d[2] - d[0] for d in done])
        t0 = min(d[0] for d in done)
        t1 = max(d[2] for d in done)
        patches = sum(d[3] for d in done)
        return dict(n=len(done), p50_ms=1e3 * float(np.percentile(lat, 50)),
                    p99_ms=1e3 * float(np.percentile(lat, 99)), mean_ms=1e3 * float(lat.mean()),
                    span_s=t1 - t0, patches=patches, patches_per_s=patches / max(t1 - t0, 1e-9),
                    requests_per_s=len(done) / max(t1 - t0, 1e-9))

    def reset_stats(self):
        with self._lock:
            self._done.clear()

    # -- scheduler -------------------------------------------------------------
    def _footprint(self, r):
        from . import api

        plan = api.get_plan(r.vol.shape, r.patch, r.stride, r.form, device=self.device,
                            **self._tuned(r))
        return plan, 2 * r.vol.nbytes + 4 * r.n_patches + plan.workspace_bytes + (1 << 20)

    def _tuned(self, r):
        if not self.autotune:
            return {}
        from .tune import tune

        return tune(r.vol.shape, r.patch, r.stride, r.form, self.device)

    def _fits(self, need):
        free, _ = self.torch.cuda.mem_get_info(self.device)
        # pooled device buffers are reused first; torch's cache is reusable too
        cached = self.torch.cuda.memory_reserved(self.device) - self.torch.cuda.memory_allocated(self.device)
        avail = free + cached + self._pool.free_bytes - self.reserve
        if need > avail and self._pool.free_bytes:
            self._pool.trim()  # give the pooled buffers back before refusing
            self.torch.cuda.empty_cache()
            free, _ = self.torch.cuda.mem_get_info(self.device)
            avail = free - self.reserve
        if need > avail:
            return False
        if self.budget is not None and self._in_flight_bytes + need > self.budget:
            return False
        return True

    def _admit(self):
        torch = self.torch
        while self._free_slots and self._pending:
            r = self._pending[0]
            try:
                plan, need = self._footprint(r)
            except Exception as e:  # invalid problem: fail this request only
                self._pending.popleft()
                r.future.set_exception(e)
                continue
            if not self._fits(need):
                if not self._running:  # nothing will free memory: fail instead of waiting forever
                    self._pending.popleft()
                    r.future.set_exception(MemoryError(
                        f"request needs {need} device bytes; not available even with the GPU idle"))
                    continue
                return
            self._pending.popleft()
            slot = self._free_slots.pop()
            r.slot, r.need, r.t_start = slot, need, time.perf_counter()
            self._in_flight_bytes += need
            st = self._streams[slot]
            dev = f"cuda:{self.device}"
            r.h_in = torch.from_numpy(r.vol).pin_memory()
            with torch.cuda.device(self.device), torch.cuda.stream(st):
                h_in = r.h_in
                vbytes, rbytes = r.vol.nbytes, 4 * r.n_patches
                raw = {k: self._pool.take(k, n) for k, n in (("d_in", vbytes), ("d_out", vbytes),
                                                           ("d_rank", rbytes), ("ws", max(plan.workspace_bytes, 1)))}
                d_in = raw["d_in"][:vbytes].view(torch.float32).view(r.vol.shape)
                d_out = raw["d_out"][:vbytes].view(torch.float32).view(r.vol.shape)
                d_rank = raw["d_rank"][:rbytes].view(torch.int32)
                # the result's pinned buffers go to the caller (torch's host allocator caches them)
                h_out = torch.empty(r.vol.shape, dtype=torch.float32, pin_memory=True)
                h_rank = torch.empty(r.n_patches, dtype=torch.int32, pin_memory=True)
                d_in.copy_(h_in, non_blocking=True)
                plan.denoise(d_in.data_ptr(), d_out.data_ptr(), d_rank.data_ptr(), raw["ws"].data_ptr(),
                             st.cuda_stream)
                h_out.copy_(d_out, non_blocking=True)
                h_rank.copy_(d_rank, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(st)
            r.bufs = dict(h_in=h_in, raw=raw, h_out=h_out, h_rank=h_rank, plan=plan)
            r.event = ev
            self._running[id(r)] = r

    def _complete(self):
        for key in list(self._running):
            r = self._running[key]
            if not r.event.query():
                continue
            del self._running[key]
            t_done = time.perf_counter()
            out = r.bufs["h_out"].numpy()
            ranks = r.bufs["h_rank"].numpy()
            for k, t in r.bufs["raw"].items():
                self._pool.give(k, t)
            r.bufs = {}
            r.h_in = None
            self._free_slots.append(r.slot)
            self._in_flight_bytes -= r.need
            self._done.append((r.t_submit, r.t_start, t_done, r.n_patches, r.vol.shape))
            r.future.set_result((out, ranks))

    def _loop(self):
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            with self._lock:
                if self._stop and not self._pending and not self._running:
                    return
                if not self._pending and not self._running:
                    self._lock.wait(timeout=0.05)
                    continue
                self._complete()
                self._admit()
            time.sleep(self.poll_s)


def poisson_arrivals(rate_per_s, duration_s, seed=0, max_count=None):
    """Arrival times (s) of a Poisson process, seeded: those before
    ``duration_s``, at most ``max_count`` of them."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while max_count is None or len(out) < max_count:
        t += rng.exponential(1.0 / rate_per_s)
        if t >= duration_s:
            break
        out.append(t)
    return np.array(out)


def draw_request_shapes(n, seed=0, big_fraction=0.1, t_choices=(32, 48, 64, 96)):
    """Request mix of the serving workload: volumes with x, y in 64..128,
    z in 32..64, T in {32, 48, 64, 96}, patch in {5^3, 7^3, 11^3}, stride in
    {1, 2, 3}, sigma in [0.02, 0.1]; a ``big_fraction`` of 128x128x64x96
    volumes with 11^3 patches at stride 2."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        if rng.uniform() < big_fraction:
            out.append(dict(shape=(128, 128, 64, 96), patch=(11, 11, 11), stride=2, sigma=0.05))
            continue
        x, y = (int(v) for v in rng.integers(64, 129, size=2))
        z = int(rng.integers(32, 65))
        T = int(rng.choice(t_choices))
        p = int(rng.choice([5, 7, 11]))
        s = int(rng.choice([1, 2, 3]))
        while p ** 3 < T:  # the Gram route needs at least T voxels per patch
            p += 2
        out.append(dict(shape=(x, y, z, T), patch=(p, p, p), stride=s, sigma=float(rng.uniform(0.02, 0.1))))
    return out
