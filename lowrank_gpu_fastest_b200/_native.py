"""ctypes binding of ``liblrd.so`` (declarations in include/lrd.h).

The library is the only compute path: if it is missing or fails to load, every
entry point raises - there is no CPU or PyTorch fallback.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblrd.so")

LRD_OK = 0
LRD_ERR_INVALID = -1
LRD_ERR_NOMEM = -2
LRD_ERR_CUDA = -3
LRD_ERR_UNSUPPORTED = -4
LRD_ERR_NODEVICE = -5
LRD_ERR_TIMEOUT = -6

FORMS = {"plain": 0, "accurate": 1, "tensor": 2, "tensor_bf16": 3}

# Every symbol include/lrd.h declares, with (restype, argtypes).
_c_i32p = ctypes.POINTER(ctypes.c_int32)
_c_f32p = ctypes.c_void_p
SIGNATURES = {
    "lrd_version": (ctypes.c_int, []),
    "lrd_last_error_string": (ctypes.c_char_p, []),
    "lrd_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "lrd_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "lrd_plan_num_patches": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "lrd_workspace_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]),
    "lrd_denoise": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 5),
    "lrd_denoise_host": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 8),
    "lrd_stage_gram": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 4),
    "lrd_stage_eigh": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 6),
    "lrd_plan_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "lrd_plan_phase_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_int32)]),
    "lrd_denoise_static": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "lrd_batch_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.POINTER(ctypes.c_void_p)]),
    "lrd_batch_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "lrd_batch_workspace_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]),
    "lrd_batch_num_launches": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "lrd_batch_denoise": (ctypes.c_int, [ctypes.c_void_p] * 6 + [ctypes.c_int32]),
    "lrd_workspace_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.c_void_p]),
    "lrd_slab_partition": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, _c_i32p]),
    "lrd_slab_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "lrd_slab_info": (ctypes.c_int, [ctypes.c_void_p, _c_i32p]),
    "lrd_noise_map": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "lrd_slab_prepare": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "lrd_slab_recon": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "lrd_selftest_wait_timeout": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]),
}
SLAB_HALO_OUT, SLAB_INTERIOR, SLAB_HALO_IN = 0, 1, 2
PHASES = ("center", "gram", "eigh_mp", "recon")


class LrdProblem(ctypes.Structure):
    """``struct lrd_problem`` (include/lrd.h)."""

    _fields_ = [(n, ctypes.c_int32) for n in
                ("nx", "ny", "nz", "nt", "px", "py", "pz", "stride", "form", "batch",
                 "brick_x", "brick_y", "brick_z", "recon_split", "gram_split", "eigh_block")]


class LrdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lrd error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def load(path: str | None = None):
    """Load (once) and return the native library. Raises if it is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise ImportError(
                f"{p} not found: build it with `python -m lowrank_gpu_fastest_b200.build` "
                "(the CUDA library is the only compute path)")
        lib = ctypes.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc: int):
    if rc != LRD_OK:
        msg = load().lrd_last_error_string().decode(errors="replace")
        raise LrdError(rc, msg)


def make_problem(shape, patch=(11, 11, 11), stride=3, form="plain", batch=0, brick=None, split=0, gram_split=0,
                 eigh_block=0):
    if form not in FORMS:
        raise ValueError(f"form must be one of {sorted(FORMS)}, got {form!r}")
    nx, ny, nz, nt = (int(s) for s in shape)
    px, py, pz = (int(p) for p in patch)
    bx, by, bz = (int(b) for b in (brick or (0, 0, 0)))
    return LrdProblem(nx, ny, nz, nt, px, py, pz, int(stride), FORMS[form], int(batch or 0),
                      bx, by, bz, int(split or 0), int(gram_split or 0), int(eigh_block or 0))


def selftest_wait_timeout(limit_ns: int, d_status: int, stream: int):
    """Run the bounded-wait self-test: a kernel waits on a device barrier that
    nothing completes and records LRD_STATUS_TMA_TIMEOUT (1) in the int32 at
    ``d_status`` after ``limit_ns`` ns (asynchronous on ``stream``)."""
    check(load().lrd_selftest_wait_timeout(int(limit_ns), d_status, stream))


def slab_partition(shape, patch, stride, n_slabs):
    """Per slab ``(first corner, end corner, x0, x1)`` (``lrd_slab_partition``;
    host-only, no device needed)."""
    pr = make_problem(shape, patch, stride)
    b = (ctypes.c_int32 * (4 * int(n_slabs)))()
    check(load().lrd_slab_partition(ctypes.byref(pr), int(n_slabs), b))
    v = list(b)
    return [tuple(v[4 * r:4 * r + 4]) for r in range(int(n_slabs))]


class Plan:
    """Owns an ``lrd_plan*`` for one problem on the current CUDA device."""

    def __init__(self, shape, patch=(11, 11, 11), stride=3, form="plain", batch=0, brick=None, split=0,
                 _slab=None, gram_split=0, eigh_block=0):
        lib = load()
        self.problem = make_problem(shape, patch, stride, form, batch, brick, split, gram_split, eigh_block)
        nx, ny, nz, nt = (int(s) for s in shape)
        self.shape = (nx, ny, nz, nt)
        self.patch = tuple(int(p) for p in patch)
        self.stride = int(stride)
        self.form = form
        h = ctypes.c_void_p()
        if _slab is None:
            check(lib.lrd_plan_create(ctypes.byref(self.problem), ctypes.byref(h)))
        else:
            check(lib.lrd_slab_plan_create(ctypes.byref(self.problem), int(_slab[1]), int(_slab[0]),
                                           ctypes.byref(h)))
        self.handle = h
        n = ctypes.c_int64()
        check(lib.lrd_plan_num_patches(h, ctypes.byref(n)))
        self.n_patches = int(n.value)
        ws = ctypes.c_size_t()
        check(lib.lrd_workspace_size(h, ctypes.byref(ws)))
        self.workspace_bytes = int(ws.value)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                load().lrd_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    def denoise(self, d_vol: int, d_out: int, d_ranks: int | None, d_ws: int, stream: int):
        check(load().lrd_denoise(self.handle, d_vol, d_out, d_ranks, d_ws, stream))

    def denoise_host(self, h_vol, h_out, h_ranks, d_in, d_out, d_ranks, d_ws, stream):
        check(load().lrd_denoise_host(self.handle, h_vol, h_out, h_ranks, d_in, d_out, d_ranks, d_ws,
                                      stream))

    def status(self, d_ws: int, stream: int) -> int:
        """Device status word of the last call on this workspace (syncs the stream)."""
        st = ctypes.c_int32()
        check(load().lrd_workspace_status(self.handle, d_ws, ctypes.byref(st), stream))
        return int(st.value)

    def set_profiling(self, enable: bool):
        check(load().lrd_plan_set_profiling(self.handle, int(bool(enable))))

    def phase_ms(self):
        """Summed ms per phase and call count since the last read (clears)."""
        ms = (ctypes.c_float * len(PHASES))()
        n = ctypes.c_int32()
        check(load().lrd_plan_phase_ms(self.handle, ms, ctypes.byref(n)))
        return dict(zip(PHASES, list(ms))), int(n.value)

    def noise_map(self, d_ws, d_sigma2, d_noise, stream):
        """Per-patch noise variance estimates and/or the voxel noise map of
        the last denoise on ``d_ws`` (either pointer may be None)."""
        check(load().lrd_noise_map(self.handle, d_ws, d_sigma2, d_noise, stream))

    def stage_gram(self, d_vol, d_gram, d_ws, stream):
        check(load().lrd_stage_gram(self.handle, d_vol, d_gram, d_ws, stream))

    def stage_eigh(self, d_gram, d_lam, d_vecs, d_ranks, d_ws, stream):
        check(load().lrd_stage_eigh(self.handle, d_gram, d_lam, d_vecs, d_ranks, d_ws, stream))


class SlabPlan(Plan):
    """Plan of slab ``slab`` of ``n_slabs`` of a volume of ``shape`` (global)."""

    def __init__(self, shape, slab, n_slabs, patch=(11, 11, 11), stride=3, form="plain", brick=None, split=0):
        super().__init__(shape, patch, stride, form, 0, brick, split, _slab=(slab, n_slabs))
        info = (ctypes.c_int32 * 8)()
        check(load().lrd_slab_info(self.handle, info))
        (self.x0, self.nx, self.hin, self.own_hi, self.ci_lo, self.ci_hi, self.slab,
         self.n_slabs) = (int(v) for v in info)
        self.global_shape = self.shape
        self.shape = (self.nx,) + self.global_shape[1:]

    def prepare(self, d_vol, d_ranks, d_ws, stream):
        check(load().lrd_slab_prepare(self.handle, d_vol, d_ranks, d_ws, stream))

    def recon(self, part, d_out, d_ws, d_halo_in, d_halo_out, stream):
        check(load().lrd_slab_recon(self.handle, d_out, d_ws, int(part), d_halo_in, d_halo_out, stream))


class BatchPlan:
    """Owns an ``lrd_batch_plan*``: many problems in packed launches (one grid
    per phase and kernel class), optionally one CUDA graph."""

    def __init__(self, problems, n_streams=4):
        """``problems``: list of dicts with shape, patch, stride, form, batch,
        brick, split, gram_split, eigh_block (all but shape optional)."""
        lib = load()
        arr = (LrdProblem * len(problems))()
        for i, pr in enumerate(problems):
            nx, ny, nz, nt = (int(v) for v in pr["shape"])
            px, py, pz = (int(v) for v in pr.get("patch", (11, 11, 11)))
            bx, by, bz = (int(v) for v in (pr.get("brick") or (0, 0, 0)))
            arr[i] = LrdProblem(nx, ny, nz, nt, px, py, pz, int(pr.get("stride", 3)),
                                FORMS[pr.get("form", "plain")], int(pr.get("batch") or 0), bx, by, bz,
                                int(pr.get("split") or 0), int(pr.get("gram_split") or 0),
                                int(pr.get("eigh_block") or 0))
        self._arr = arr
        self.n = len(problems)
        h = ctypes.c_void_p()
        check(lib.lrd_batch_plan_create(arr, self.n, int(n_streams), ctypes.byref(h)))
        self.handle = h
        ws = ctypes.c_size_t()
        check(lib.lrd_batch_workspace_size(h, ctypes.byref(ws)))
        self.workspace_bytes = int(ws.value)
        nl = ctypes.c_int32()
        check(lib.lrd_batch_num_launches(h, ctypes.byref(nl)))
        self.launches = int(nl.value)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                load().lrd_batch_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    def denoise(self, d_vols, d_outs, d_ranks, d_ws, stream, use_graph=True):
        vp = (ctypes.c_void_p * self.n)(*d_vols)
        op = (ctypes.c_void_p * self.n)(*d_outs)
        rp = (ctypes.c_void_p * self.n)(*d_ranks) if d_ranks is not None else None
        check(load().lrd_batch_denoise(self.handle, vp, op, rp, d_ws, stream, int(bool(use_graph))))
