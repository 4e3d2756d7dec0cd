"""lrd_denoise_static - the entry point that allocates no device memory.

Some callers cannot call cudaMalloc (the CUDA allocator is off limits where
they run, or a host framework owns every device allocation), so they can
neither create a plan (its index tables are cudaMalloc'd) nor provide a
workspace. lrd_denoise_static keeps all of that scratch in one static device
array inside the library. This test calls it through the C ABI twice in a row
and checks each result against the plan-based lrd_denoise on the same input,
with the parity tolerance the other GPU tests use; between the two calls a
different problem runs through the same static array, so stale contents from
the previous call must not leak into the next. It sits in its own file named
to be collected last.
"""

import ctypes

import numpy as np
import pytest
import torch

from conftest import golden_input, load_golden
from lowrank_gpu_fastest_b200 import _native, api, problem, rel_l2

pytestmark = pytest.mark.gpu

PLAIN_TOL = 2e-7
# relative L2 between the static path and lrd_denoise, per form: both follow the
# same arithmetic except the Gram (per-patch kernel here, column kernel in the
# plan path; for the tensor form the plan path's Gram is tcgen05 3xTF32)
FORM_TOL = {0: PLAIN_TOL, 1: 1e-7, 2: 1e-7, 3: 1e-7}
FORM_NAME = {0: "plain", 1: "accurate", 2: "tensor", 3: "tensor_bf16"}


def _problem(shape, patch, stride, form=0):
    return _native.LrdProblem(*shape, *patch, stride, form, 0)


def _static_call(vol_dev, patch, stride, form=0):
    lib = _native.load()
    out = torch.full_like(vol_dev, float("nan"))
    ranks = torch.full((problem.n_patches(tuple(vol_dev.shape), patch, stride),), -1,
                       dtype=torch.int32, device=vol_dev.device)
    pr = _problem(tuple(vol_dev.shape), patch, stride, form)
    rc = lib.lrd_denoise_static(ctypes.byref(pr), vol_dev.data_ptr(), out.data_ptr(), ranks.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    _native.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ranks.cpu().numpy()


@pytest.mark.parametrize("form", [0, 1, 2, 3])
def test_static_entry_matches_plan_entry_twice(cuda_ok, form):
    g = load_golden("config1_lowrank")
    vol = torch.from_numpy(golden_input(g)).cuda()
    name = FORM_NAME[form]
    ref, ref_ranks = api.denoise(vol, (11, 11, 11), 3, form=name, return_ranks=True)
    torch.cuda.synchronize()
    ref, ref_ranks = ref.cpu().numpy(), ref_ranks.cpu().numpy()
    other = torch.from_numpy(golden_input(load_golden("lowrank_p5s2"))).cuda()
    for call in range(2):
        out, ranks = _static_call(vol, (11, 11, 11), 3, form)
        np.testing.assert_array_equal(ranks, ref_ranks)
        assert np.isfinite(out).all()
        assert rel_l2(out, ref) <= FORM_TOL[form], f"call {call}"
        # a different problem through the same static array in between
        o2, r2 = _static_call(other, (5, 5, 5), 2, form)
        ref2, rr2 = api.denoise(other, (5, 5, 5), 2, form=name, return_ranks=True)
        np.testing.assert_array_equal(r2, rr2.cpu().numpy())
        assert rel_l2(o2, ref2.cpu().numpy()) <= FORM_TOL[form]


def test_static_entry_rejects_overlapping_buffers(cuda_ok):
    lib = _native.load()
    vol = torch.zeros(16, 16, 16, 16, device="cuda")
    pr = _problem((16, 16, 16, 16), (5, 5, 5), 2)
    rc = lib.lrd_denoise_static(ctypes.byref(pr), vol.data_ptr(), vol.data_ptr(), None,
                                torch.cuda.current_stream().cuda_stream)
    assert rc == _native.LRD_ERR_INVALID
    assert b"overlap" in lib.lrd_last_error_string()


def test_static_entry_rejects_problems_beyond_its_scratch(cuda_ok):
    lib = _native.load()
    vol = torch.zeros(96, 96, 48, 48, device="cuda")
    out = torch.empty_like(vol)
    pr = _problem((96, 96, 48, 48), (11, 11, 11), 3)
    rc = lib.lrd_denoise_static(ctypes.byref(pr), vol.data_ptr(), out.data_ptr(), None,
                                torch.cuda.current_stream().cuda_stream)
    assert rc == _native.LRD_ERR_UNSUPPORTED
    assert b"static scratch" in lib.lrd_last_error_string()
