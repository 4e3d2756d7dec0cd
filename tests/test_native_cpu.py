"""The C-ABI library builds for sm_100a, loads, and exports every declared symbol.

No compute call runs here (no GPU in this container); host-side argument
checks that return before touching the device are exercised.
"""

import ctypes
import os
import re

import pytest

from lowrank_gpu_fastest_b200 import _native, build

HEADER = os.path.join(os.path.dirname(build.HERE), "include", "lrd.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(lrd_\w+)\s*\(", txt, re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _native.load()


def test_header_and_binding_agree():
    syms = declared_symbols()
    assert "lrd_denoise" in syms and "lrd_plan_create" in syms
    assert set(syms) == set(_native.SIGNATURES), set(syms) ^ set(_native.SIGNATURES)


def test_library_exports_every_declared_symbol(lib):
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert lib.lrd_version() == 1


def test_null_arguments_rejected(lib):
    h = ctypes.c_void_p()
    assert lib.lrd_plan_create(None, ctypes.byref(h)) == _native.LRD_ERR_INVALID
    assert b"NULL" in lib.lrd_last_error_string()
    assert lib.lrd_denoise(None, None, None, None, None, None) == _native.LRD_ERR_INVALID
    assert lib.lrd_plan_destroy(None) == _native.LRD_OK


@pytest.mark.parametrize("fields,code", [
    ((10, 10, 10, 48, 11, 11, 11, 3, 0, 0), _native.LRD_ERR_INVALID),   # patch > volume
    ((16, 16, 16, 1, 5, 5, 5, 2, 0, 0), _native.LRD_ERR_INVALID),      # one frame
    ((16, 16, 16, 48, 5, 5, 5, 0, 0, 0), _native.LRD_ERR_INVALID),     # stride 0
    ((16, 16, 16, 48, 5, 5, 5, 2, 7, 0), _native.LRD_ERR_INVALID),     # unknown form
    ((16, 16, 16, 48, 5, 5, 5, 2, 0, -1), _native.LRD_ERR_INVALID),    # negative batch
    ((16, 16, 16, 200, 7, 7, 7, 2, 0, 0), _native.LRD_ERR_UNSUPPORTED),  # T above the compiled limit
    ((16, 16, 16, 48, 3, 3, 3, 2, 0, 0), _native.LRD_ERR_UNSUPPORTED),   # N = 27 < T
    ((16, 16, 16, 48, 5, 5, 5, 2, 0, 0, 0, 0, 0, 0, 3, 0), _native.LRD_ERR_INVALID),  # Gram split 3
    ((16, 16, 16, 48, 5, 5, 5, 2, 0, 0, 0, 0, 0, 0, 0, 3), _native.LRD_ERR_INVALID),  # eigh_block 3
    ((16, 16, 16, 80, 7, 7, 7, 2, 0, 0, 0, 0, 0, 0, 0, 1), _native.LRD_ERR_INVALID),  # warp per matrix at T = 80
])
def test_invalid_problems_rejected_before_device(lib, fields, code):
    pr = _native.LrdProblem(*fields)
    h = ctypes.c_void_p()
    assert lib.lrd_plan_create(ctypes.byref(pr), ctypes.byref(h)) == code
    assert not h.value
    assert lib.lrd_last_error_string()


def test_valid_problem_without_device_reports_nodevice(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    pr = _native.LrdProblem(48, 48, 24, 48, 11, 11, 11, 3, 0, 0)
    h = ctypes.c_void_p()
    assert lib.lrd_plan_create(ctypes.byref(pr), ctypes.byref(h)) == _native.LRD_ERR_NODEVICE


def test_selftest_wait_timeout_checks_arguments(lib):
    """Bad arguments are rejected on the host, before any device work."""
    assert lib.lrd_selftest_wait_timeout(10_000_000, None, None) == _native.LRD_ERR_INVALID
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the limit check fails first
    assert lib.lrd_selftest_wait_timeout(10, fake, None) == _native.LRD_ERR_INVALID
    assert lib.lrd_selftest_wait_timeout(20_000_000_000, fake, None) == _native.LRD_ERR_INVALID
    assert b"limit_ns" in lib.lrd_last_error_string()
