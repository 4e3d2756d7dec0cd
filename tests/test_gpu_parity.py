"""Parity of the CUDA path (through the C ABI) with the step-0 oracle.

Bars: MP ranks bit-exact; plain form within 2e-7 relative L2 of the
reference's step-0 output; accurate form within 2e-7 (target 1e-7) of the
float64 run of the algorithm.
"""

import numpy as np
import pytest
import torch

from conftest import LARGE_CASES, SMALL_CASES, golden_input, load_golden
from lowrank_gpu_fastest_b200 import _native, api, rel_l2
from oracle import mppca as orc

pytestmark = pytest.mark.gpu

PLAIN_TOL = 2e-7          # relative L2 vs step 0 (plain form)
ACCURATE_TOL = 2e-7       # relative L2 vs the float64 oracle (accurate form)
ACCURATE_TOL_LARGE = 1e-7  # measured ~5e-8 at the 96x96x48x48 headline


def run_dev(vol, patch, stride, form="plain", batch=None):
    d = torch.from_numpy(vol).cuda()
    out, ranks = api.denoise(d, patch, stride, batch, form=form, return_ranks=True)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ranks.cpu().numpy()


@pytest.mark.parametrize("name", SMALL_CASES)
def test_small_plain_vs_step0(cuda_ok, name):
    g = load_golden(name)
    vol = golden_input(g)
    out, ranks = run_dev(vol, tuple(g["patch"]), int(g["stride"]))
    np.testing.assert_array_equal(ranks, g["ranks"])
    assert rel_l2(out, g["out"]) <= PLAIN_TOL


@pytest.mark.parametrize("form", ["accurate", "tensor", "tensor_bf16"])
@pytest.mark.parametrize("name", SMALL_CASES)
def test_small_accurate_vs_fp64(cuda_ok, name, form):
    g = load_golden(name)
    vol = golden_input(g)
    out, ranks = run_dev(vol, tuple(g["patch"]), int(g["stride"]), form=form)
    np.testing.assert_array_equal(ranks, g["ranks"])
    idx = g["sample_idx"]
    assert rel_l2(out.reshape(-1)[idx], g["out64_sample"]) <= ACCURATE_TOL


@pytest.mark.parametrize("name", LARGE_CASES)
def test_large_ranks_and_sample(cuda_ok, name):
    g = load_golden(name)
    vol = golden_input(g)
    out, ranks = run_dev(vol, tuple(g["patch"]), int(g["stride"]))
    np.testing.assert_array_equal(ranks, g["ranks"])
    idx = g["sample_idx"]
    assert rel_l2(out.reshape(-1)[idx], g["out_sample"]) <= PLAIN_TOL
    for form in ("accurate", "tensor", "tensor_bf16"):
        outa, ra = run_dev(vol, tuple(g["patch"]), int(g["stride"]), form=form)
        np.testing.assert_array_equal(ra, g["ranks"])
        assert rel_l2(outa.reshape(-1)[idx], g["out64_sample"]) <= ACCURATE_TOL_LARGE


def test_config1_full_volume_vs_live_oracle(cuda_ok):
    g = load_golden("config1_lowrank")
    vol = golden_input(g)
    ref, ref_ranks = orc.denoise(vol, (11, 11, 11), 3)
    out, ranks = run_dev(vol, (11, 11, 11), 3)
    np.testing.assert_array_equal(ranks, ref_ranks)
    assert rel_l2(out, ref) <= PLAIN_TOL


def test_headline_region_vs_region_oracle(cuda_ok):
    """A 9x9x9 box of the 96x96x48x48 volume against the step-0 loop run over
    exactly the patches touching the box (bit-for-bit the full loop there)."""
    g = load_golden("headline_ref")
    vol = golden_input(g)
    out, _ = run_dev(vol, (11, 11, 11), 3)
    lo, hi = (40, 17, 20), (49, 26, 29)
    box, _, _ = orc.denoise_region(vol, (11, 11, 11), 3, lo, hi)
    assert rel_l2(out[40:49, 17:26, 20:29], box) <= PLAIN_TOL


def test_deterministic_and_batch_invariant(cuda_ok):
    g = load_golden("lowrank_p5s2")
    vol = golden_input(g)
    a, ra = run_dev(vol, (5, 5, 5), 2)
    b, rb = run_dev(vol, (5, 5, 5), 2)
    c, rc = run_dev(vol, (5, 5, 5), 2, batch=7)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(ra, rc)


@pytest.mark.parametrize("form", ["plain", "tensor"])
@pytest.mark.parametrize("shape", [(96, 96, 48, 48), (48, 48, 24, 48)])
def test_column_cut_is_bit_identical(cuda_ok, shape, form):
    """A Gram launch whose last wave holds a few whole patch columns cuts them
    into window ranges; launches of 100 columns (batch = 100 columns of
    patches) are never cut. Both give the same output and ranks bit for bit."""
    from lowrank_gpu_fastest_b200 import make_phantom_lowrank
    vol = make_phantom_lowrank(shape, seed=5)[0]
    ncz = len(orc.axis_corners(shape[2], 11, 3))
    a, ra = run_dev(vol, (11, 11, 11), 3, form=form)
    b, rb = run_dev(vol, (11, 11, 11), 3, form=form, batch=100 * ncz)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(ra, rb)


def test_host_api_matches_device_api(cuda_ok):
    g = load_golden("ref_small")
    vol = golden_input(g)
    host = api.denoise(vol, (11, 11, 11), 3)
    assert isinstance(host, np.ndarray)
    dev, _ = run_dev(vol, (11, 11, 11), 3)
    np.testing.assert_array_equal(host, dev)


def test_constant_volume_is_fixed_point(cuda_ok):
    vol = np.full((9, 8, 10, 20), 2.5, dtype=np.float32)
    out, ranks = run_dev(vol, (5, 5, 5), 2)
    assert (ranks == 0).all()
    ref, _ = orc.denoise(vol, (5, 5, 5), 2)
    np.testing.assert_array_equal(out, ref)


def test_uncovered_voxels_follow_ladder(cuda_ok):
    """stride > patch side leaves voxels no patch covers: 0 / max(0, 1e-12) = 0."""
    rng = np.random.default_rng(3)
    vol = (rng.standard_normal((14, 12, 13, 24)) + 5).astype(np.float32)
    ref, rref = orc.denoise(vol, (5, 5, 5), 7)
    out, ranks = run_dev(vol, (5, 5, 5), 7)
    np.testing.assert_array_equal(ranks, rref)
    assert rel_l2(out, ref) <= PLAIN_TOL
    outa, _ = run_dev(vol, (5, 5, 5), 7, form="accurate")
    np.testing.assert_array_equal(outa[5:7], 0.0)


def test_stage_gram_and_eigh_vs_fp64_oracle(cuda_ok):
    g = load_golden("lowrank_p5s2")
    vol = golden_input(g)
    shape, patch, stride = vol.shape, (5, 5, 5), 2
    plan = api.get_plan(shape, patch, stride)
    T, P = shape[3], plan.n_patches
    d = torch.from_numpy(vol).cuda()
    ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device="cuda")
    gram = torch.empty(P, T, T, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    plan.stage_gram(d.data_ptr(), gram.data_ptr(), ws.data_ptr(), s)
    lam = torch.empty(P, T, device="cuda")
    vecs = torch.zeros(P, T, T, device="cuda")
    ranks = torch.empty(P, dtype=torch.int32, device="cuda")
    plan.stage_eigh(gram.data_ptr(), lam.data_ptr(), vecs.data_ptr(), ranks.data_ptr(), ws.data_ptr(), s)
    torch.cuda.synchronize()
    gram, lam, vecs, ranks = (t.cpu().numpy() for t in (gram, lam, vecs, ranks))
    corners = orc.patch_corners(shape, patch, stride)
    for idx in range(0, P, 13):
        i, j, k = corners[idx]
        x = vol[i:i + 5, j:j + 5, k:k + 5].reshape(-1, T)
        st = orc.gram_route_patch(x)
        gscale = np.abs(st["G"]).max()
        assert np.abs(gram[idx] - st["G"]).max() <= 1e-5 * gscale
        # eigenvalues of our own Gram, to float32 round-off of its norm
        lam_ref = np.linalg.eigvalsh(gram[idx].astype(np.float64))
        assert np.abs(lam[idx] - lam_ref).max() <= 1e-5 * np.abs(lam_ref).max()
        p = int(ranks[idx])
        assert p == st["p"]
        V = vecs[idx].reshape(-1)[: T * p].reshape(p, T).T.astype(np.float64)
        np.testing.assert_allclose(V.T @ V, np.eye(p), atol=1e-5)
        assert np.abs(V @ V.T - st["P"]).max() <= 1e-4


def test_error_is_raised_for_bad_shapes(cuda_ok):
    with pytest.raises(_native.LrdError):
        api.denoise(torch.zeros(4, 4, 4, 8, device="cuda"), (5, 5, 5), 2)


@pytest.mark.parametrize("form", ["tensor", "tensor_bf16"])
@pytest.mark.parametrize("name", ["lowrank_p5s2", "ref_small", "lowrank_t64", "aniso"])
def test_tensor_core_gram_vs_fp64(cuda_ok, name, form):
    """The tcgen05 Grams (3xTF32 and 3-term BF16 split products) against
    float64 Grams of the same centred patches: within 4e-6 of the largest
    entry (FP32 FFMA: ~1e-6)."""
    g = load_golden(name)
    vol = golden_input(g)
    shape, patch, stride = vol.shape, tuple(int(v) for v in g["patch"]), int(g["stride"])
    plan = api.get_plan(shape, patch, stride, form=form)
    T, P = shape[3], plan.n_patches
    d = torch.from_numpy(vol).cuda()
    ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device="cuda")
    gram = torch.empty(P, T, T, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    plan.stage_gram(d.data_ptr(), gram.data_ptr(), ws.data_ptr(), s)
    assert plan.status(ws.data_ptr(), s) == 0
    gram = gram.cpu().numpy()
    corners = orc.patch_corners(shape, patch, stride)
    for idx in range(0, P, max(1, P // 25)):
        i, j, k = corners[idx]
        x = vol[i:i + patch[0], j:j + patch[1], k:k + patch[2]].reshape(-1, T).astype(np.float64)
        xc = x - x.mean(1, keepdims=True)
        G = xc.T @ xc
        assert np.abs(gram[idx] - G).max() <= 4e-6 * np.abs(G).max()


def test_bounded_wait_gives_up_and_reports(cuda_ok):
    """The device-wait failure path without a GPU fault: a kernel waits on a
    barrier that nothing completes, gives up after 20 ms and sets the timeout
    bit; the context stays usable (a denoise afterwards equals one before)."""
    import time

    g = load_golden("lowrank_p5s2")
    vol = golden_input(g)
    before, rb = run_dev(vol, (5, 5, 5), 2)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _native.selftest_wait_timeout(20_000_000, st.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert int(st.item()) == 1  # LRD_STATUS_TMA_TIMEOUT
    assert 0.015 <= dt < 5.0
    after, ra = run_dev(vol, (5, 5, 5), 2)
    np.testing.assert_array_equal(before, after)
    np.testing.assert_array_equal(rb, ra)


def test_status_word_clear_after_runs(cuda_ok):
    g = load_golden("ref_small")
    vol = torch.from_numpy(golden_input(g)).cuda()
    for form in ("plain", "tensor", "tensor_bf16"):
        plan = api.get_plan(tuple(vol.shape), (11, 11, 11), 3, form=form)
        ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device="cuda")
        out = torch.empty_like(vol)
        s = torch.cuda.current_stream().cuda_stream
        plan.denoise(vol.data_ptr(), out.data_ptr(), None, ws.data_ptr(), s)
        assert plan.status(ws.data_ptr(), s) == 0


@pytest.mark.parametrize("form", ["plain", "tensor"])
@pytest.mark.parametrize("name", ["headline_ref", "aniso", "lowrank_t96"])
def test_pipelined_host_call_equals_device_call(cuda_ok, name, form):
    """lrd_denoise_host (x-slab copy/compute pipeline) gives the device path's
    output and ranks bit for bit."""
    g = load_golden(name)
    vol = golden_input(g)
    patch, stride = tuple(int(v) for v in g["patch"]), int(g["stride"])
    host, hr = api.denoise(vol, patch, stride, form=form, return_ranks=True)
    dev, dr = run_dev(vol, patch, stride, form=form)
    np.testing.assert_array_equal(host, dev)
    np.testing.assert_array_equal(hr, dr)


@pytest.mark.parametrize("shape,patch,stride", [
    ((16, 14, 12, 96), (7, 7, 7), 2),   # one CTA per matrix, 96 threads
    ((14, 12, 12, 128), (7, 7, 7), 2),  # 128 threads
    ((13, 12, 11, 80), (5, 6, 5), 2),   # T between the kernels' sizes
])
def test_long_series_vs_live_oracle(cuda_ok, shape, patch, stride):
    """T > 64 (block eigensolver, block float64 near-tie pass) against the
    step-0 loop run live: ranks exact, plain within the step-0 bar, accurate
    within the float64 bar."""
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    vol = make_phantom_lowrank(shape, seed=11)[0]
    ref, ref_ranks = orc.denoise(vol, patch, stride)
    out, ranks = run_dev(vol, patch, stride)
    np.testing.assert_array_equal(ranks, ref_ranks)
    assert rel_l2(out, ref) <= PLAIN_TOL
    ref64, _ = orc.denoise_fp64(vol, patch, stride)
    outa, ra = run_dev(vol, patch, stride, form="accurate")
    np.testing.assert_array_equal(ra, ref_ranks)
    assert rel_l2(outa, ref64) <= ACCURATE_TOL


@pytest.mark.parametrize("T", [48, 96, 128])
def test_stage_eigenvalues_vs_float64(cuda_ok, T):
    """The eigensolve stage's eigenvalues of each patch's Gram matrix against
    numpy's float64 eigvalsh of the same (device-formed) matrix."""
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    shape, patch, stride = (12, 12, 10, T), (7, 7, 5), 3
    vol = torch.from_numpy(make_phantom_lowrank(shape, seed=2)[0]).cuda()
    plan = api.get_plan(shape, patch, stride)
    P = plan.n_patches
    ws = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device="cuda")
    gram = torch.empty((P, T, T), dtype=torch.float32, device="cuda")
    vecs = torch.empty_like(gram)
    lam = torch.empty((P, T), dtype=torch.float32, device="cuda")
    rk = torch.empty(P, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    plan.stage_gram(vol.data_ptr(), gram.data_ptr(), ws.data_ptr(), s)
    plan.stage_eigh(gram.data_ptr(), lam.data_ptr(), vecs.data_ptr(), rk.data_ptr(), ws.data_ptr(), s)
    torch.cuda.synchronize()
    g64 = gram.double().cpu().numpy()
    ref = np.linalg.eigvalsh(g64)
    got = lam.cpu().numpy().astype(np.float64)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.abs(got - ref).max() / scale.max() < 2e-6
    # the top eigenvectors returned as rows: unit norm, G v = lambda v
    v = vecs.cpu().numpy()
    rks = rk.cpu().numpy()
    for i in range(0, P, max(1, P // 8)):
        for q in range(rks[i]):
            x = v[i, q].astype(np.float64)
            assert abs(np.linalg.norm(x) - 1) < 1e-5
            lq = ref[i, T - 1 - q]
            assert np.linalg.norm(g64[i] @ x - lq * x) <= 1e-5 * scale[i, 0]


@pytest.mark.parametrize("name", ["ref_small", "lowrank_p5s2", "lowrank_t64", "lowrank_t96", "aniso"])
def test_noise_estimates_vs_oracle(cuda_ok, name):
    """Per-patch MP noise variance estimates and the voxel noise map against
    the oracle (its SVD eigenvalues differ from the Gram route's in the last
    float32 bits, relative to the largest eigenvalue)."""
    from lowrank_gpu_fastest_b200 import denoise_with_noise

    g = load_golden(name)
    vol = golden_input(g)
    patch, stride = tuple(int(v) for v in g["patch"]), int(g["stride"])
    res = denoise_with_noise(vol, patch, stride)
    ranks, sig2, nmap = orc.noise_map(vol, patch, stride)
    np.testing.assert_array_equal(res["ranks"], g["ranks"])
    np.testing.assert_array_equal(res["ranks"], ranks)
    assert np.abs(res["sigma2"] - sig2).max() <= 1e-3 * np.abs(sig2).max()
    assert rel_l2(res["noise"], nmap) <= 1e-3
    plain, _ = run_dev(vol, patch, stride)
    np.testing.assert_array_equal(res["out"], plain)


def test_host_pipeline_with_patch_batches(cuda_ok):
    """The ladder's BATCH (patches per Gram / eigensolver launch) through the
    pipelined host call equals the device call without batching."""
    g = load_golden("lowrank_p5s2")
    vol = golden_input(g)
    host, hr = api.denoise(vol, (5, 5, 5), 2, batch=23, return_ranks=True)
    dev, dr = run_dev(vol, (5, 5, 5), 2)
    np.testing.assert_array_equal(hr, dr)
    np.testing.assert_array_equal(host, dev)


@pytest.mark.parametrize("T", [30, 37, 101])
def test_frame_counts_off_the_column_kernel(cuda_ok, T):
    """T not a multiple of 4 takes the per-patch Gram kernel (the column and
    tensor Grams need T % 4 == 0); against the live step-0 loop."""
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    shape, patch, stride = (12, 11, 10, T), (5, 5, 5), 2
    vol = make_phantom_lowrank(shape, seed=4)[0]
    ref, ref_ranks = orc.denoise(vol, patch, stride)
    for form in ("plain", "accurate", "tensor"):
        out, ranks = run_dev(vol, patch, stride, form=form)
        np.testing.assert_array_equal(ranks, ref_ranks)
        tol = PLAIN_TOL if form == "plain" else 4e-7  # accurate/tensor follow float64, step 0 is ~2e-7 away
        assert rel_l2(out, ref) <= tol, (form, rel_l2(out, ref))


@pytest.mark.parametrize("T", [2, 3, 5, 8])
def test_few_frames_vs_live_oracle(cuda_ok, T):
    """The shortest series (one to seven non-null eigenvalues) against the
    live step-0 loop."""
    rng = np.random.default_rng(T)
    vol = (rng.standard_normal((9, 8, 7, T)) * 0.1 + np.linspace(0, 1, T)).astype(np.float32)
    patch, stride = (3, 3, 3), 2
    ref, ref_ranks = orc.denoise(vol, patch, stride)
    for form in ("plain", "accurate"):
        out, ranks = run_dev(vol, patch, stride, form=form)
        np.testing.assert_array_equal(ranks, ref_ranks)
        tol = PLAIN_TOL if form == "plain" else 4e-7
        assert rel_l2(out, ref) <= tol, (form, rel_l2(out, ref))
