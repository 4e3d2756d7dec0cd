"""The CPU oracle against the golden vectors made by the reference's own step 0."""

import hashlib

import numpy as np
import pytest

from conftest import LARGE_CASES, SMALL_CASES, golden_input, load_golden
from oracle import mppca as orc
from lowrank_gpu_fastest_b200 import problem


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", SMALL_CASES + LARGE_CASES)
def test_golden_inputs_regenerate(name):
    g = load_golden(name)
    assert sha(golden_input(g)) == str(g["input_sha256"])


@pytest.mark.parametrize("name", SMALL_CASES)
def test_oracle_matches_reference_step0_bitwise(name):
    g = load_golden(name)
    vol = golden_input(g)
    out, ranks = orc.denoise(vol, tuple(g["patch"]), int(g["stride"]))
    np.testing.assert_array_equal(ranks, g["ranks"])
    np.testing.assert_array_equal(out, g["out"])


@pytest.mark.parametrize("name", ["lowrank_p5s2", "aniso"])
def test_fp64_oracle_matches_reference_fp64(name):
    g = load_golden(name)
    vol = golden_input(g)
    out64, ranks64 = orc.denoise_fp64(vol, tuple(g["patch"]), int(g["stride"]))
    np.testing.assert_array_equal(ranks64, g["ranks64"])
    np.testing.assert_allclose(out64.reshape(-1)[g["sample_idx"]], g["out64_sample"], rtol=1e-12)


def test_oracle_config1_ranks_and_sample():
    g = load_golden("config1_lowrank")
    vol = golden_input(g)
    out, ranks = orc.denoise(vol, tuple(g["patch"]), int(g["stride"]))
    np.testing.assert_array_equal(ranks, g["ranks"])
    np.testing.assert_array_equal(out.reshape(-1)[g["sample_idx"]], g["out_sample"])
    assert abs(np.linalg.norm(out.astype(np.float64)) - float(g["norm_out"])) == 0.0


def test_region_oracle_equals_full_loop():
    g = load_golden("lowrank_p5s2")
    vol = golden_input(g)
    patch, step = tuple(g["patch"]), int(g["stride"])
    lo, hi = (3, 2, 4), (9, 7, 8)
    box, idx, ranks = orc.denoise_region(vol, patch, step, lo, hi)
    np.testing.assert_array_equal(box, g["out"][3:9, 2:7, 4:8])
    np.testing.assert_array_equal(ranks, g["ranks"][idx])


@pytest.mark.parametrize("shape,patch,step,count", [
    ((48, 48, 24, 48), (11, 11, 11), 3, 1176),
    ((96, 96, 48, 48), (11, 11, 11), 3, 12600),
    ((128, 128, 64, 96), (11, 11, 11), 2, 100800),
])
def test_patch_counts(shape, patch, step, count):
    assert problem.n_patches(shape, patch, step) == count
    assert len(orc.patch_corners(shape, patch, step)) == count


@pytest.mark.parametrize("shape,patch,step", [
    ((17, 15, 13, 4), (11, 11, 11), 3), ((14, 13, 12, 4), (5, 5, 5), 2), ((13, 12, 11, 4), (5, 7, 3), 2),
    ((9, 9, 8, 4), (5, 5, 5), 3), ((11, 11, 11, 4), (11, 11, 11), 3), ((20, 7, 30, 4), (3, 7, 4), 5)])
def test_corners_and_cover(shape, patch, step):
    c = problem.patch_corners(shape, patch, step)
    np.testing.assert_array_equal(c, orc.patch_corners(shape, patch, step))
    bases = problem.patch_bases(shape, patch, step)
    _, ny, nz = shape[:3]
    np.testing.assert_array_equal(bases, c[:, 0] * ny * nz + c[:, 1] * nz + c[:, 2])
    for a in range(3):
        ac = problem.axis_corners(shape[a], patch[a], step)
        cov = problem.cover_range(shape[a], patch[a], step)
        for x in range(shape[a]):
            want = [i for i, cc in enumerate(ac) if cc <= x <= cc + patch[a] - 1]
            # stride > patch leaves voxels no patch covers: an empty range
            assert list(range(cov[x, 0], cov[x, 1] + 1)) == want


def test_gram_route_stage_checker_agrees_with_svd():
    g = load_golden("single_patch")
    vol = golden_input(g).astype(np.float64)
    x = vol.reshape(-1, vol.shape[-1])
    st = orc.gram_route_patch(x)
    assert st["p"] == int(g["ranks64"][0])
    s = np.linalg.svd(x - x.mean(1, keepdims=True), compute_uv=False)
    np.testing.assert_allclose(np.sort(st["lam"])[::-1][:-1], s[:-1] ** 2, rtol=1e-9, atol=1e-6)


def test_noise_map_oracle_ranks_and_scale():
    """The noise oracle picks step 0's ranks, and on pure noise its patch
    estimates recover the noise variance."""
    from oracle import mppca as orc
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    vol = make_phantom_lowrank((14, 13, 12, 32), seed=0)[0]
    ranks, sig2, nmap = orc.noise_map(vol, (5, 5, 5), 2)
    _, ref_ranks = orc.denoise(vol, (5, 5, 5), 2)
    np.testing.assert_array_equal(ranks, ref_ranks)
    assert nmap.shape == vol.shape[:3] and (nmap > 0).all()
    rng = np.random.default_rng(4)
    noise = (rng.standard_normal((12, 12, 12, 24)) * 0.1 + 3.0).astype(np.float32)
    r2, s2, m2 = orc.noise_map(noise, (7, 7, 7), 3)
    assert (r2 <= 1).all() and (r2 == 0).mean() > 0.9  # the ladder's test is approximate
    # the mean noise eigenvalue of the centred patch is sigma^2 (t-1)/t
    assert abs(float(np.median(s2)) / (0.01 * 23 / 24) - 1) < 0.05
    assert abs(float(m2.mean()) / (0.01 * 23 / 24) - 1) < 0.05


def test_parallel_fp64_oracle_matches_serial():
    from oracle import mppca as orc
    from lowrank_gpu_fastest_b200.harness import make_phantom_lowrank

    vol = make_phantom_lowrank((12, 11, 10, 16), seed=1)[0]
    ref, rr = orc.denoise_fp64(vol, (5, 5, 5), 2)
    par, rp = orc.denoise_fp64_parallel(vol, (5, 5, 5), 2, processes=3)
    np.testing.assert_array_equal(rp, rr)
    assert np.abs(par - ref).max() <= 1e-13 * np.abs(ref).max()
