"""Regenerate the golden fixtures from the reference ladder's own step-0 loop.

Run where a checkout of the reference exists (it is only read), giving its
path as an argument or in ``LRD_REFERENCE``:

    python tests/golden/make_golden.py --reference <checkout> [--skip-large]

The reference's ``common.py`` writes a ``results/`` folder next to itself on
import, so the script copies the reference's Python files into a temporary
directory and imports them from there. For each case it records:

* the input volume's SHA-256 (the tests regenerate the input with the
  package's phantom generators and check the hash, which pins those
  generators to the ladder's ``common.make_phantom``);
* the per-patch ranks chosen by ``step0_numpy_loop.mppca_patch``;
* the step-0 output (in full for small volumes; a seeded sample of elements
  plus float64 norms for the large ones), and the same for the float64 run of
  the reference's step-0 code (``denoise(vol.astype(float64))``).

Other patch shapes and strides are obtained by rebinding ``PATCH`` and
``patch_corners`` inside the imported step-0 module; the loop itself is the
reference's, unmodified.
"""

from __future__ import annotations

import argparse
import hashlib
import importlib
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from lowrank_gpu_fastest_b200.harness import make_phantom, make_phantom_lowrank  # noqa: E402

SMALL = [
    # name, generator, shape, patch, stride, gen kwargs
    ("ref_small", "ref", (17, 15, 13, 24), (11, 11, 11), 3, {}),
    ("lowrank_p5s2", "lowrank", (14, 13, 12, 32), (5, 5, 5), 2, {}),
    ("ref_p7s1", "ref", (12, 11, 10, 16), (7, 7, 7), 1, {}),
    ("lowrank_t96", "lowrank", (9, 9, 8, 96), (5, 5, 5), 3, {}),
    ("lowrank_t64", "lowrank", (10, 9, 8, 64), (5, 5, 5), 2, {"sigma": 0.02}),
    ("aniso", "lowrank", (13, 12, 11, 20), (5, 7, 3), 2, {}),
    ("single_patch", "ref", (11, 11, 11, 16), (11, 11, 11), 3, {}),
    ("constant", "const", (8, 8, 8, 12), (5, 5, 5), 2, {}),
    ("rank8_s0.01", "lowrank", (13, 12, 11, 48), (7, 7, 7), 3, {"rank": 8, "sigma": 0.01}),
]
LARGE = [
    ("config1_lowrank", "lowrank", (48, 48, 24, 48), (11, 11, 11), 3, {}),
    ("config1_ref", "ref", (48, 48, 24, 48), (11, 11, 11), 3, {}),
    ("headline_lowrank", "lowrank", (96, 96, 48, 48), (11, 11, 11), 3, {}),
    ("headline_ref", "ref", (96, 96, 48, 48), (11, 11, 11), 3, {}),
]
N_SAMPLE = 20000


def make_input(gen, shape, kw):
    if gen == "ref":
        return make_phantom(shape, **kw)[0]
    if gen == "lowrank":
        return make_phantom_lowrank(shape, **kw)[0]
    if gen == "const":
        return np.full(shape, 3.0, dtype=np.float32)
    raise ValueError(gen)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load_reference(tmp, reference):
    for f in os.listdir(reference):
        if f.endswith(".py"):
            shutil.copy(os.path.join(reference, f), tmp)
    sys.path.insert(0, tmp)
    common = importlib.import_module("common")
    s0 = importlib.import_module("step0_numpy_loop")
    return common, s0


def run_step0(common, s0, vol, patch, stride):
    ranks = []
    orig = s0.mppca_patch

    def rec(x):
        xd, p = orig(x)
        ranks.append(p)
        return xd, p

    s0.mppca_patch = rec
    s0.PATCH = patch
    s0.patch_corners = lambda: common.patch_corners(vol.shape, patch, stride)
    try:
        out = s0.denoise(vol)
    finally:
        s0.mppca_patch = orig
    return out, np.array(ranks, dtype=np.int32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-large", action="store_true")
    ap.add_argument("--reference", default=os.environ.get("LRD_REFERENCE"),
                    help="path of the reference checkout (default: $LRD_REFERENCE)")
    args = ap.parse_args()
    if not args.reference or not os.path.isdir(args.reference):
        ap.error("give the reference checkout with --reference or LRD_REFERENCE")
    tmp = tempfile.mkdtemp(prefix="lrd_ref_")
    common, s0 = load_reference(tmp, args.reference)
    # the package's phantom must reproduce the ladder's bit for bit
    for shape in [(17, 15, 13, 24), (12, 11, 10, 16)]:
        a = common.make_phantom(shape)[0]
        b = make_phantom(shape)[0]
        assert a.tobytes() == b.tobytes(), "make_phantom differs from common.make_phantom"
    cases = SMALL + ([] if args.skip_large else LARGE)
    for name, gen, shape, patch, stride, kw in cases:
        vol = make_input(gen, shape, kw)
        if gen == "ref":
            assert common.make_phantom(shape, **kw)[0].tobytes() == vol.tobytes()
        out, ranks = run_step0(common, s0, vol, patch, stride)
        out64, ranks64 = run_step0(common, s0, vol.astype(np.float64), patch, stride)
        rec = dict(
            gen=gen, shape=np.array(shape), patch=np.array(patch), stride=stride,
            gen_kwargs=repr(kw), input_sha256=sha(vol), ranks=ranks, ranks64=ranks64,
            norm_out=np.linalg.norm(out.astype(np.float64)),
            norm_out64=np.linalg.norm(out64),
            diff_step0_fp64=np.linalg.norm(out.astype(np.float64) - out64),
        )
        if out.size <= 200_000:
            rec["out"] = out
        idx = np.random.default_rng(1234).choice(out.size, min(N_SAMPLE, out.size), replace=False)
        idx.sort()
        rec["sample_idx"] = idx.astype(np.int64)
        rec["out_sample"] = out.reshape(-1)[idx]
        rec["out64_sample"] = out64.reshape(-1)[idx]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print(f"{name}: {len(ranks)} patches, ranks {np.bincount(ranks)}, "
              f"step0 vs fp64 {rec['diff_step0_fp64'] / rec['norm_out64']:.3e}")
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
