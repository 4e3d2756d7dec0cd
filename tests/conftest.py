import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built liblrd.so")


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False)
    return {k: d[k] for k in d.files}


def golden_input(g):
    """Regenerate a golden case's input volume with the package's generators."""
    import ast

    from lowrank_gpu_fastest_b200.harness import make_phantom, make_phantom_lowrank

    shape = tuple(int(s) for s in g["shape"])
    kw = ast.literal_eval(str(g["gen_kwargs"]))
    gen = str(g["gen"])
    if gen == "ref":
        return make_phantom(shape, **kw)[0]
    if gen == "lowrank":
        return make_phantom_lowrank(shape, **kw)[0]
    if gen == "const":
        return np.full(shape, 3.0, dtype=np.float32)
    raise ValueError(gen)


SMALL_CASES = ["ref_small", "lowrank_p5s2", "ref_p7s1", "lowrank_t96", "lowrank_t64", "aniso",
               "single_patch", "constant", "rank8_s0.01"]
LARGE_CASES = ["config1_lowrank", "config1_ref", "headline_lowrank", "headline_ref"]


@pytest.fixture(scope="session")
def cuda_ok():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
