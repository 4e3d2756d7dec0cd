"""Seeded workload generators of the serving form (no GPU)."""

import numpy as np

from lowrank_gpu_fastest_b200.serve import draw_request_shapes, poisson_arrivals


def test_workload_generators_are_seeded():
    a = poisson_arrivals(40.0, 5.0, seed=3)
    b = poisson_arrivals(40.0, 5.0, seed=3)
    np.testing.assert_array_equal(a, b)
    assert 100 < len(a) < 300
    s = draw_request_shapes(50, seed=1)
    assert s == draw_request_shapes(50, seed=1)
    for r in s:
        assert r["patch"][0] ** 3 >= r["shape"][3]
        assert 64 <= r["shape"][0] <= 128 and 32 <= r["shape"][2] <= 64
