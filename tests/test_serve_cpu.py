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


def test_buffer_pool_reuses_by_size_class():
    """Device buffers of finished requests are reused by later requests of the
    same (2 MiB) size class; a larger request gets a new buffer."""
    import torch

    from lowrank_gpu_fastest_b200.serve import _Pool

    made = []

    def alloc(kind, nbytes):
        made.append((kind, nbytes))
        return torch.empty(nbytes, dtype=torch.uint8)

    pool = _Pool(alloc)
    a = pool.take("ws", 3 << 20)
    assert a.numel() == 4 << 20 and len(made) == 1
    pool.give("ws", a)
    assert pool.free_bytes == 4 << 20
    b = pool.take("ws", (3 << 20) + 5)
    assert b.data_ptr() == a.data_ptr() and len(made) == 1 and pool.free_bytes == 0
    pool.give("ws", b)
    c = pool.take("ws", 9 << 20)
    assert c.numel() == 10 << 20 and len(made) == 2
    d = pool.take("d_in", 1)
    assert d.numel() == 2 << 20 and len(made) == 3
    pool.trim()
    assert pool.free_bytes == 0
