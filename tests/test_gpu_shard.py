"""Device side of frame sharding: the plan's FP64 sums are one device buffer;
adding the buffers of two plans that each saw half of the frames and setting
the frame count reproduces one plan over all frames (what the NCCL all-reduce
in sqcalc_b200.shard.reduce_plan does across ranks)."""
import numpy as np
import pytest

from sqcalc_b200 import _lib
from sqcalc_b200.shard import _DeviceArray, frame_block

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("want_grid", [False, True])
def test_two_plans_add_to_one(want_grid):
    import torch
    rng = np.random.default_rng(5)
    natoms, box = 2000, 16.0
    types = rng.integers(1, 4, size=natoms).astype(np.int32)
    frames = rng.random((6, natoms, 3)) * box
    kw = dict(weight=_lib.WEIGHT_NEUTRON, amp_const=np.array([4.149, 5.803, 9.45]), qmin=0.0,
              qmax=5.0, nq=60, partials=True, precision=_lib.PREC_DOUBLE, eps=1e-10,
              want_grid=want_grid)
    cell = np.eye(3).reshape(9) * box
    with _lib.Plan(cell, np.zeros(3), types, **kw) as full, \
            _lib.Plan(cell, np.zeros(3), types, **kw) as a, \
            _lib.Plan(cell, np.zeros(3), types, **kw) as b:
        full.accumulate(frames)
        for plan, r in ((a, 0), (b, 1)):
            lo, hi = frame_block(len(frames), r, 2)
            plan.accumulate(frames[lo:hi])
        pa, na, fa = a.accumulator_view()
        pb, nb, fb = b.accumulator_view()
        assert na == nb and fa + fb == len(frames)
        ta = torch.as_tensor(_DeviceArray(pa, na), device="cuda")
        tb = torch.as_tensor(_DeviceArray(pb, nb), device="cuda")
        ta += tb
        torch.cuda.synchronize()
        a.set_frame_count(fa + fb)
        s1, p1, g1, n1 = full.finalize(grid=want_grid)
        s2, p2, g2, n2 = a.finalize(grid=want_grid)
    assert n1 == n2 == len(frames)
    np.testing.assert_allclose(s2, s1, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(p2, p1, rtol=1e-12, atol=1e-12)
    if want_grid:
        np.testing.assert_allclose(g2, g1, rtol=1e-12, atol=1e-12)


def test_single_rank_nccl_reduce_is_identity():
    import os
    import torch
    import torch.distributed as dist
    from sqcalc_b200.shard import reduce_plan
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29517")
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        rng = np.random.default_rng(6)
        types = rng.integers(1, 3, size=500).astype(np.int32)
        frames = rng.random((3, 500, 3)) * 10.0
        with _lib.Plan(np.eye(3).reshape(9) * 10.0, np.zeros(3), types, qmax=4.0, nq=40) as p:
            p.accumulate(frames)
            s0 = p.finalize()[0]
            assert reduce_plan(p) == 3
            s1, _, _, n = p.finalize()
        assert n == 3
        np.testing.assert_array_equal(s0, s1)
    finally:
        dist.destroy_process_group()
