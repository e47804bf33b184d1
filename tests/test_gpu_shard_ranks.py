"""Frame sharding through the product's own reduce with two ranks: two
processes (spawned, one GPU shared, a gloo process group) each accumulate their
block of frames into their own plan, sqcalc_b200.shard.reduce_plan sums the
plans' device accumulators (sqn_accumulator_view) in place and sets the frame
count, and rank 0's S(q), partials and per-mode grid must equal one plan over
all frames.  The ranks' kernels never wait on each other: the only exchange is
the host-side collective between frames."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system():
    rng = np.random.default_rng(19)
    natoms, box = 3000, 18.0
    types = rng.integers(1, 4, size=natoms).astype(np.int32)
    frames = rng.random((5, natoms, 3)) * box
    kw = dict(weight=1, amp_const=np.array([4.149, 5.803, 9.45]), qmin=0.0, qmax=5.0, nq=80,
              partials=True, precision=0, eps=1e-10, want_grid=True)
    return types, frames, box, kw


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from sqcalc_b200 import _lib
    from sqcalc_b200.shard import frame_block, reduce_plan
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        types, frames, box, kw = _system()
        with _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), types, **kw) as p:
            lo, hi = frame_block(len(frames), rank, world)
            p.accumulate(frames[lo:hi])
            p.sync()
            total = reduce_plan(p)
            S, Sp, G, n = p.finalize(grid=True)
        if rank == 0:
            np.savez(out, S=S, Sp=Sp, G=G, n=n, total=total)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_reduce_plan_matches_one_plan(tmp_path):
    import torch.multiprocessing as mp
    from sqcalc_b200 import _lib
    out = str(tmp_path / "rank0.npz")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    types, frames, box, kw = _system()
    with _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), types, **kw) as p:
        p.accumulate(frames)
        S, Sp, G, n = p.finalize(grid=True)
    assert int(got["n"]) == int(got["total"]) == n == len(frames)
    np.testing.assert_allclose(got["S"], S, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got["Sp"], Sp, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got["G"], G, rtol=1e-12, atol=1e-12)
