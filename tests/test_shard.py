"""Frame sharding over ranks (CPU, gloo, world size 2): each rank accumulates a
contiguous block of frames and one sum all-reduce combines the FP64 sums;
the result equals accumulating every frame in one process
(src/sqc_structure_factor.f90:457-470)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sqcalc_b200.shard import frame_block


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7])
def test_frame_blocks_cover_each_frame_once(world):
    for n in [0, 1, 2, 5, 16, 101]:
        seen = []
        sizes = []
        for r in range(world):
            lo, hi = frame_block(n, r, world)
            seen.extend(range(lo, hi))
            sizes.append(hi - lo)
        assert seen == list(range(n))
        assert max(sizes) - min(sizes) <= 1


def test_frame_block_rejects_bad_rank():
    with pytest.raises(ValueError):
        frame_block(10, 2, 2)


def _system():
    rng = np.random.default_rng(11)
    natoms, box = 300, 9.0
    types = rng.integers(1, 3, size=natoms).astype(np.int32)
    frames = [rng.random((natoms, 3)) * box for _ in range(5)]
    return types, frames, np.eye(3) * box


def _accumulate(frames):
    from oracle import oracle as O
    types, _, cell = _system()
    w = O.Weights(kind=O.WEIGHT_NEUTRON, amp_const=np.array([3.0, 5.0]))
    _, acc = O.direct_sq(frames, types, cell, np.zeros(3), w, 0.5, 4.0, 40)
    return acc


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from sqcalc_b200.shard import reduce_host
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        _, frames, _ = _system()
        lo, hi = frame_block(len(frames), rank, world)
        acc = _accumulate(frames[lo:hi])
        tot = reduce_host({"num": acc.num, "partial_num": acc.partial_num,
                           "nframes": acc.nframes})
        if rank == 0:
            np.savez(out, num=tot["num"], partial_num=tot["partial_num"],
                     nframes=tot["nframes"], den=acc.den)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gloo_two_ranks_match_one_process(tmp_path):
    from oracle import oracle as O
    O.build()
    out = str(tmp_path / "rank0.npz")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    _, frames, _ = _system()
    ref = _accumulate(frames)
    assert int(got["nframes"]) == len(frames)
    np.testing.assert_allclose(got["num"], ref.num, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(got["partial_num"], ref.partial_num, rtol=1e-12, atol=1e-9)
    S_sharded = np.where(ref.den > 0, got["num"] / (len(frames) * np.where(ref.den > 0, ref.den, 1)), 0)
    np.testing.assert_allclose(S_sharded, ref.shell_value(), rtol=1e-12, atol=1e-12)
