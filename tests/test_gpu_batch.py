"""Batches of independent systems behind one CUDA graph: every system of the
batch gives what a plan of its own gives on the same frames, on the
multi-system path (each frame stage of all systems in one launch) and on the
branch-per-system path it falls back to for mixed systems.  The bin sort
places the points of a bin in atomic order, so the order of the FP32 sums, and
with it the last bits, may differ between any two runs: FP32 results agree to
rtol 1e-6 (absolute 1e-7 for values near zero), FP64 to 1e-12."""
import numpy as np
import pytest

from sqcalc_b200 import _lib
from sqcalc_b200.synthetic import batched_systems

pytestmark = pytest.mark.gpu


def system_kw(n, box, types, precision, eps):
    return dict(cell=np.eye(3).reshape(9) * box, origin=np.zeros(3), type_id=types, qmin=0.0,
                qmax=6.0, nq=120, partials=True, precision=precision, eps=eps)


def tols(precision):
    return (1e-6, 1e-7) if precision == _lib.PREC_SINGLE else (1e-12, 1e-13)


@pytest.mark.parametrize("precision,eps", [(_lib.PREC_SINGLE, 1e-6), (_lib.PREC_DOUBLE, 1e-9)])
def test_batch_matches_separate_plans(precision, eps):
    systems = batched_systems(5, seed=8, nmin=400, nmax=9000)
    rng = np.random.default_rng(1)
    frames = [rng.random((3, n, 3)) * box for n, box, _ in systems]
    kws = [system_kw(n, box, t, precision, eps) for n, box, t in systems]
    with _lib.Batch(kws) as b:
        assert b.multi
        b.accumulate(frames)
        b.sync()
        assert b.graph_launches() == 3
        got = [v.finalize() for v in b.plans]
        n512 = sum(v.info.pruned_fft512 for v in b.plans)
        # prep, scan, scatter, spread and bin of all systems, plus the pruned FFT
        # passes of the 512^3 systems (cuFFT's kernels are not counted)
        assert b.launch_count() == 3 * (5 + 3 * n512)
    rtol, atol = tols(precision)
    for k, kw in enumerate(kws):
        with _lib.Plan(**kw) as p:
            p.accumulate(frames[k])
            S, Sp, _, n = p.finalize()
        assert got[k][3] == n == 3
        np.testing.assert_allclose(got[k][0], S, rtol=rtol, atol=atol)
        np.testing.assert_allclose(got[k][1], Sp, rtol=rtol, atol=atol)


def test_mixed_batch_runs_one_branch_per_system():
    systems = batched_systems(3, seed=4, nmin=600, nmax=3000)
    rng = np.random.default_rng(2)
    frames = [rng.random((2, n, 3)) * box for n, box, _ in systems]
    kws = [system_kw(n, box, t, _lib.PREC_SINGLE if k != 1 else _lib.PREC_DOUBLE,
                     1e-6 if k != 1 else 1e-9) for k, (n, box, t) in enumerate(systems)]
    with _lib.Batch(kws) as b:
        assert not b.multi
        b.accumulate(frames)
        b.sync()
        got = [v.finalize()[0] for v in b.plans]
    for k, kw in enumerate(kws):
        rtol, atol = tols(kw["precision"])
        with _lib.Plan(**kw) as p:
            p.accumulate(frames[k])
            np.testing.assert_allclose(got[k], p.finalize()[0], rtol=rtol, atol=atol)


def test_autotuned_batch_matches_autotuned_plans():
    systems = batched_systems(3, seed=12, nmin=2000, nmax=6000)
    rng = np.random.default_rng(3)
    frames = [rng.random((2, n, 3)) * box for n, box, _ in systems]
    kws = [dict(system_kw(n, box, t, _lib.PREC_SINGLE, 1e-6), autotune=True)
           for n, box, t in systems]
    with _lib.Batch(kws) as b:
        assert b.multi and all(v.info.autotuned for v in b.plans)
        grids = [tuple(v.info.nf) + (v.info.kernel_width,) for v in b.plans]
        b.accumulate(frames)
        b.sync()
        got = [v.finalize()[0] for v in b.plans]
    rtol, atol = tols(_lib.PREC_SINGLE)
    for k, kw in enumerate(kws):
        with _lib.Plan(**kw) as p:
            assert tuple(p.info.nf) + (p.info.kernel_width,) == grids[k]  # the cached choice
            p.accumulate(frames[k])
            np.testing.assert_allclose(got[k], p.finalize()[0], rtol=rtol, atol=atol)


def test_batch_device_positions_and_repeated_steps():
    import torch
    systems = batched_systems(3, seed=9, nmin=1000, nmax=4000)
    kws = [system_kw(n, box, t, _lib.PREC_SINGLE, 1e-6) for n, box, t in systems]
    gen = torch.Generator(device="cuda").manual_seed(3)
    dev = [torch.rand((4, n, 3), generator=gen, device="cuda", dtype=torch.float64) * box
           for n, box, _ in systems]
    torch.cuda.synchronize()
    with _lib.Batch(kws) as b:
        for f in range(4):
            b.accumulate([d[f].data_ptr() for d in dev], where=_lib.DEVICE, nframes=1)
        b.sync()
        got = [v.finalize()[0] for v in b.plans]
        assert b.graph_launches() == 4
    rtol, atol = tols(_lib.PREC_SINGLE)
    for k, kw in enumerate(kws):
        with _lib.Plan(**kw) as p:
            p.accumulate(dev[k].cpu().numpy())
            np.testing.assert_allclose(got[k], p.finalize()[0], rtol=rtol, atol=atol)


def test_batch_rejects_bad_input():
    with pytest.raises(_lib.SqnError):
        _lib.Batch([])
    systems = batched_systems(2, seed=10, nmin=500, nmax=600)
    kws = [system_kw(n, box, t, _lib.PREC_SINGLE, 1e-6) for n, box, t in systems]
    with _lib.Batch(kws) as b:
        with pytest.raises(ValueError):
            b.accumulate([np.zeros((1, 7, 3)), np.zeros((1, 7, 3))])
