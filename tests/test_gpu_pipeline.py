"""Frame pipeline: the FFT and binning of frame f on the plan's FFT stream
beside the sort and spread of frame f + 1 (two fine grids) give the sums of a
serial plan (without SQN_FLAG_PIPELINE), for host and device frames, through peek, reset,
the accumulator view and the single-frame entry points that share the plan."""
import numpy as np
import pytest

from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def make(frames, tid, cell, precision, serial, **kw):
    return _lib.Plan(cell.reshape(9), np.zeros(3), tid, ntypes=2, weight=_lib.WEIGHT_NEUTRON,
                     amp_const=np.array([0.6, 1.4]), qmin=0.5, qmax=6.0, nq=60, partials=True,
                     precision=precision, eps=1e-6 if precision == _lib.PREC_SINGLE else 1e-10,
                     pipeline=not serial, **kw)


def system(n=20000, nframes=7, seed=4):
    rng = np.random.default_rng(seed)
    L = (n / 0.05) ** (1 / 3)
    cell = np.diag([L, L * 1.05, L * 0.97])
    tid = rng.integers(1, 3, n).astype(np.int32)
    frames = rng.random((nframes, n, 3)) @ cell
    return frames, tid, cell


@pytest.mark.parametrize("precision,rtol", [(_lib.PREC_DOUBLE, 1e-12), (_lib.PREC_SINGLE, 1e-6)])
def test_pipelined_equals_serial(precision, rtol):
    frames, tid, cell = system()
    with make(frames, tid, cell, precision, True) as ps, make(frames, tid, cell, precision,
                                                              False) as pp:
        assert ps.info.pipelined == 0 and pp.info.pipelined == 1
        for p in (ps, pp):
            p.accumulate(frames)
        a, b = ps.finalize(), pp.finalize()
        assert a[3] == b[3] == len(frames)
        np.testing.assert_allclose(b[0], a[0], rtol=rtol, atol=rtol)
        np.testing.assert_allclose(b[1], a[1], rtol=rtol, atol=rtol)


def test_pipeline_device_frames_peek_reset_view():
    import torch
    frames, tid, cell = system(nframes=5)
    dev = torch.tensor(frames, device="cuda")
    with make(frames, tid, cell, _lib.PREC_DOUBLE, True) as ps, make(frames, tid, cell,
                                                                     _lib.PREC_DOUBLE,
                                                                     False) as pp:
        pin = torch.zeros(60, dtype=torch.float64).pin_memory()
        for f in range(len(frames)):
            pp.accumulate((dev[f].data_ptr(), 1), where=_lib.DEVICE)
            pp.peek_num_async(pin.data_ptr())
        pp.join()
        pp.sync()
        ps.accumulate(frames)
        num_s = ps.accumulators()["num"]
        np.testing.assert_allclose(pin.numpy(), num_s, rtol=1e-12)
        # the accumulator view sees every frame's sums
        ptr, count, nf = pp.accumulator_view()
        assert nf == len(frames) and count > 0
        # reset, then the same frames again from the host
        pp.reset()
        pp.accumulate(frames)
        np.testing.assert_allclose(pp.accumulators()["num"], num_s, rtol=1e-12)
        # a single-frame entry point after queued frames (it joins both streams)
        pp.accumulate(frames[:3])
        rho = pp.density_modes(frames[0], np.array([[1, 0, 0], [0, 2, 1]], dtype=np.int32))
        with make(frames, tid, cell, _lib.PREC_DOUBLE, True) as q:
            ref = q.density_modes(frames[0], np.array([[1, 0, 0], [0, 2, 1]], dtype=np.int32))
        np.testing.assert_allclose(rho, ref, rtol=0, atol=1e-9 * len(tid))
        assert pp.finalize()[3] == len(frames) + 3


def test_timing_and_grad_plans_stay_serial():
    frames, tid, cell = system(n=3000, nframes=2)
    with make(frames, tid, cell, _lib.PREC_SINGLE, False, timing=True) as p:
        assert p.info.pipelined == 0
    with make(frames, tid, cell, _lib.PREC_SINGLE, False, grad=True) as p:
        assert p.info.pipelined == 0
    # serial unless asked for
    with _lib.Plan(cell.reshape(9), np.zeros(3), tid, ntypes=2, qmax=3.0, nq=20) as p:
        assert p.info.pipelined == 0
