"""sqn_spread_frame_noalloc: the allocation-free spread entry point.

It serves callers that cannot call cudaMalloc (a framework that owns every
device byte through its own pool, a plugin inside an application that has
already reserved the device memory, a service that must keep a fixed
footprint): they pass device positions and device output grids, and the sort
scratch comes from a fixed static device array.

The check: two calls in a row through the C ABI; each call's grids are carried
through the rest of the pipeline on the test side (FFT, the oracle's
deconvolution and shell binning) and must give the same S(q) and partials as
the existing plan entry point, within the FP32 tolerances of the other tests
(max |dS| <= 1e-5 and max|d|/max(|ref|,1) <= 1e-4).  This file runs last so a
failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def noalloc_spread(L, pos_dev, species, strength, cell, origin, nf, w, beta, grid, stream):
    nf64 = np.ascontiguousarray(nf, dtype=np.int64)
    cellf = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    orig = np.ascontiguousarray(origin, dtype=np.float64)
    return L.sqn_spread_frame_noalloc(
        ctypes.c_void_p(pos_dev.data_ptr()), int(pos_dev.shape[0]),
        ctypes.c_void_p(species.ctypes.data), int(len(strength)),
        ctypes.c_void_p(strength.ctypes.data), ctypes.c_void_p(cellf.ctypes.data),
        ctypes.c_void_p(orig.ctypes.data), ctypes.c_void_p(nf64.ctypes.data), int(w),
        float(beta), ctypes.c_void_p(grid.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_spread_matches_plan_entry_point():
    import torch

    L = _lib.load()
    rng = np.random.default_rng(31)
    box, natoms, qmax, nq = 24.0, 6000, 6.0, 80
    types = rng.integers(1, 3, size=natoms).astype(np.int32)
    cell = np.eye(3) * box
    frames = [rng.random((natoms, 3)) * box for _ in range(2)]

    plan = _lib.Plan(cell.reshape(9), np.zeros(3), types, qmin=0.0, qmax=qmax, nq=nq,
                     norm=_lib.NORM_MEAN, partials=True, precision=_lib.PREC_SINGLE, eps=1e-6)
    info = plan.info
    nf = [int(x) for x in info.nf]
    w, beta = int(info.kernel_width), float(info.beta)
    modes = np.array(info.modes, dtype=np.int32)

    # kernel Fourier coefficients and reciprocal basis for the test-side binning
    ph = [np.zeros((m - 1) // 2 + 1) for m in modes]
    for d in range(3):
        O.lib().sqo_kernel_fseries(nf[d], w, beta, int((modes[d] - 1) // 2), ph[d])
    grid_cfg = O.configure_grid(cell, 0.0, qmax, nq)
    recip = np.ascontiguousarray(grid_cfg.recip.reshape(9))

    species = np.ascontiguousarray(types - 1, dtype=np.uint8)
    strength = np.ones(2, dtype=np.float32)
    stream = torch.cuda.Stream()
    for call, pos in enumerate(frames):
        # existing entry point: one frame through the plan
        plan.reset()
        plan.accumulate(pos)
        S_ref, P_ref, _, _ = plan.finalize()

        # new entry point: spread only, into a caller-owned grid
        pos_dev = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
        grid = torch.empty((2, nf[2], nf[1], nf[0]), dtype=torch.float32, device="cuda")
        grid.fill_(float("nan"))  # every cell must be written by the call
        torch.cuda.synchronize()
        rc = noalloc_spread(L, pos_dev, species, strength, cell, np.zeros(3), nf, w, beta, grid,
                            stream.cuda_stream)
        assert rc == 0, _lib.error_string(rc)
        stream.synchronize()
        assert bool(torch.isfinite(grid).all()), "call %d left cells unwritten" % call

        G = torch.fft.rfftn(grid.double(), dim=(1, 2, 3)).cpu().numpy()
        G = np.ascontiguousarray(G).view(np.float64).reshape(-1)
        num = np.zeros(nq)
        pp = np.zeros(3 * nq)
        O.lib().sqo_bin_halfspace(G, 2, np.array(nf, dtype=np.int64), modes, recip, 0.0, qmax,
                                  nq, ph[0], ph[1], ph[2], None, num, pp)
        acc = plan.accumulators()
        den, cnt = acc["den"], np.maximum(acc["shell_count"], 1)
        S = np.where(den > 0, num / np.where(den > 0, den, 1.0), 0.0)
        pp = pp.reshape(3, nq)
        for (a, b), k in (((0, 0), 0), ((0, 1), 1), ((1, 1), 2)):
            part = pp[k] / (natoms * cnt)
            assert float(np.max(np.abs(part - P_ref[a, b]))) <= 1e-5, (call, a, b)
        assert float(np.max(np.abs(S - S_ref))) <= 1e-5, call
        assert float(np.max(np.abs(S - S_ref) / np.maximum(np.abs(S_ref), 1.0))) <= 1e-4
    plan.close()


def test_noalloc_rejects_oversized_requests():
    import torch

    L = _lib.load()
    natoms = 2_000_000  # 24 B of records/keys per atom alone exceed the 32 MiB array
    pos = torch.zeros((natoms, 3), dtype=torch.float64, device="cuda")
    species = np.zeros(natoms, dtype=np.uint8)
    strength = np.ones(1, dtype=np.float32)
    grid = torch.empty((1, 32, 32, 32), dtype=torch.float32, device="cuda")
    rc = noalloc_spread(L, pos, species, strength, np.eye(3) * 10.0, np.zeros(3),
                        [32, 32, 32], 8, 18.0, grid, 0)
    assert rc == _lib.ERR_SCRATCH_LIMIT
    bad = np.ones(1000, dtype=np.uint8)  # species index 1 with ntr = 1
    rc = noalloc_spread(L, torch.zeros((1000, 3), dtype=torch.float64, device="cuda"), bad,
                        strength, np.eye(3) * 10.0, np.zeros(3), [32, 32, 32], 8, 18.0, grid, 0)
    assert rc == 21
