"""Pruned 512-point FFT passes (k_fft512_x, k_fft512_cols) on 512^3 fine grids:
S(q), the partials and the per-mode grid against the same plan on cuFFT R2C
(SQN_FLAG_CUFFT), FP32 and FP64, serial and pipelined."""
import numpy as np
import pytest

from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu

L, N = 100.0, 60000
QMAX = 211.4 * 2 * np.pi / L  # 423 modes per axis: a 512^3 fine grid at sigma ~1.21


def frames(nframes=3, seed=8):
    rng = np.random.default_rng(seed)
    tid = rng.choice(np.array([1, 2, 3], dtype=np.int32), N, p=[0.5, 0.3, 0.2])
    base = rng.random((N, 3)) * L
    return tid, [base + rng.normal(0, 0.3, (N, 3)) for _ in range(nframes)]


def plan(tid, precision, eps, cufft, **kw):
    return _lib.Plan(np.eye(3).reshape(9) * L, np.zeros(3), tid, ntypes=3,
                     weight=_lib.WEIGHT_NEUTRON, amp_const=np.array([4.149, 5.803, 9.45]),
                     qmin=0.0, qmax=QMAX, nq=300, partials=True, precision=precision, eps=eps,
                     fused_fft=False if cufft else None, **kw)


@pytest.mark.parametrize("precision,eps,tol,serial,grid", [
    (_lib.PREC_SINGLE, 1e-6, 2e-6, False, False),
    (_lib.PREC_SINGLE, 1e-6, 2e-6, True, True),
    (_lib.PREC_DOUBLE, 1e-6, 1e-12, False, False),
])
def test_pruned_passes_match_cufft(precision, eps, tol, serial, grid):
    tid, fr = frames()
    with plan(tid, precision, eps, False, pipeline=not serial, want_grid=grid) as pp, \
            plan(tid, precision, eps, True, pipeline=not serial, want_grid=grid) as pc:
        assert list(pp.info.nf) == [512, 512, 512]
        assert pp.info.pruned_fft512 == 1 and pc.info.pruned_fft512 == 0
        for p in (pp, pc):
            for f in fr:
                p.accumulate(f)
        a = pp.finalize(grid=grid)
        b = pc.finalize(grid=grid)
        scale = max(1.0, float(np.max(np.abs(b[0]))))
        assert np.max(np.abs(a[0] - b[0])) / scale < tol
        assert np.max(np.abs(a[1] - b[1])) / max(1.0, float(np.max(np.abs(b[1])))) < tol
        if grid:
            assert np.max(np.abs(a[2] - b[2])) / max(1.0, float(np.max(np.abs(b[2])))) < 10 * tol
        # three more kernels per frame than the cuFFT plan
        assert pp.launch_count() - pc.launch_count() == 3 * len(fr)
