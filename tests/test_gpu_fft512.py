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


def test_pruned_passes_xray_weights_and_powder_pattern():
    """q-dependent (x-ray) amplitudes and the two-theta histogram of the powder
    pattern read from the compact spectrum, against the cuFFT plan."""
    tid, fr = frames(2)
    coef = np.array([[2.0, 1.5, 1.0, 0.5, 10.0, 5.0, 1.0, 0.2, 0.3],
                     [3.0, 2.0, 1.0, 0.4, 12.0, 4.0, 0.8, 0.1, 0.5],
                     [6.0, 3.0, 2.0, 1.0, 8.0, 3.0, 0.9, 0.3, 1.0]])
    xrd = dict(lam=1.5406, range=(10.0, 60.0), step=0.5, lp=True)

    def mk(cufft):
        return _lib.Plan(np.eye(3).reshape(9) * L, np.zeros(3), tid, ntypes=3,
                         weight=_lib.WEIGHT_XRAY, xray_coef=coef, qmin=0.0, qmax=QMAX, nq=200,
                         partials=True, precision=_lib.PREC_SINGLE, eps=1e-6,
                         fused_fft=False if cufft else None, xrd=xrd)
    with mk(False) as pp, mk(True) as pc:
        assert pp.info.pruned_fft512 == 1 and pc.info.pruned_fft512 == 0
        for p in (pp, pc):
            for f in fr:
                p.accumulate(f)
        a, b = pp.finalize(), pc.finalize()
        for x, y in ((a[0], b[0]), (a[1], b[1])):
            assert np.max(np.abs(x - y)) / max(1.0, float(np.max(np.abs(y)))) < 2e-6
        xa, xb = pp.xrd(), pc.xrd()
        np.testing.assert_array_equal(xa[3], xb[3])
        for x, y in ((xa[1], xb[1]), (xa[2], xb[2])):
            assert np.max(np.abs(x - y)) / max(1.0, float(np.max(np.abs(y)))) < 2e-6
