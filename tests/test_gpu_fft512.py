"""Pruned 512-point FFT passes (k_fft512_x, k_fft512_cols) on 512^3 fine grids:
S(q), the partials and the per-mode grid against the same plan on cuFFT R2C
(SQN_FLAG_CUFFT), FP32 and FP64."""
import numpy as np
import pytest

from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu

L, N = 100.0, 60000
QMAX = 211.4 * 2 * np.pi / L  # 425 modes per axis: a 512^3 fine grid at sigma ~1.2


def frames(nframes=3, seed=8):
    rng = np.random.default_rng(seed)
    tid = rng.choice(np.array([1, 2, 3], dtype=np.int32), N, p=[0.5, 0.3, 0.2])
    base = rng.random((N, 3)) * L
    return tid, [base + rng.normal(0, 0.3, (N, 3)) for _ in range(nframes)]


def plan(tid, precision, eps, cufft, qmax=QMAX, **kw):
    return _lib.Plan(np.eye(3).reshape(9) * L, np.zeros(3), tid, ntypes=3,
                     weight=_lib.WEIGHT_NEUTRON, amp_const=np.array([4.149, 5.803, 9.45]),
                     qmin=0.0, qmax=qmax, nq=300, partials=True, precision=precision, eps=eps,
                     cufft=cufft, **kw)


@pytest.mark.parametrize("precision,eps,tol,grid", [
    (_lib.PREC_SINGLE, 1e-6, 2e-6, False),
    (_lib.PREC_SINGLE, 1e-6, 2e-6, True),
    (_lib.PREC_DOUBLE, 1e-6, 1e-12, False),
])
def test_pruned_passes_match_cufft(precision, eps, tol, grid):
    tid, fr = frames()
    with plan(tid, precision, eps, False, want_grid=grid) as pp, \
            plan(tid, precision, eps, True, want_grid=grid) as pc:
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


@pytest.mark.parametrize("ntypes", [1, 2, 4, 5])
def test_pruned_passes_transform_counts(ntypes):
    """Every transform count k_bin instantiates on the compact spectrum (1, 2, 4
    unrolled; 5 on the generic path), with mixed-sign partials, against the
    cuFFT plan (FP32, 2e-6 of max |S|; shell counts identical)."""
    rng = np.random.default_rng(30 + ntypes)
    n = 20000
    tid = (rng.integers(0, ntypes, n) + 1).astype(np.int32)
    base = rng.random((n, 3)) * L
    fr = [base + rng.normal(0, 0.3, (n, 3)) for _ in range(2)]
    b = np.linspace(3.0, 9.0, ntypes)

    def mk(cufft):
        return _lib.Plan(np.eye(3).reshape(9) * L, np.zeros(3), tid, ntypes=ntypes,
                         weight=_lib.WEIGHT_NEUTRON, amp_const=b, qmin=0.5, qmax=QMAX, nq=250,
                         partials=True, precision=_lib.PREC_SINGLE, eps=1e-6, cufft=cufft)
    with mk(False) as pp, mk(True) as pc:
        assert pp.info.pruned_fft512 == 1 and pp.info.ntransforms == ntypes
        for p in (pp, pc):
            for f in fr:
                p.accumulate(f)
        ca, cb = pp.accumulators()["shell_count"], pc.accumulators()["shell_count"]
        np.testing.assert_array_equal(ca, cb)
        a, c = pp.finalize(), pc.finalize()
        for x, y in ((a[0], c[0]), (a[1], c[1])):
            assert np.max(np.abs(x - y)) / max(1.0, float(np.max(np.abs(y)))) < 2e-6


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
                         cufft=cufft, xrd=xrd)
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


def test_default_512_path_against_direct_sum():
    """The benchmark's frame path itself -- L = 220 A, q_max 6 (423^3 modes), a
    512^3 fine grid, the pruned passes -- against the FP64 direct sum of the
    reference's --method direct (oracle.direct_sq_separable, pinned to
    oracle.direct_sq by tests/test_oracle.py) on a few hundred atoms: FP64
    within 1e-7 relative (shells and partials; the reference's own NUFFT-vs-direct
    bar is 1e-6, test/test_sqcalc.py:389-396), FP32 within max |dS| 1e-5."""
    from oracle import oracle as O

    rng = np.random.default_rng(11)
    box, n = 220.0, 500
    tid = rng.choice(np.array([1, 2, 3], dtype=np.int32), n, p=[0.5, 0.3, 0.2])
    base = rng.random((n, 3)) * box
    fr = [base + rng.normal(0, 0.3, (n, 3)) for _ in range(2)]
    b = np.array([4.149, 5.803, 9.45])
    w = O.Weights(kind=O.WEIGHT_NEUTRON, amp_const=b)
    modes, acc = O.direct_sq_separable(fr, tid, np.eye(3) * box, np.zeros(3), w, 0.0, 6.0, 500)
    assert list(modes) == [423, 423, 423]
    ref = acc.shell_value()
    refp = [acc.partial_value(a, c) for a in (1, 2, 3) for c in (1, 2, 3) if c >= a]
    for prec, eps in ((_lib.PREC_DOUBLE, 1e-9), (_lib.PREC_SINGLE, 1e-6)):
        with _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), tid, ntypes=3,
                       weight=_lib.WEIGHT_NEUTRON, amp_const=b, qmin=0.0, qmax=6.0, nq=500,
                       partials=True, precision=prec, eps=eps) as p:
            assert list(p.info.nf) == [512, 512, 512] and p.info.pruned_fft512 == 1
            for f in fr:
                p.accumulate(f)
            counts = p.accumulators()["shell_count"]
            S, Sp, _, nfr = p.finalize()
        assert nfr == 2
        np.testing.assert_array_equal(counts, acc.shell_count)
        got = [Sp[a - 1, c - 1] for a in (1, 2, 3) for c in (1, 2, 3) if c >= a]
        dS = float(np.max(np.abs(S - ref)))
        rel = dS / max(1.0, float(np.max(np.abs(ref))))
        dP = max(float(np.max(np.abs(x - y))) for x, y in zip(got, refp))
        if prec == _lib.PREC_DOUBLE:
            assert rel < 1e-7 and dP < 1e-7, (rel, dP)
        else:
            assert dS < 1e-5 and dP < 1e-5, (dS, dP)



def test_pruned_passes_triclinic_skips():
    """A triclinic cell on the pruned 512^3 path: the columns and rows the
    passes skip (derived from the binning rows of the tilted reciprocal lattice)
    must still hold every mode the binning reads -- S(q) and the partials equal
    the cuFFT plan's (FP32, 2e-6 of max |S|; shell counts identical)."""
    rng = np.random.default_rng(17)
    a = np.array([[L, 0.0, 0.0], [10.0, 99.5, 0.0], [5.0, 8.0, 99.4]])
    n = 20000
    tid = rng.choice(np.array([1, 2, 3], dtype=np.int32), n, p=[0.5, 0.3, 0.2])
    frac = rng.random((n, 3))
    fr = [(frac + rng.normal(0, 0.003, (n, 3))) @ a for _ in range(2)]

    def mk(cufft):
        return _lib.Plan(a.reshape(9), np.zeros(3), tid, ntypes=3, weight=_lib.WEIGHT_NEUTRON,
                         amp_const=np.array([4.149, 5.803, 9.45]), qmin=0.0, qmax=QMAX, nq=300,
                         partials=True, precision=_lib.PREC_SINGLE, eps=1e-6, cufft=cufft)
    with mk(False) as pp, mk(True) as pc:
        assert list(pp.info.nf) == [512, 512, 512] and pp.info.pruned_fft512 == 1
        for p in (pp, pc):
            for f in fr:
                p.accumulate(f)
        np.testing.assert_array_equal(pp.accumulators()["shell_count"],
                                      pc.accumulators()["shell_count"])
        x, y = pp.finalize(), pc.finalize()
        for u, v in ((x[0], y[0]), (x[1], y[1])):
            assert np.max(np.abs(u - v)) / max(1.0, float(np.max(np.abs(v)))) < 2e-6
