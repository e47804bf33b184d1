"""The fused pruned FFT passes (x rows, y columns, z columns + binning) against
the cuFFT R2C + bin-kernel path of the same plan settings, on power-of-two and
mixed-radix (2, 3, 5) fine grids, cubic and triclinic cells, partials, x-ray
weights and the per-mode grid.  Both are checked against the FP64 oracle
elsewhere; here they must agree to FP32 / FP64 rounding: shells and partials
rtol 1e-5 (FP32, absolute 1e-7) and 1e-11 (FP64); single modes of the grid in
FP32 to the reference's FP32 tolerance rtol 1e-4 (absolute 1e-5)."""
import numpy as np
import pytest

from sqcalc_b200 import _lib
from sqcalc_b200.weights import WeightScheme

pytestmark = pytest.mark.gpu


def radices(n):
    out = set()
    for p in (2, 3, 5):
        while n % p == 0:
            out.add(p)
            n //= p
    return out


def run(cufft, pos, types, cell, **kw):
    with _lib.Plan(cell.reshape(9), np.zeros(3), types, fused_fft=not cufft, **kw) as p:
        assert p.info.fused_fft == (0 if cufft else 1)
        p.accumulate(pos)
        S, Sp, Sg, _ = p.finalize(grid=kw.get("want_grid", False))
        return S, Sp, Sg, tuple(p.info.nf)


CASES = {
    # name: (natoms, box, tilt, qmax, upsampfac)
    "cubic_pow2": (6000, 24.0, (0.0, 0.0, 0.0), 6.0, 0.0),
    "cubic_mixed": (5000, 22.0, (0.0, 0.0, 0.0), 5.0, 1.25),
    "triclinic_mixed": (4000, 20.0, (3.0, 2.0, 1.0), 6.0, 1.3),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", [_lib.PREC_SINGLE, _lib.PREC_DOUBLE])
def test_fused_matches_cufft(name, precision):
    natoms, box, tilt, qmax, ups = CASES[name]
    rng = np.random.default_rng(len(name))
    xy, xz, yz = tilt
    cell = np.array([[box, 0.0, 0.0], [xy, box, 0.0], [xz, yz, box]])
    types = rng.integers(1, 4, size=natoms).astype(np.int32)
    pos = rng.random((2, natoms, 3)) @ cell
    kw = dict(weight=_lib.WEIGHT_NEUTRON, amp_const=np.array([4.149, 5.803, 9.45]), qmin=0.3,
              qmax=qmax, nq=90, partials=True, precision=precision, upsampfac=ups,
              eps=1e-6 if precision == _lib.PREC_SINGLE else 1e-10, want_grid=True)
    a = run(False, pos, types, cell, **kw)
    b = run(True, pos, types, cell, **kw)
    if "mixed" in name:
        assert any(radices(n) - {2} for n in a[3]), a[3]
    fp32 = precision == _lib.PREC_SINGLE
    rtol, atol = (1e-5, 1e-7) if fp32 else (1e-11, 1e-13)
    np.testing.assert_allclose(a[0], b[0], rtol=rtol, atol=atol)
    np.testing.assert_allclose(a[1], b[1], rtol=rtol, atol=atol)
    rtol, atol = (1e-4, 1e-5) if fp32 else (1e-11, 1e-13)
    np.testing.assert_allclose(a[2], b[2], rtol=rtol, atol=atol)


def test_fused_xray_no_partials_and_single_transform():
    rng = np.random.default_rng(12)
    cell = np.eye(3) * 18.0
    types = rng.integers(1, 3, size=3000).astype(np.int32)
    pos = rng.random((1, 3000, 3)) * 18.0
    scheme = WeightScheme.from_options("xray", "1:Si,2:O")
    for kw in (dict(weight=_lib.WEIGHT_XRAY, xray_coef=scheme.xray_rows(2), partials=True),
               dict(weight=_lib.WEIGHT_UNIT, partials=False)):
        kw.update(qmax=7.0, nq=70, precision=_lib.PREC_DOUBLE, eps=1e-10)
        a = run(False, pos, types, cell, **kw)
        b = run(True, pos, types, cell, **kw)
        np.testing.assert_allclose(a[0], b[0], rtol=1e-11, atol=1e-13)
        np.testing.assert_allclose(a[1], b[1], rtol=1e-11, atol=1e-13)
