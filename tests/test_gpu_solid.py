"""Structured solid with x-ray weights: a triclinic FCC crystal (a = 4 A, tilts
xy = 5 A, xz = 3 A), two types alternating on the sublattices, Gaussian thermal
displacement sigma = 0.1 A, IT92 x-ray form factors (src/sqc_elements.f90:226-239).

Small crystals are checked against the FP64 direct sum.  The full 64^3-cell
crystal (N = 1,048,576, q_max = 10: 817^3 modes) is above the reference's
mode cap of 4e8 (src/sqc_structure_factor.f90:340-345), so the plan refuses it
by default and accepts it with max_grid_modes raised; its FP32 Bragg peaks are
then checked against the FP64 path at eps 1e-10.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib
from sqcalc_b200.synthetic import fcc_solid, thermal_frames
from sqcalc_b200.weights import WeightScheme

pytestmark = pytest.mark.gpu

SCHEME = WeightScheme.from_options("xray", "1:Cu,2:Au")


def plan_for(pos, types, cell, precision, eps, qmax, nq, max_grid_modes=0):
    return _lib.Plan(cell.reshape(9), np.zeros(3), types, ntypes=2, weight=_lib.WEIGHT_XRAY,
                     xray_coef=SCHEME.xray_rows(2), qmin=0.0, qmax=qmax, nq=nq,
                     norm=_lib.NORM_MEAN, partials=True, precision=precision, eps=eps,
                     max_grid_modes=max_grid_modes)


@pytest.mark.parametrize("precision,eps,tol", [(_lib.PREC_DOUBLE, 1e-10, 1e-6),
                                               (_lib.PREC_SINGLE, 1e-6, 1e-4)])
def test_small_fcc_vs_direct_sum(precision, eps, tol):
    pos0, types, cell = fcc_solid(5)
    frames = thermal_frames(pos0, 0.1, 2, seed=55)
    w = O.Weights(kind=O.WEIGHT_XRAY, xray=SCHEME.xray_rows(2))
    _, acc = O.direct_sq(frames, types, cell, np.zeros(3), w, 0.0, 8.0, 160, ntypes=2)
    ref = acc.shell_value()
    with plan_for(pos0, types, cell, precision, eps, 8.0, 160) as p:
        for f in frames:
            p.accumulate(f)
        S, Sp, _, n = p.finalize()
    assert n == 2
    scale = np.maximum(np.abs(ref), 1.0)
    assert np.max(np.abs(S - ref) / scale) < tol
    for a in (1, 2):
        for b in (1, 2):
            r = acc.partial_value(a, b)
            assert np.max(np.abs(Sp[a - 1, b - 1] - r) / np.maximum(np.abs(r), 1.0)) < tol
    # the strongest shells are Bragg peaks, far above the diffuse background
    top = np.argsort(ref)[-5:]
    assert np.all(ref[top] > 5.0)
    assert np.max(np.abs(S[top] - ref[top]) / ref[top]) < tol


def test_full_crystal_refused_by_default_then_run_with_cap_raised():
    import gc
    pos0, types, cell = fcc_solid(64)
    assert len(types) == 1_048_576
    with pytest.raises(_lib.SqnError) as e:
        plan_for(pos0, types, cell, _lib.PREC_SINGLE, 1e-6, 10.0, 500)
    assert e.value.code == 42
    frame = thermal_frames(pos0, 0.1, 1, seed=77)[0]
    out = {}
    for name, prec, eps in (("f32", _lib.PREC_SINGLE, 1e-6), ("f64", _lib.PREC_DOUBLE, 1e-10)):
        with plan_for(pos0, types, cell, prec, eps, 10.0, 500, max_grid_modes=-1) as p:
            assert p.modes == (817, 817, 817)
            assert p.gridpoints == 817 ** 3
            p.accumulate(frame)
            S, Sp, _, n = p.finalize()
            out[name] = (S, Sp)
        gc.collect()
    S32, Sp32 = out["f32"]
    S64, Sp64 = out["f64"]
    scale = np.maximum(np.abs(S64), 1.0)
    assert np.max(np.abs(S32 - S64) / scale) < 1e-4
    top = np.argsort(S64)[-10:]
    assert np.all(S64[top] > 5.0)  # Bragg shells, well above the diffuse level
    assert np.max(np.abs(S32[top] - S64[top]) / S64[top]) < 1e-5
    assert np.max(np.abs(Sp32 - Sp64) / np.maximum(np.abs(Sp64), 1.0)) < 1e-4
