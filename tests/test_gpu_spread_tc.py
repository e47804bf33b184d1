"""Tensor-core spread (SQN_FLAG_SPREAD_TC: tcgen05 3xTF32, FP32 plans) against
the CUDA-core spread (the default) of the same plan: S(q), the partials and the per-mode
grid for 1 to 4 transforms, neutron and x-ray amplitudes, grids with partial
tiles, and several frames; and against the FP64 plan."""
import numpy as np
import pytest

from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def system(n, L, types, seed):
    rng = np.random.default_rng(seed)
    tid = rng.choice(np.asarray(types, dtype=np.int32), n)
    cell = np.array([[L, 0.0, 0.0], [0.3, L * 0.93, 0.0], [-0.5, 0.8, L * 1.07]])
    frames = [rng.random((n, 3)) @ cell for _ in range(3)]
    return cell, tid, frames


def mk(cell, tid, tc, precision=_lib.PREC_SINGLE, weight=_lib.WEIGHT_NEUTRON, partials=True,
       qmax=7.0, grid=False, eps=1e-6):
    T = int(tid.max())
    amp = np.linspace(3.0, 9.0, T)
    coef = np.array([[2.0 + t, 1.5, 1.0, 0.5, 10.0, 5.0, 1.0, 0.2, 0.3] for t in range(T)])
    return _lib.Plan(cell.reshape(9), np.array([0.5, -1.0, 2.0]), tid, ntypes=T, weight=weight,
                     amp_const=amp if weight == _lib.WEIGHT_NEUTRON else None,
                     xray_coef=coef if weight == _lib.WEIGHT_XRAY else None, qmin=0.3,
                     qmax=qmax, nq=150, partials=partials, want_grid=grid, precision=precision,
                     eps=eps, spread_tc=tc)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


@pytest.mark.parametrize("types,weight,partials", [
    ((1,), _lib.WEIGHT_NEUTRON, True),
    ((1, 2), _lib.WEIGHT_NEUTRON, True),
    ((1, 2, 3), _lib.WEIGHT_XRAY, True),
    ((1, 2, 3, 4), _lib.WEIGHT_NEUTRON, True),
    ((1, 2, 3), _lib.WEIGHT_NEUTRON, False),
])
def test_tensor_core_spread_matches_cuda_core_spread(types, weight, partials):
    cell, tid, frames = system(7000, 37.0, types, seed=len(types))
    with mk(cell, tid, True, weight=weight, partials=partials, grid=True) as pt, \
            mk(cell, tid, False, weight=weight, partials=partials, grid=True) as ps:
        for p in (pt, ps):
            for f in frames:
                p.accumulate(f)
        a, b = pt.finalize(grid=True), ps.finalize(grid=True)
        assert a[3] == b[3] == len(frames)
        assert rel(a[0], b[0]) < 2e-6
        assert rel(a[1], b[1]) < 2e-6
        assert rel(a[2], b[2]) < 2e-5


def test_tensor_core_spread_against_fp64_at_benchmark_like_density():
    cell, tid, frames = system(60000, 80.0, (1, 2, 3), seed=9)
    with mk(cell, tid, True, eps=1e-6) as pt, \
            mk(cell, tid, False, precision=_lib.PREC_DOUBLE, eps=1e-12) as pd:
        for p in (pt, pd):
            for f in frames[:2]:
                p.accumulate(f)
        a, b = pt.finalize(), pd.finalize()
        assert rel(a[0], b[0]) < 1e-5
        assert rel(a[1], b[1]) < 1e-5
