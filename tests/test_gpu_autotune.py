"""SQN_FLAG_AUTOTUNE: the plan times its candidate (sigma, w) pairs on its own
shape and keeps the fastest.  The tuned plan must still meet the accuracy bar
(FP64 direct sum, rtol 1e-6 as test/test_sqcalc.py:389-396), report how it was
tuned, and a second plan of the same shape must reuse the cached choice."""
import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def test_autotuned_plan_meets_the_bar_and_caches():
    rng = np.random.default_rng(5)
    box, n, qmax, nq = 18.0, 3000, 7.0, 120
    tid = rng.integers(1, 3, size=n).astype(np.int32)
    frames = [rng.random((n, 3)) * box for _ in range(2)]
    kw = dict(qmin=0.0, qmax=qmax, nq=nq, norm=_lib.NORM_MEAN, partials=True,
              precision=_lib.PREC_DOUBLE, eps=1e-10, autotune=True)
    cell = np.eye(3).reshape(9) * box
    with _lib.Plan(cell, np.zeros(3), tid, **kw) as p:
        info = p.info
        assert info.autotuned == 1 and info.tune_candidates >= 2 and info.tune_ms > 0
        for f in frames:
            p.accumulate(f)
        S, Sp, _, _ = p.finalize()
        chosen = (tuple(info.nf), info.kernel_width)
    _, acc = O.direct_sq(frames, tid, np.eye(3) * box, np.zeros(3), O.Weights(), 0.0, qmax, nq)
    ref = acc.shell_value()
    assert np.max(np.abs(S - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-6
    for a in (1, 2):
        for b in range(a, 3):
            assert np.max(np.abs(Sp[a - 1, b - 1] - acc.partial_value(a, b))) < 1e-6
    with _lib.Plan(cell, np.zeros(3), tid, **kw) as q:
        assert q.info.autotuned == 1 and q.info.tune_candidates == 0  # from the cache
        assert (tuple(q.info.nf), q.info.kernel_width) == chosen


def test_autotuned_gradient_plan_meets_the_bar():
    """A dS/dr plan tuned on its gradient evaluation: FP64 gradient within 1e-6
    relative of the FP64 direct-sum gradient (the differentiation form's bar)."""
    rng = np.random.default_rng(17)
    n, box = 2000, 30.0
    types = np.repeat([1, 2], [n // 3, n - n // 3]).astype(np.int32)
    rng.shuffle(types)
    pos = rng.random((n, 3)) * box
    with _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), types, qmin=0.5, qmax=8.0, nq=150,
                   norm=_lib.NORM_MEAN, partials=True, precision=_lib.PREC_DOUBLE, eps=1e-12,
                   grad=True, autotune=True) as plan:
        assert plan.info.autotuned == 1
        dLdS = rng.standard_normal(plan.nq)
        _, g = plan.sq_grad(pos, dLdS)
        den = plan.accumulators()["den"]
    grid = O.configure_grid(np.eye(3) * box, 0.5, 8.0, 150)
    wgt = np.where(den > 0, dLdS / np.where(den > 0, den, 1.0), 0.0)
    ref = O.direct_grad(pos, np.ones(n), np.eye(3) * box, np.zeros(3), grid, wgt)
    assert np.max(np.abs(g - ref)) / np.max(np.abs(ref)) < 1e-6
