"""dS(q)/dr through the adjoint (type-2 NUFFT) against the FP64 direct-sum
gradient, central finite differences and torch autograd.

The differentiation form: 2 types 1:2, uniform positions, loss over shells with
q in [0.5, 8] 1/A; the FP64 direct-sum check runs on an N = 2000, L = 30 A
system.  Tolerance: 1e-6 relative (max |d| / max |g_ref|) for FP64.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def system(n=2000, box=30.0, seed=17):
    rng = np.random.default_rng(seed)
    types = np.repeat([1, 2], [n // 3, n - n // 3]).astype(np.int32)
    rng.shuffle(types)
    return rng.random((n, 3)) * box, types, np.eye(3) * box


def make_plan(types, box, precision=_lib.PREC_DOUBLE, eps=1e-12, nq=150, weight=_lib.WEIGHT_UNIT,
              amp=None):
    return _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), types, weight=weight,
                     amp_const=amp, qmin=0.5, qmax=8.0, nq=nq, norm=_lib.NORM_MEAN,
                     partials=True, precision=precision, eps=eps, grad=True)


def reference_grad(pos, types, cell, plan, dLdS, strength):
    grid = O.configure_grid(cell, 0.5, 8.0, plan.nq)
    den = plan.accumulators()["den"]
    wgt = np.where(den > 0, dLdS / np.where(den > 0, den, 1.0), 0.0)
    return O.direct_grad(pos, strength, cell, np.zeros(3), grid, wgt)


def test_single_frame_S_matches_accumulate():
    pos, types, cell = system()
    with make_plan(types, 30.0) as plan:
        S1, _ = plan.sq_grad(pos)
        plan.accumulate(pos)
        S2 = plan.finalize()[0]
    assert np.max(np.abs(S1 - S2) / np.maximum(np.abs(S2), 1.0)) < 1e-9


@pytest.mark.parametrize("weight", ["unit", "neutron"])
def test_grad_vs_direct_sum_fp64(weight):
    pos, types, cell = system()
    rng = np.random.default_rng(3)
    if weight == "unit":
        kw, strength = {}, np.ones(len(types))
    else:
        b = np.array([4.149, 5.803])
        kw = dict(weight=_lib.WEIGHT_NEUTRON, amp=b)
        strength = b[types - 1]
    with make_plan(types, 30.0, **kw) as plan:
        dLdS = rng.standard_normal(plan.nq)
        _, g = plan.sq_grad(pos, dLdS)
        ref = reference_grad(pos, types, cell, plan, dLdS, strength)
    err = np.max(np.abs(g - ref)) / np.max(np.abs(ref))
    assert err < 1e-6, err


def test_grad_fp32_vs_direct_sum():
    """FP32 spread / FFT / interpolation (eps 1e-6) with FP64 accumulation: within
    1e-5 relative of the FP64 direct-sum gradient (measured ~4.5e-6: FP32 does
    not meet the 1e-6 bar, the FP64 adjoint above does)."""
    pos, types, cell = system(n=1500, seed=5)
    with make_plan(types, 30.0, precision=_lib.PREC_SINGLE, eps=1e-6) as plan:
        dLdS = np.random.default_rng(9).standard_normal(plan.nq)
        _, g = plan.sq_grad(pos, dLdS)
        ref = reference_grad(pos, types, cell, plan, dLdS, np.ones(len(types)))
    err = np.max(np.abs(g - ref)) / np.max(np.abs(ref))
    assert err < 1e-5, err


def test_grad_vs_central_differences():
    # central FD with h = 1e-4 A in FP64 on a few coordinates
    pos, types, cell = system(n=600, box=20.0, seed=23)
    h = 1e-4
    rng = np.random.default_rng(4)
    with make_plan(types, 20.0) as plan:
        S0, _ = plan.sq_grad(pos)
        target = S0 + 0.05 * rng.standard_normal(plan.nq)
        loss = lambda S: float(np.sum((S - target) ** 2))  # noqa: E731
        _, g = plan.sq_grad(pos, 2.0 * (S0 - target))
        for (j, r) in [(0, 0), (5, 1), (17, 2), (123, 0), (599, 2)]:
            p1, p2 = pos.copy(), pos.copy()
            p1[j, r] += h
            p2[j, r] -= h
            fd = (loss(plan.sq_grad(p1)[0]) - loss(plan.sq_grad(p2)[0])) / (2 * h)
            assert abs(fd - g[j, r]) <= 2e-5 * np.max(np.abs(g)), (j, r, fd, g[j, r])


def test_torch_autograd_matches_adjoint():
    import torch
    from sqcalc_b200.autograd import structure_factor

    pos, types, cell = system(n=800, box=22.0, seed=31)
    with make_plan(types, 22.0) as plan:
        target = torch.ones(plan.nq, dtype=torch.float64, device="cuda")
        x = torch.tensor(pos, dtype=torch.float64, device="cuda", requires_grad=True)
        S = structure_factor(x, plan)
        loss = ((S - target) ** 2).sum()
        loss.backward()
        S_np = S.detach().cpu().numpy()
        _, g = plan.sq_grad(pos, 2.0 * (S_np - 1.0))
        xc = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
        Sc = structure_factor(xc, plan)
        ((Sc - 1.0) ** 2).sum().backward()
    assert np.max(np.abs(x.grad.cpu().numpy() - g)) <= 1e-12 * np.max(np.abs(g)) + 1e-300
    assert np.max(np.abs(xc.grad.numpy() - g)) <= 1e-12 * np.max(np.abs(g)) + 1e-300


def test_grad_needs_flag_and_q_independent_weights():
    pos, types, cell = system(n=100, box=10.0)
    with _lib.Plan(np.eye(3).reshape(9) * 10.0, np.zeros(3), types, qmax=4.0, nq=20) as plan:
        with pytest.raises(_lib.SqnError):
            plan.sq_grad(pos)
    with pytest.raises(_lib.SqnError):
        _lib.Plan(np.eye(3).reshape(9) * 10.0, np.zeros(3), types, qmax=4.0, nq=20,
                  weight=_lib.WEIGHT_XRAY, xray_coef=np.ones((2, 9)), grad=True)
