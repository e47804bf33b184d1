"""Density amplitudes rho_a(q_h) of one frame at reciprocal lattice points
(sqn_density_modes, the per-frame input of sqcalc dyn on a grid) against the
FP64 direct sum of dyn_accumulate (src/sqc_dynamics.f90:860-875, restated as
oracle.direct_density)."""
import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def system(seed, n=3000, types=(1, 2, 5)):
    rng = np.random.default_rng(seed)
    cell = np.array([[23.0, 0.0, 0.0], [1.7, 21.5, 0.0], [-0.9, 2.2, 24.8]])
    origin = np.array([-3.1, 0.4, 7.25])
    s = rng.random((n, 3))
    pos = origin + s @ cell + rng.normal(0, 0.01, (n, 3))  # a few atoms just outside the box
    tid = rng.choice(np.asarray(types, dtype=np.int32), n)
    return cell, origin, pos, tid


def plan(cell, origin, tid, precision, eps, weight=_lib.WEIGHT_UNIT, partials=True, **kw):
    T = int(tid.max())
    amp = np.linspace(0.5, 2.0, T) if weight == _lib.WEIGHT_NEUTRON else None
    return _lib.Plan(cell.reshape(9), origin, tid, ntypes=T, weight=weight, amp_const=amp,
                     qmin=0.5, qmax=QMAX, nq=50, partials=partials, precision=precision,
                     eps=eps, **kw)


QMAX = 5.0


def lattice_points(modes, rng, k=400, cell=None, corners=True):
    """k random lattice points of the plan's mode cube (with cell: only those with
    |q| <= QMAX, the modes a dyn grid asks for), after h = 0, +-e1 and, with
    corners, the cube's extreme points."""
    hm = (np.asarray(modes) - 1) // 2
    h = np.stack([rng.integers(-m, m + 1, 8 * k) for m in hm], axis=1).astype(np.int32)
    if cell is not None:
        B = 2 * np.pi * np.linalg.inv(np.asarray(cell)).T
        h = h[np.linalg.norm(h @ B, axis=1) <= QMAX]
    head = [[0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], [1, 0, 0],
            [-1, 0, 0]]
    if corners:
        head[1:6] = [hm, -hm, [hm[0], -hm[1], 0], [-hm[0], 0, hm[2]], [0, hm[1], -hm[2]]]
    return np.concatenate([np.array(head, dtype=np.int32), h[:k]])


# FP32 accuracy is stated for |q| <= qmax: at the corners of the mode cube
# (|q| up to sqrt(3) qmax) the deconvolution 1/phihat(h1) phihat(h2) phihat(h3)
# amplifies the FP32 rounding of the fine grid well beyond eps.
@pytest.mark.parametrize("precision,eps,tol,corners", [(_lib.PREC_DOUBLE, 1e-12, 1e-9, True),
                                                       (_lib.PREC_SINGLE, 1e-6, 2e-5, False)])
def test_density_modes_vs_direct_sum(precision, eps, tol, corners):
    cell, origin, pos, tid = system(3)
    with plan(cell, origin, tid, precision, eps) as p:
        h = lattice_points(p.info.modes, np.random.default_rng(7), cell=cell, corners=corners)
        rho = p.density_modes(pos, h)
        ref = O.direct_density(pos, tid, cell, h)
        assert rho.shape == ref.shape == (3, len(h))
        # error relative to the largest amplitude of the species (its atom count at h = 0)
        scale = np.abs(ref[:, :1])
        assert np.max(np.abs(rho - ref) / scale) < tol
        # h = 0 is the atom count of each species
        np.testing.assert_allclose(rho[:, 0].real, [np.sum(tid == t) for t in (1, 2, 5)],
                                   rtol=tol)
        # rho(-h) = conj rho(h)
        np.testing.assert_allclose(rho[:, 7], np.conj(rho[:, 6]), rtol=0, atol=tol * scale.max())
        # the accumulators are untouched
        assert p.finalize()[3] == 0


def test_density_modes_device_input_and_repeat():
    import torch
    cell, origin, pos, tid = system(11, n=2000, types=(1, 2))
    with plan(cell, origin, tid, _lib.PREC_DOUBLE, 1e-12, weight=_lib.WEIGHT_NEUTRON) as p:
        h = lattice_points(p.info.modes, np.random.default_rng(1), k=50)
        a = p.density_modes(pos, h)
        b = p.density_modes(torch.tensor(pos, device="cuda"), h)
        # the bin sort's atomic order changes the summation order between calls
        assert np.max(np.abs(a - b)) / len(pos) < 1e-12
        # more modes than the first call grows the request buffers
        h2 = lattice_points(p.info.modes, np.random.default_rng(2), k=900)
        c = p.density_modes(pos, h2)
        ref = O.direct_density(pos, tid, cell, h2)
        assert np.max(np.abs(c - ref)) / len(pos) < 1e-9


def test_density_modes_outside_cube_and_errors():
    cell, origin, pos, tid = system(5, n=500, types=(1, 2))
    with plan(cell, origin, tid, _lib.PREC_DOUBLE, 1e-10) as p:
        hm = (np.asarray(p.info.modes) - 1) // 2
        rho = p.density_modes(pos, np.array([[hm[0] + 1, 0, 0], [0, 0, -hm[2] - 3]]))
        assert np.all(rho == 0)
        with pytest.raises(_lib.SqnError) as e:
            p.density_modes(pos, np.zeros((0, 3), dtype=np.int32))
        assert e.value.code == _lib.ERR_INVALID_ARGUMENT
    # one transform for all species: no per-species amplitudes to return
    with plan(cell, origin, tid, _lib.PREC_DOUBLE, 1e-10, partials=False) as p:
        if p.info.ntransforms != p.info.nspecies:
            with pytest.raises(_lib.SqnError):
                p.density_modes(pos, np.zeros((1, 3), dtype=np.int32))
