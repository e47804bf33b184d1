"""The cuFINUFFT-shaped type-1 entry points against the direct type-1 sum
(the check FINUFFT's own tests use, external/finufft/test/utils/dirft3d.hpp:13-20):
relative l2 error <= 10 eps in FP64 (eps 1e-10) and <= 10 eps in FP32 (eps 1e-5),
for both signs, both mode orders, odd and even mode counts, several transforms,
points outside [-pi, pi) (periodic) and repeated setpts."""
import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib

pytestmark = pytest.mark.gpu


def points(M, seed, span=1.0):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.random((3, M)) * 2 - 1) * np.pi * span
    c = rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))
    return x, y, z, c


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("precision,eps", [(_lib.PREC_DOUBLE, 1e-10), (_lib.PREC_SINGLE, 1e-5)])
@pytest.mark.parametrize("iflag,modeord", [(1, 0), (-1, 0), (1, 1)])
def test_type1_vs_direct(precision, eps, iflag, modeord):
    import torch
    x, y, z, c = points(2500, seed=3 + iflag + 5 * modeord, span=3.0)
    nm = (24, 17, 20)
    ref = O.dirft3d1(x, y, z, c, nm, iflag=iflag, modeord=modeord)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    with _lib.Type1Plan(nm, iflag=iflag, ntransf=2, eps=eps, precision=precision,
                        modeord=modeord) as p:
        p.setpts(dev(x), dev(y), dev(z))
        fk = p.execute(dev(c)).cpu().numpy()
    assert fk.shape == ref.shape
    assert rel_l2(fk, ref) < 10 * eps, rel_l2(fk, ref)


def test_type1_setpts_again_and_bad_arguments():
    import torch
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    nm = (16, 16, 16)
    with _lib.Type1Plan(nm, iflag=1, ntransf=1, eps=1e-9) as p:
        for M, seed in ((500, 1), (3000, 2), (200, 3)):
            x, y, z, c = points(M, seed)
            p.setpts(dev(x), dev(y), dev(z))
            fk = p.execute(dev(c[:1])).cpu().numpy()
            ref = O.dirft3d1(x, y, z, c[:1], nm, iflag=1)
            assert rel_l2(fk, ref) < 1e-8
    with pytest.raises(_lib.SqnError):
        _lib.Type1Plan(nm, nufft_type=2)
    with pytest.raises(_lib.SqnError):
        _lib.Type1Plan(nm, dim=2)
    with pytest.raises(_lib.SqnError):
        _lib.Type1Plan((0, 4, 4))
