"""Powder XRD pattern (--xrd) on the GPU binning against the FP64 direct-sum
restatement of the reference's sums (oracle.direct_xrd: sf_configure_xrd,
sf_accumulate_values, sf_accumulate_xrd_partials, sf_write_xrd), the
reference's own fcc Ni known answer (test/test_sqcalc.py 9d: line ratios
m |F|^2 LP to 1 %, a perfect lattice leaves every other bin empty, the Ni-Ni
column equals the total) and the written table."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib
from sqcalc_b200.dump import read_frames
from sqcalc_b200.synthetic import fcc_solid
from sqcalc_b200.weights import WeightScheme

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GAS = os.path.join(ROOT, "tests", "golden", "gas.dump")


def xrd_plan(frame, scheme, xrd, precision=_lib.PREC_DOUBLE, eps=1e-10, partials=True):
    lam, (lo, hi) = xrd["lam"], xrd["range"]
    qmin = 4.0 * np.pi * np.sin(0.5 * np.radians(lo)) / lam
    qmax = 4.0 * np.pi * np.sin(0.5 * np.radians(hi)) / lam
    T = max(int(frame.type_id.max()), scheme.mapped_types())
    return _lib.Plan(frame.cell.flat(), frame.cell.origin, frame.type_id, ntypes=T,
                     weight=scheme.kind, amp_const=scheme.neutron_b(T) if scheme.kind == 1 else None,
                     xray_coef=scheme.xray_rows(T) if scheme.kind == 2 else None, qmin=qmin,
                     qmax=qmax, nq=40, partials=partials, precision=precision, eps=eps, xrd=xrd)


@pytest.mark.parametrize("weight,lp,step", [("xray", True, 1.0), ("neutron", False, 0.5),
                                            ("xray", True, 0.0)])
def test_xrd_vs_direct_sum(weight, lp, step):
    frames = list(read_frames(GAS))
    f0 = frames[0]
    scheme = WeightScheme.from_options(weight, "1:Si,2:O")
    xrd = dict(lam=1.5406, range=(10.0, 60.0), step=step, lp=lp)
    with xrd_plan(f0, scheme, xrd) as p:
        for f in frames:
            p.accumulate(f.pos)
        tth, I, Ip, cnt, nf = p.xrd()
    T = 2
    w = O.Weights(kind=scheme.kind, amp_const=scheme.neutron_b(T), xray=scheme.xray_rows(T))
    rt, rI, rIp, rcnt, _, _ = O.direct_xrd([f.pos for f in frames], f0.type_id, f0.cell.a,
                                           f0.cell.origin, w, 1.5406, 10.0, 60.0, step, lp, T)
    assert nf == len(frames) and len(tth) == len(rt)
    np.testing.assert_allclose(tth, rt, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(cnt, rcnt)
    scale = max(float(np.max(np.abs(rI))), 1.0)
    assert np.max(np.abs(I - rI)) / scale < 1e-6
    for a in range(T):
        for b in range(a, T):
            assert np.max(np.abs(Ip[a, b] - rIp[a, b])) / scale < 1e-6
    # the pair columns add up to the total
    tot = Ip[0, 0] + Ip[1, 1] + 2 * Ip[0, 1]
    assert np.max(np.abs(tot - I)) / scale < 1e-10


def test_xrd_fp32_close_to_fp64():
    frames = list(read_frames(GAS))
    scheme = WeightScheme.from_options("xray", "1:Si,2:O")
    xrd = dict(lam=1.5406, range=(10.0, 60.0), step=1.0, lp=True)
    out = []
    for prec, eps in ((_lib.PREC_SINGLE, 1e-6), (_lib.PREC_DOUBLE, 1e-10)):
        with xrd_plan(frames[0], scheme, xrd, precision=prec, eps=eps) as p:
            for f in frames:
                p.accumulate(f.pos)
            out.append(p.xrd()[1])
    scale = max(float(np.max(np.abs(out[1]))), 1.0)
    assert np.max(np.abs(out[0] - out[1])) / scale < 1e-4


def test_xrd_fcc_ni_known_answer():
    pos, types, cell = fcc_solid(20, a=3.52, tilt=(0.0, 0.0, 0.0), types_on_basis=(1, 1, 1, 1))
    assert len(types) == 32000
    scheme = WeightScheme.from_options("xray", "1:Ni")

    class Fr:
        pass
    f = Fr()
    f.type_id = types
    from sqcalc_b200.cell import Cell
    f.cell = Cell(a=cell, origin=np.zeros(3))
    xrd = dict(lam=1.541838, range=(40.0, 80.0), step=0.2, lp=True)
    with xrd_plan(f, scheme, xrd) as p:
        p.accumulate(pos)
        tth, I, Ip, cnt, _ = p.xrd()
    assert len(tth) == 200
    assert np.max(np.abs(I - Ip[0, 0]) / np.maximum(np.abs(I), 1.0)) < 1e-9
    a_ = [12.8376, 7.2920, 4.4438, 2.3800]
    b_ = [3.8785, 0.2565, 12.1763, 66.3421]

    def ff(q):
        return 1.0341 + sum(ai * np.exp(-bi * (q / (4.0 * np.pi)) ** 2) for ai, bi in zip(a_, b_))

    lines = [((1, 1, 1), 8), ((2, 0, 0), 6), ((2, 2, 0), 12)]
    want = []
    for hkl, m in lines:
        q = np.sqrt(sum(h * h for h in hkl)) * 2.0 * np.pi / 3.52
        t = O.two_theta_deg(q, 1.541838)
        want.append((t, m * ff(q) ** 2 * O.lorentz_polarization(t)))
    peak = float(I.max())
    for t, v in want:
        j = int(np.argmin(np.abs(tth - t)))
        assert abs(tth[j] - t) <= 0.15
        assert abs(I[j] / peak - v / want[0][1]) <= 0.01 * v / want[0][1]
    assert float(np.sort(I)[-4]) <= 1e-6 * peak


def test_cli_xrd_table(tmp_path):
    out, xo = str(tmp_path / "sq.dat"), str(tmp_path / "p.xrd")
    r = subprocess.run([sys.executable, "-m", "sqcalc_b200", "static", "-i", GAS, "-m", "1:Si,2:O",
                        "--xrd", xo, "--xrd-lambda", "1.5406", "--xrd-range", "10", "60",
                        "--xrd-step", "1", "--nq", "40", "--eps", "1e-10", "-q", out], cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    head = [l for l in open(xo) if l.startswith("#")]
    assert "lambda 1.540600 A" in head[0] and "50 bins" in head[0]
    assert "Lorentz-polarization" in head[1]
    assert head[3].split() == ["#", "2theta[deg]", "I", "I(Si-Si)", "I(Si-O)", "I(O-O)"]
    t = np.loadtxt(xo)
    assert t.shape == (50, 5)
    assert np.max(np.abs(t[:, 2] + 2 * t[:, 3] + t[:, 4] - t[:, 1])) <= 1e-9 * max(1.0, t[:, 1].max())
    r = subprocess.run([sys.executable, "-m", "sqcalc_b200", "static", "-i", GAS, "--xrd", xo,
                        out], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 2 and "xrd-lambda" in r.stderr
