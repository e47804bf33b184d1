"""The CPU oracle against the reference's golden vectors and known answers.

Golden tables: tests/golden/*.dat, written by the reference's own numpy direct
sum (test/ref_sq.py) on dumps from its own generator (test/gen_dump.py), see
tests/golden/make_golden.py.  Known answers: test/test_sqcalc.py sections 9, 9c.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200.dump import read_frames
from sqcalc_b200.weights import WeightScheme

NORMS = {"mean": O.NORM_MEAN, "self": O.NORM_SELF, "n": O.NORM_NATOM}


def load_case(golden_dir, case):
    meta = json.load(open(os.path.join(golden_dir, "cases.json")))
    c = [m for m in meta["cases"] if m["case"] == case][0]
    frames = list(read_frames(os.path.join(golden_dir, c["dump"])))
    return c, frames


def weights_for(c, ntypes):
    s = WeightScheme.from_options(c["weight"], c["mapping"])
    return O.Weights(kind=s.kind, amp_const=s.neutron_b(ntypes), xray=s.xray_rows(ntypes))


def rel_dev(ref, cand):
    return float(np.max(np.abs(cand - ref) / np.maximum(np.abs(ref), 1.0)))


CASES = ["gas_unit_self", "gas_neutron_mean", "gas_xray_mean", "gas_ion_xray_mean",
         "gas_unit_n_window", "tri_unit_self", "lattice_unit_self", "ka_unit_mean"]


@pytest.mark.parametrize("case", CASES)
def test_direct_oracle_matches_reference_numpy(golden_dir, case):
    c, frames = load_case(golden_dir, case)
    f0 = frames[0]
    ntypes = max(int(f0.type_id.max()), 1)
    grid, acc = O.direct_sq([f.pos for f in frames], f0.type_id, f0.cell.a, f0.cell.origin,
                            weights_for(c, ntypes), c["qmin"], c["qmax"], c["nq"],
                            norm=NORMS[c["norm"]])
    ref = np.loadtxt(os.path.join(golden_dir, c["table"]))
    # ref_sq.py prints 12 significant digits: agreement to ~1e-11 pins the
    # grid, the shells, the weights and the normalisation bit for bit.
    assert rel_dev(ref[:, 1], acc.shell_value()) < 1e-10
    dq = (c["qmax"] - c["qmin"]) / c["nq"]
    assert np.allclose(ref[:, 0], c["qmin"] + (np.arange(c["nq"]) + 0.5) * dq, atol=5e-7)


def test_partial_sum_rule_and_limits(golden_dir):
    # test/test_sqcalc.py:758-783: S = Saa + 2Sab + Sbb to 1e-9, high-q limits.
    c, frames = load_case(golden_dir, "gas_unit_n_window")
    f0 = frames[0]
    grid, acc = O.direct_sq([f.pos for f in frames], f0.type_id, f0.cell.a, f0.cell.origin,
                            O.Weights(), 0.5, 5.9, 27, norm=O.NORM_NATOM)
    S = acc.shell_value()
    s11, s12, s22 = acc.partial_value(1, 1), acc.partial_value(1, 2), acc.partial_value(2, 2)
    assert np.max(np.abs(S - (s11 + 2 * s12 + s22))) < 1e-9
    q = 0.5 + (np.arange(27) + 0.5) * (5.4 / 27)
    hi = q > 3.0
    assert abs(np.mean(s11[hi]) - 0.5) < 0.05
    assert np.mean(np.abs(s12[hi])) < 0.1
    a12 = acc.partial_value(1, 2, faber_ziman=True)
    assert abs(np.mean(a12[hi]) - 1.0) < 0.05


def test_bragg_shell_known_answer():
    # test/test_sqcalc.py:912-931: simple-cubic 32^3 lattice, L = 20; the
    # <100> Bragg shell holds S = N = 32768 and S(q) = S(a-a).
    side, L = 32, 20.0
    g = np.arange(side) * (L / side)
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    types = np.ones(len(pos), dtype=np.int32)
    grid, acc = O.direct_sq([pos], types, np.eye(3) * L, np.zeros(3), O.Weights(), 10.05,
                            10.056, 1, norm=O.NORM_NATOM)
    assert grid.nmodes == 6
    S = acc.shell_value()[0]
    assert abs(S - 32768.0) / 32768.0 < 1e-6
    assert abs(S - acc.partial_value(1, 1)[0]) / S < 1e-9


def test_nufft_cpu_restatement_matches_direct(golden_dir):
    c, frames = load_case(golden_dir, "ka_unit_mean")
    f0 = frames[0]
    pos = [f.pos for f in frames]
    _, d = O.direct_sq(pos, f0.type_id, f0.cell.a, f0.cell.origin, O.Weights(), 0.0, 6.0, 120)
    for sigma in (1.25, 2.0):
        _, n, info = O.nufft_cpu_sq(pos, f0.type_id, f0.cell.a, f0.cell.origin, O.Weights(), 0.0,
                                    6.0, 120, eps=1e-10, sigma=sigma)
        assert rel_dev(d.shell_value(), n.shell_value()) < 1e-8, info
        for a, b in ((1, 1), (1, 2), (2, 2)):
            assert rel_dev(d.partial_value(a, b), n.partial_value(a, b)) < 1e-8


def test_enumeration_counts_match_reference_formula():
    # modes = 2 ceil(qmax |a| / 2pi) + 1 (:336-337): the headline box gives 423.
    g = O.configure_grid(np.eye(3) * 220.0, 0.0, 0.2, 4)
    assert list(g.modes) == [17, 17, 17]  # 0.2*220/2pi = 7.003 -> 2*8+1
    m = np.zeros(3, dtype=np.int32)
    O.lib().sqo_modes(np.ascontiguousarray((np.eye(3) * 220.0).reshape(9)), 6.0, m)
    assert list(m) == [423, 423, 423]


def test_xrd_conversions_known_answers():
    # the reference's own checks of the two-theta and LP conversions
    # (test/test_xrd.f90): fcc Ni (a = 3.52 A) reflections at Cu Kalpha
    lam = 1.541838
    for hkl, want in (((1, 1, 1), 44.585405), ((2, 0, 0), 51.955510), ((2, 2, 0), 76.552967)):
        q = np.sqrt(sum(h * h for h in hkl)) * 2.0 * np.pi / 3.52
        assert abs(O.two_theta_deg(q, lam) - want) / want < 1e-7
    q = 4.0 * np.pi * np.sin(np.pi / 8.0) / lam
    assert abs(O.two_theta_deg(q, lam) - 45.0) < 1e-9
    assert O.two_theta_deg(1e9, lam) == 180.0
    assert abs(O.lorentz_polarization(90.0) - 2.0 * np.sqrt(2.0)) < 1e-12
    assert O.lorentz_polarization(1.0) > O.lorentz_polarization(90.0) < O.lorentz_polarization(179.0)


@pytest.mark.parametrize("norm", [O.NORM_MEAN, O.NORM_SELF, O.NORM_NATOM])
def test_separable_direct_sum_equals_direct_sum(norm):
    """oracle.direct_sq_separable (the direct sum as per-axis phase products,
    used where the per-mode loop is too slow) against oracle.direct_sq on a
    triclinic cell with an offset origin: identical kept modes and shells, S and
    the partials to ~1e-13."""
    rng = np.random.default_rng(3)
    cell = np.array([[14.0, 0, 0], [2.0, 13.0, 0], [1.0, 1.5, 12.0]])
    n = 300
    tid = rng.integers(1, 4, size=n).astype(np.int32)
    frames = [rng.random((n, 3)) @ cell + rng.normal(0, 1, (n, 3)) for _ in range(2)]
    w = O.Weights(kind=O.WEIGHT_NEUTRON, amp_const=np.array([4.1, 5.8, 9.4]))
    origin = np.array([0.5, -1.0, 2.0])
    _, a = O.direct_sq(frames, tid, cell, origin, w, 0.3, 5.0, 60, norm=norm)
    _, b = O.direct_sq_separable(frames, tid, cell, origin, w, 0.3, 5.0, 60, norm=norm)
    np.testing.assert_array_equal(a.shell_count, b.shell_count)
    np.testing.assert_allclose(b.den, a.den, rtol=1e-13)
    assert np.max(np.abs(a.shell_value() - b.shell_value())) < 1e-12
    for i in (1, 2, 3):
        for j in range(i, 4):
            assert np.max(np.abs(a.partial_value(i, j) - b.partial_value(i, j))) < 1e-12
