"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Tolerances are the reference's own (test/test_sqcalc.py): NUFFT vs direct
rtol 1e-6 as max|d|/max(|ref|, 1); FP32 vs FP64 rtol 1e-4 (:398-404); the sum
rule 1e-9 and a<->b symmetry 1e-12 (:755-800); the Bragg shell S = N to 1e-6
(:912-931).  The FP32 form must also meet max |dS| <= 1e-5 against the FP64
oracle at eps = 1e-6.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from sqcalc_b200 import _lib
from sqcalc_b200.cell import Cell
from sqcalc_b200.dump import read_frames
from sqcalc_b200.static import GpuStructureFactor, SqcalcError
from sqcalc_b200.weights import WeightScheme

pytestmark = pytest.mark.gpu

NORMS = {"mean": O.NORM_MEAN, "self": O.NORM_SELF, "n": O.NORM_NATOM}


class F:  # minimal frame for synthetic inputs
    def __init__(self, pos, types, cell):
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.type_id = np.ascontiguousarray(types, dtype=np.int32)
        self.natoms = len(types)
        self.cell = cell


def rel_dev(ref, cand):
    return float(np.max(np.abs(np.asarray(cand) - ref) / np.maximum(np.abs(ref), 1.0)))


def gpu_run(frames, scheme, **kw):
    m = GpuStructureFactor(**kw)
    m.configure(frames[0], scheme)
    for f in frames:
        m.accumulate_frame(f)
    S, Sp, Sg, nf = m.results()
    assert nf == len(frames)
    assert m.plan.launch_count() >= 5 * len(frames)
    m.close()
    return S, Sp, Sg


def oracle_run(frames, scheme, qmin, qmax, nq, norm, want_grid=False):
    f0 = frames[0]
    ntypes = max(int(f0.type_id.max()), scheme.mapped_types(), 1)
    w = O.Weights(kind=scheme.kind, amp_const=scheme.neutron_b(ntypes),
                  xray=scheme.xray_rows(ntypes))
    return O.direct_sq([f.pos for f in frames], f0.type_id, f0.cell.a, f0.cell.origin, w, qmin,
                       qmax, nq, norm=NORMS[norm], want_grid=want_grid, ntypes=ntypes)


def load_case(golden_dir, case):
    meta = json.load(open(os.path.join(golden_dir, "cases.json")))
    c = [m for m in meta["cases"] if m["case"] == case][0]
    return c, list(read_frames(os.path.join(golden_dir, c["dump"])))


CASES = ["gas_unit_self", "gas_neutron_mean", "gas_xray_mean", "gas_ion_xray_mean",
         "gas_unit_n_window", "tri_unit_self", "lattice_unit_self", "ka_unit_mean"]


@pytest.mark.parametrize("case", CASES)
def test_golden_tables_fp64(golden_dir, case):
    c, frames = load_case(golden_dir, case)
    scheme = WeightScheme.from_options(c["weight"], c["mapping"])
    S, _, _ = gpu_run(frames, scheme, norm=c["norm"], qmin=c["qmin"], qmax=c["qmax"],
                      nq=c["nq"], eps=1e-10)
    ref = np.loadtxt(os.path.join(golden_dir, c["table"]))
    assert rel_dev(ref[:, 1], S) < 1e-6


@pytest.mark.parametrize("weight,norm", [("unit", "self"), ("neutron", "mean"), ("xray", "mean")])
def test_partials_vs_direct_oracle(golden_dir, weight, norm):
    c, frames = load_case(golden_dir, "gas_unit_self")
    scheme = WeightScheme.from_options(weight, "1:Si,2:O")
    S, Sp, _ = gpu_run(frames, scheme, norm=norm, qmax=6.0, nq=40, eps=1e-10)
    _, acc = oracle_run(frames, scheme, 0.0, 6.0, 40, norm)
    assert rel_dev(acc.shell_value(), S) < 1e-6
    for a, b in ((1, 1), (1, 2), (2, 2)):
        assert rel_dev(acc.partial_value(a, b), Sp[a - 1, b - 1]) < 1e-6


def test_sum_rule_symmetry_and_fz(golden_dir):
    _, frames = load_case(golden_dir, "gas_unit_self")
    kw = dict(norm="n", qmin=0.5, qmax=5.9, nq=27, eps=1e-10)
    S, Sp, _ = gpu_run(frames, WeightScheme.from_options("unit", "1:Si,2:O"), **kw)
    assert np.max(np.abs(S - (Sp[0, 0] + 2 * Sp[0, 1] + Sp[1, 1]))) < 1e-9
    _, Sw, _ = gpu_run(frames, WeightScheme.from_options("unit", "1:O,2:Si"), **kw)
    assert np.max(np.abs(Sw[0, 1] - Sp[0, 1])) < 1e-12
    _, Afz, _ = gpu_run(frames, WeightScheme.from_options("unit", "1:Si,2:O"),
                        faber_ziman=True, **kw)
    q = 0.5 + (np.arange(27) + 0.5) * (5.4 / 27)
    assert abs(np.mean(Afz[0, 1][q > 3.0]) - 1.0) < 0.05


def test_sparse_type_ids_match_dense(golden_dir):
    # test/test_sqcalc.py:840-876: types 1 and 3 of 3 give the same columns.
    _, frames = load_case(golden_dir, "gas_unit_self")
    dense = gpu_run(frames, WeightScheme.from_options("unit", "1:Si,2:O"), qmax=6, nq=30,
                    eps=1e-10)
    sparse_frames = [F(f.pos, np.where(f.type_id == 2, 3, f.type_id), f.cell) for f in frames]
    sparse = gpu_run(sparse_frames, WeightScheme.from_options("unit", "1:Si,3:O"), qmax=6,
                     nq=30, eps=1e-10)
    assert np.max(np.abs(dense[0] - sparse[0])) < 1e-12
    assert np.max(np.abs(dense[1][0, 1] - sparse[1][0, 2])) < 1e-12
    assert np.max(np.abs(sparse[1][0, 2])) > 0


def test_single_species_total_equals_partial():
    rng = np.random.default_rng(5)
    cell = Cell.cubic(20.0)
    frames = [F(rng.random((400, 3)) * 20.0, np.ones(400), cell) for _ in range(3)]
    S, Sp, _ = gpu_run(frames, WeightScheme.from_options("unit"), norm="n", qmax=6, nq=60,
                       eps=1e-10)
    assert rel_dev(S, Sp[0, 0]) < 1e-6


def test_bragg_shell_fp64():
    side, L = 32, 20.0
    g = np.arange(side) * (L / side)
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    frames = [F(pos, np.ones(len(pos)), Cell.cubic(L))]
    S, Sp, _ = gpu_run(frames, WeightScheme.from_options("unit"), norm="n", qmin=10.05,
                       qmax=10.056, nq=1, eps=1e-10)
    assert abs(S[0] - 32768.0) / 32768.0 < 1e-6
    assert abs(S[0] - Sp[0, 0, 0]) / S[0] < 1e-9


def test_grid_table_vs_oracle(golden_dir):
    _, frames = load_case(golden_dir, "gas_unit_self")
    scheme = WeightScheme.from_options("unit", "1:Si,2:O")
    _, _, Sg = gpu_run(frames, scheme, norm="self", qmax=6.0, nq=40, eps=1e-10, want_grid=True)
    grid, acc = oracle_run(frames, scheme, 0.0, 6.0, 40, "self", want_grid=True)
    ref = acc.grid_value(grid)
    assert Sg.shape == ref.shape
    assert rel_dev(ref, Sg) < 1e-6


def test_fp32_form_within_budget(golden_dir):
    # the FP32 precision form (FP32 spread/FFT, FP64 accumulation): max |dS| <= 1e-5.
    _, frames = load_case(golden_dir, "ka_unit_mean")
    scheme = WeightScheme.from_options("neutron", "1:Si,2:O")
    S, Sp, _ = gpu_run(frames, scheme, norm="mean", qmax=6.0, nq=120, eps=1e-6,
                       precision="single")
    _, acc = oracle_run(frames, scheme, 0.0, 6.0, 120, "mean")
    ref = acc.shell_value()
    assert float(np.max(np.abs(S - ref))) <= 1e-5
    assert rel_dev(ref, S) < 1e-4
    for a, b in ((1, 1), (1, 2), (2, 2)):
        assert float(np.max(np.abs(Sp[a - 1, b - 1] - acc.partial_value(a, b)))) <= 1e-5


def test_fp32_default_eps_matches_reference_rtol(golden_dir):
    # app/main.f90:191-198: float32 without --eps runs at 1e-5; rtol 1e-4 vs FP64.
    c, frames = load_case(golden_dir, "gas_unit_self")
    scheme = WeightScheme.from_options("unit", "1:Si,2:O")
    S, _, _ = gpu_run(frames, scheme, norm="self", qmax=6.0, nq=40, precision="single")
    _, acc = oracle_run(frames, scheme, 0.0, 6.0, 40, "self")
    assert rel_dev(acc.shell_value(), S) < 1e-4


def test_config1_box_fp64():
    # Plain FP64 form: L = 20, N = 8000 (2667 / 5333 shuffled), 65^3 modes,
    # eps 1e-9, qmax 10, nq 500, unit weights, norm mean, partials.
    rng = np.random.default_rng(2024)
    types = np.repeat([1, 2], [2667, 5333]).astype(np.int32)
    rng.shuffle(types)
    cell = Cell.cubic(20.0)
    frames = [F(rng.random((8000, 3)) * 20.0, types, cell) for _ in range(2)]
    scheme = WeightScheme.from_options("unit")
    S, Sp, _ = gpu_run(frames, scheme, norm="mean", qmax=10.0, nq=500, eps=1e-9)
    grid, acc = oracle_run(frames, scheme, 0.0, 10.0, 500, "mean")
    assert tuple(grid.modes) == (65, 65, 65)
    dS = float(np.max(np.abs(S - acc.shell_value())))
    assert dS < 1e-8, dS
    for a, b in ((1, 1), (1, 2), (2, 2)):
        assert float(np.max(np.abs(Sp[a - 1, b - 1] - acc.partial_value(a, b)))) < 1e-8


def test_wraparound_edges_and_triclinic():
    # Atoms on and just inside every face, outside the box and at negative
    # coordinates: the spread must wrap its support across the periodic edges.
    rng = np.random.default_rng(11)
    cell = Cell.from_bounds([0.0, 0.0, 0.0], [18.0, 17.0, 16.0], [1.5, 0.5, -2.0])
    base = rng.random((300, 3))
    base[:20, 0] = 0.0
    base[20:40, 1] = 1.0 - 1e-13
    base[40:60, 2] = 1.0
    base[60:80] = -base[60:80] * 3.0
    pos = base @ cell.a + cell.origin
    types = rng.integers(1, 4, size=300).astype(np.int32)
    frames = [F(pos, types, cell)]
    scheme = WeightScheme.from_options("xray", "1:Si,2:O,3:Na")
    S, Sp, _ = gpu_run(frames, scheme, norm="mean", qmax=7.0, nq=50, eps=1e-10)
    _, acc = oracle_run(frames, scheme, 0.0, 7.0, 50, "mean")
    assert rel_dev(acc.shell_value(), S) < 1e-6
    for a in range(1, 4):
        for b in range(a, 4):
            assert rel_dev(acc.partial_value(a, b), Sp[a - 1, b - 1]) < 1e-6


def test_no_partials_weighted_single_transform(golden_dir):
    _, frames = load_case(golden_dir, "gas_unit_self")
    for weight in ("neutron", "xray"):
        scheme = WeightScheme.from_options(weight, "1:Si,2:O")
        S, _, _ = gpu_run(frames, scheme, norm="mean", qmax=6.0, nq=40, eps=1e-10,
                          partials=False)
        _, acc = oracle_run(frames, scheme, 0.0, 6.0, 40, "mean")
        assert rel_dev(acc.shell_value(), S) < 1e-6


def test_multi_frame_call_and_device_positions(golden_dir):
    import torch
    _, frames = load_case(golden_dir, "gas_unit_self")
    f0 = frames[0]
    stack = np.stack([f.pos for f in frames])
    kw = dict(cell=f0.cell.flat(), origin=f0.cell.origin, type_id=f0.type_id, qmax=6.0, nq=40,
              eps=1e-10)
    with _lib.Plan(**kw) as a, _lib.Plan(**kw) as b, _lib.Plan(**kw) as c:
        a.accumulate(stack)
        for f in frames:
            b.accumulate(f.pos)
        dev = torch.from_numpy(stack).cuda()
        c.accumulate((dev.data_ptr(), len(frames)), where=_lib.DEVICE)
        c.sync()
        sa, sb, sc = a.finalize()[0], b.finalize()[0], c.finalize()[0]
    assert rel_dev(sa, sb) < 1e-13 and rel_dev(sa, sc) < 1e-13


def test_errors_surface_as_status_codes():
    cell = Cell.cubic(10.0)
    f = F(np.zeros((4, 3)), np.ones(4), cell)
    with pytest.raises(SqcalcError, match="no reciprocal lattice points"):
        GpuStructureFactor(qmin=0.01, qmax=0.02, nq=4).configure(f, WeightScheme())
    with pytest.raises(SqcalcError, match="limit"):
        GpuStructureFactor(qmax=400.0, nq=4).configure(f, WeightScheme())


def test_stage_timing_and_reset(golden_dir):
    _, frames = load_case(golden_dir, "gas_unit_self")
    m = GpuStructureFactor(qmax=6.0, nq=40, eps=1e-10, timing=True)
    m.configure(frames[0], WeightScheme())
    for f in frames:
        m.accumulate_frame(f)
    t = m.plan.stage_times()
    assert t["frames"] == len(frames) and t["spread_ms"] > 0 and t["bin_ms"] > 0
    m.plan.reset()
    assert m.plan.accumulators()["nframes"] == 0
    assert float(np.max(np.abs(m.plan.accumulators()["num"]))) == 0.0
    m.close()


@pytest.mark.parametrize("precision,tol", [("double", 1e-9), ("single", 1e-5)])
def test_edge_shapes_against_oracle(precision, tol):
    """Small and degenerate inputs the reference accepts: one atom (S = 1 on
    every populated shell, exactly |rho|^2 / N = 1), two atoms of two types, a
    5-mode grid (two shells of lattice points), a single shell, a thin q window
    with empty shells, a triclinic cell with an offset origin -- each against
    the FP64 direct sum (partials included)."""
    rng = np.random.default_rng(21)
    unit = WeightScheme.from_options("unit")
    neutron = WeightScheme.from_options("neutron", "1:Si,2:O")
    tri = Cell(a=np.array([[9.0, 0.0, 0.0], [2.5, 7.0, 0.0], [-1.5, 3.0, 11.0]]),
               origin=np.array([-2.0, 1.0, 0.5]))
    cases = [
        # (frames, scheme, kw)
        ([F(rng.random((1, 3)) * 10, [1], Cell.cubic(10.0))], unit,
         dict(norm="mean", qmax=5.0, nq=40)),
        ([F(rng.random((2, 3)) * 12, [1, 2], Cell.cubic(12.0)) for _ in range(3)], neutron,
         dict(norm="mean", qmax=4.0, nq=25)),
        ([F(rng.random((50, 3)) * 30, rng.integers(1, 3, 50), Cell.cubic(30.0))], unit,
         dict(norm="n", qmax=0.3, nq=3)),   # 5 modes per axis
        ([F(rng.random((300, 3)) * 15, rng.integers(1, 3, 300), Cell.cubic(15.0))
          for _ in range(2)], neutron, dict(norm="self", qmin=0.0, qmax=3.0, nq=1)),
        ([F(rng.random((300, 3)) * 15, rng.integers(1, 3, 300), Cell.cubic(15.0))], unit,
         dict(norm="mean", qmin=2.40, qmax=2.47, nq=5)),
        ([F(rng.random((200, 3)) @ tri.a + tri.origin, rng.integers(1, 3, 200), tri)
          for _ in range(2)], neutron, dict(norm="mean", qmax=4.5, nq=30)),
    ]
    for frames, scheme, kw in cases:
        kw = dict(kw)
        qmin = kw.pop("qmin", 0.0)
        S, Sp, _ = gpu_run(frames, scheme, precision=precision,
                           eps=1e-10 if precision == "double" else 1e-6, qmin=qmin, **kw)
        _, acc = oracle_run(frames, scheme, qmin, kw["qmax"], kw["nq"], kw["norm"])
        ref = acc.shell_value()
        assert rel_dev(ref, S) < tol, (kw, rel_dev(ref, S))
        T = Sp.shape[0]
        for a in range(1, T + 1):
            for b in range(a, T + 1):
                assert rel_dev(acc.partial_value(a, b), Sp[a - 1, b - 1]) < tol
        if len(frames[0].type_id) == 1:
            pop = acc.shell_count > 0
            assert np.all(np.abs(S[pop] - 1.0) < tol)
