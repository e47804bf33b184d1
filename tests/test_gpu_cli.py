"""`python -m sqcalc_b200 static` end to end (the drop-in form of `sqcalc
static`): the dump goes through the library's reader and ingest driver, the
tables it writes match the reference's own result tables for the golden dumps
(test/ref_sq.py output, rtol 1e-6 as in test/test_sqcalc.py), and the
reference's exit codes come back for broken input."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def cli(args):
    return subprocess.run([sys.executable, "-m", "sqcalc_b200", "static", *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=300)


def cases():
    return json.load(open(os.path.join(GOLDEN, "cases.json")))["cases"]


@pytest.mark.parametrize("c", cases(), ids=lambda c: c["case"])
def test_cli_tables_match_reference(tmp_path, c):
    out = str(tmp_path / "sq.dat")
    args = ["-i", os.path.join(GOLDEN, c["dump"]), "-w", c["weight"], "--norm", c["norm"],
            "--qmin", str(c["qmin"]), "--qmax", str(c["qmax"]), "--nq", str(c["nq"]),
            "--eps", "1e-10", "-q", out]
    if c.get("mapping"):
        args[2:2] = ["-m", c["mapping"]]
    r = cli(args)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(out)
    ref = np.loadtxt(os.path.join(GOLDEN, c["table"]))
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=0, atol=1e-6)
    dev = np.max(np.abs(got[:, 1] - ref[:, 1]) / np.maximum(np.abs(ref[:, 1]), 1.0))
    assert dev < 1e-6, dev


FRAME = ("ITEM: TIMESTEP\n{ts}\nITEM: NUMBER OF ATOMS\n{n}\nITEM: BOX BOUNDS pp pp pp\n"
         "0 {L}\n0 {L}\n0 {L}\nITEM: ATOMS id type x y z\n{rows}")


def frame(ts, n, L, seed):
    rng = np.random.default_rng(seed)
    rows = "".join("%d %d %.10f %.10f %.10f\n" % (i + 1, 1 + i % 2, *(rng.random(3) * L))
                   for i in range(n))
    return FRAME.format(ts=ts, n=n, L=L, rows=rows)


@pytest.mark.parametrize("text,code", [
    (None, 4),                                                       # no such file
    ("garbage\n", 5),                                                # no complete frame
    (frame(0, 40, 8.0, 1) + frame(1, 40, 9.0, 2), 9),                # box changes
    (frame(0, 40, 8.0, 1) + frame(1, 41, 8.0, 2), 8),                # atom count changes
    (frame(0, 40, 8.0, 1) + frame(1, 40, 8.0, 2).replace("ATOMS id type x y z",
                                                         "ATOMS id type x y"), 7),
])
def test_cli_exit_codes(tmp_path, text, code):
    path = str(tmp_path / "in.dump")
    if text is not None:
        open(path, "w").write(text)
    r = cli(["-i", path, "-m", "1:Si,2:O", "--qmax", "3", "--nq", "20", "-q",
             str(tmp_path / "o.dat")])
    assert r.returncode == code, (r.returncode, r.stderr)


def test_cli_multi_frame_matches_library(tmp_path):
    from sqcalc_b200 import _lib
    from sqcalc_b200.dump import read_frames
    path = str(tmp_path / "m.dump")
    open(path, "w").write("".join(frame(t, 300, 10.0, 10 + t) for t in range(5)))
    out = str(tmp_path / "o.dat")
    r = cli(["-i", path, "-m", "1:Si,2:O", "--qmax", "5", "--nq", "50", "--eps", "1e-10",
             "--no-partials", "-q", out])
    assert r.returncode == 0, r.stderr
    frames = list(read_frames(path))
    f0 = frames[0]
    with _lib.Plan(f0.cell.flat(), f0.cell.origin, f0.type_id, qmax=5.0, nq=50, eps=1e-10,
                   partials=False) as p:
        p.accumulate(np.stack([f.pos for f in frames]))
        S = p.finalize()[0]
    got = np.loadtxt(out)
    np.testing.assert_allclose(got[:, 1], S, rtol=1e-9, atol=1e-12)


def test_cli_hdf5_grid_and_xrd_match_text_tables(tmp_path):
    """--grid x.h5 / --xrd y.h5 (src/sqc_hdf5.f90:46-210, :1050-1200): the HDF5
    datasets hold the same numbers as the text tables of the same run."""
    import h5read
    path = str(tmp_path / "m.dump")
    open(path, "w").write("".join(frame(t, 300, 10.0, 20 + t) for t in range(3)))
    base = ["-i", path, "-m", "1:Si,2:O", "-w", "neutron", "--eps", "1e-10",
            "--xrd-lambda", "1.5406", "--xrd-range", "10", "120", "-q"]
    txt = ["--grid", str(tmp_path / "g.txt"), "--xrd", str(tmp_path / "x.txt"),
           str(tmp_path / "s.txt")]
    h5 = ["--grid", str(tmp_path / "g.h5"), "--xrd", str(tmp_path / "x.h5"),
          str(tmp_path / "s2.txt")]
    for extra in (txt, h5):
        r = cli(base + extra)
        assert r.returncode == 0, r.stderr
    shell = np.loadtxt(str(tmp_path / "s.txt"))
    grid = np.loadtxt(str(tmp_path / "g.txt"))
    xrd = np.loadtxt(str(tmp_path / "x.txt"))
    f = h5read.read(str(tmp_path / "g.h5"))
    assert f.attrs["nframes"] == 3 and f.attrs["natoms"] == 300
    assert f.attrs["nmodes"] == grid.shape[0] == f["shell/count"].value.sum()
    assert f.attrs["mapping"] == "1:Si,2:O" and f.attrs["device"] == "gpu"
    assert f.attrs["weight"] == "neutron bound coherent scattering lengths"
    assert f.attrs["norm"] == "mean" and f.attrs["precision"] == "double"
    assert f.attrs["cell"].shape == (3, 3) and f.attrs["cell"][0, 0] == 10.0
    np.testing.assert_allclose(f["shell/q"].value, shell[:, 0], atol=1e-6)
    np.testing.assert_allclose(f["shell/S"].value, shell[:, 1], rtol=1e-11, atol=1e-300)
    assert f["shell/pairs"].value == ["Si-Si", "Si-O", "O-O"]
    assert f["shell"].attrs["partial_normalization"] == "ovito"
    for j, lab in enumerate(["Si-Si", "Si-O", "O-O"]):
        np.testing.assert_allclose(f["shell/S_partial/" + lab].value, shell[:, 2 + j],
                                   rtol=1e-11, atol=1e-300)
    for j, name in enumerate(["qx", "qy", "qz"]):
        np.testing.assert_allclose(f["grid/" + name].value, grid[:, j], atol=1e-8)
    np.testing.assert_allclose(f["grid/S"].value, grid[:, 3], rtol=1e-11, atol=1e-300)
    b = 2.0 * np.pi / 10.0
    np.testing.assert_allclose(f["grid/h"].value * b, grid[:, 0], atol=1e-8)
    np.testing.assert_allclose(f["grid/l"].value * b, grid[:, 2], atol=1e-8)
    x = h5read.read(str(tmp_path / "x.h5"))
    assert x.attrs["lambda"] == 1.5406 and x.attrs["bins"] == xrd.shape[0]
    assert x.attrs["lorentz_polarization"] == "on"
    np.testing.assert_allclose(x["xrd/two_theta"].value, xrd[:, 0], atol=1e-4)
    np.testing.assert_allclose(x["xrd/I"].value, xrd[:, 1], rtol=1e-11, atol=1e-300)
    assert x["xrd/count"].value.sum() > 0
    for j, lab in enumerate(["Si-Si", "Si-O", "O-O"]):
        np.testing.assert_allclose(x["xrd/I_partial/" + lab].value, xrd[:, 2 + j],
                                   rtol=1e-11, atol=1e-300)
    # --format text keeps a .h5 name a text table; an unknown format is exit 2
    r = cli(base[:-1] + ["--format", "text", "--grid", str(tmp_path / "t.h5"),
                         "--xrd", str(tmp_path / "x3.h5"), "-q", str(tmp_path / "s3.txt")])
    assert r.returncode == 0, r.stderr
    assert open(str(tmp_path / "t.h5")).readline().startswith("# qx qy qz")
    assert open(str(tmp_path / "x3.h5")).readline().startswith("# xrd: lambda")
    r = cli(base + ["--format", "csv", str(tmp_path / "s4.txt")])
    assert r.returncode == 2
