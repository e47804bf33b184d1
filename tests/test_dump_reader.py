"""The library's multithreaded LAMMPS dump reader (sqn_dump_*, host code: runs
without a GPU) against the Python reader that mirrors lammps_next_frame
(src/sqc_dump.f90:162-313): same frames, same doubles bit for bit, same
column rules, and the reference's error codes for malformed input."""
import os

import numpy as np
import pytest

from sqcalc_b200 import _lib
from sqcalc_b200.dump import read_frames

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def dumps():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".dump") or f.endswith(".lammpstrj"))


def all_frames(path, nthreads=0):
    out = []
    with _lib.DumpReader(path, nthreads=nthreads) as r:
        while True:
            f = r.next()
            if f is None:
                return out
            out.append(f)


@pytest.mark.parametrize("name", dumps())
@pytest.mark.parametrize("nthreads", [1, 3, 0])
def test_reader_matches_python_reader(name, nthreads):
    path = os.path.join(GOLDEN, name)
    ref = list(read_frames(path))
    got = all_frames(path, nthreads)
    assert len(got) == len(ref)
    for (ts, n, bounds, pos, types, ids), f in zip(got, ref):
        assert ts == f.timestep and n == f.natoms
        np.testing.assert_array_equal(pos, f.pos)
        np.testing.assert_array_equal(types, f.type_id)
        np.testing.assert_array_equal(ids, f.id)


def write(tmp_path, text):
    p = tmp_path / "t.dump"
    p.write_text(text)
    return str(p)


HEAD = "ITEM: TIMESTEP\n7\nITEM: NUMBER OF ATOMS\n{n}\nITEM: BOX BOUNDS pp pp pp\n0 10\n0 10\n0 10\n"


def test_large_frame_many_threads_and_columns(tmp_path):
    rng = np.random.default_rng(2)
    n = 50000
    pos = rng.random((n, 3)) * 10
    types = rng.integers(1, 4, n)
    lines = [HEAD.format(n=n) + "ITEM: ATOMS id type vx xu yu zu q\n"]
    lines += ["%d %d 0.5 %.17g %.17g %.17g -1\n" % (i + 1, t, *p) for i, (t, p) in
              enumerate(zip(types, pos))]
    path = write(tmp_path, "".join(lines) * 2)
    got = all_frames(path, nthreads=7)
    assert len(got) == 2
    for f in got:
        np.testing.assert_array_equal(f[3], pos)
        np.testing.assert_array_equal(f[4], types)


@pytest.mark.parametrize("text,code", [
    ("ITEM: TIMESTEP\nx\n", 4),
    (HEAD.format(n=0) + "ITEM: ATOMS id type x y z\n", 5),
    ("ITEM: TIMESTEP\n1\nITEM: NUMBER OF ATOMS\n1\nITEM: BOX BOUNDS pp pp pp\n0 a\n0 1\n0 1\n"
     "ITEM: ATOMS id type x y z\n1 1 0 0 0\n", 6),
    ("ITEM: TIMESTEP\n1\nITEM: ATOMS id type x y z\n1 1 0 0 0\n", 7),
    (HEAD.format(n=2) + "ITEM: ATOMS id type x y z\n1 1 0 0 0\n2 1 0 0\n", 8),
    (HEAD.format(n=1) + "ITEM: ATOMS id type x y\n1 1 0 0\n", 9),
])
def test_reader_error_codes(tmp_path, text, code):
    path = write(tmp_path, text)
    with _lib.DumpReader(path) as r:
        with pytest.raises(_lib.SqnError):
            r.next()
        assert r.last_error() == code


def test_end_of_file_and_rewind(tmp_path):
    path = write(tmp_path, HEAD.format(n=1) + "ITEM: ATOMS id type x y z\n1 2 1.5 2.5 3.5\n")
    with _lib.DumpReader(path) as r:
        f = r.next()
        assert f[1] == 1 and list(f[3][0]) == [1.5, 2.5, 3.5] and f[4][0] == 2
        assert r.next() is None
        r.rewind()
        assert r.next() is not None


def test_coordinate_parsing_is_correctly_rounded(tmp_path):
    """The reader's fast decimal path (Clinger's: an integer significand below
    2^53 and a power of ten up to 22) and its fallback give the correctly rounded
    double of every coordinate, whatever the format: fixed, %.17g, exponents,
    signs, leading zeros, 20-digit significands, huge and tiny values."""
    rng = np.random.default_rng(12)
    n = 3000
    vals = np.concatenate([rng.random(n) * 220.0, -rng.random(n) * 1e-3,
                           rng.standard_normal(n) * 1e6, 10.0 ** rng.uniform(-30, 30, n)])
    fmts = ["%.6f", "%.17g", "%.3e", "%+.9f", "%.20f", "%.15g", "%.1f", "%.12E"]
    texts = [fmts[i % len(fmts)] % v for i, v in enumerate(vals)]
    texts[:6] = ["0", "-0.0", ".5", "5.", "000123.4500", "1e22"]
    m = len(texts) // 3
    lines = ["%d 1 %s %s %s" % (i + 1, texts[3 * i], texts[3 * i + 1], texts[3 * i + 2])
             for i in range(m)]
    path = str(tmp_path / "fmt.dump")
    with open(path, "w") as fh:
        fh.write("ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n%d\nITEM: BOX BOUNDS pp pp pp\n"
                 "0 1\n0 1\n0 1\nITEM: ATOMS id type x y z\n" % m)
        fh.write("\n".join(lines) + "\n")
    want = np.array([float(t) for t in texts[:3 * m]]).reshape(m, 3)
    for nt in (1, 4):
        got = all_frames(path, nt)
        assert len(got) == 1
        pos = got[0][3]
        assert np.array_equal(pos.view(np.uint64), want.view(np.uint64))


def test_threaded_block_split_with_ragged_lines(tmp_path):
    """Frames large enough for several reader threads (the atom block split by
    parallel line counts over a byte region estimated from the first lines):
    short lines first and much longer lines later force the region to be
    widened; extra columns, tabs and a missing final newline are handled like
    the one-thread reader, and every frame equals the Python reader's."""
    rng = np.random.default_rng(4)
    n = 30000
    path = str(tmp_path / "big.dump")
    with open(path, "w") as fh:
        for f in range(3):
            fh.write("ITEM: TIMESTEP\n%d\nITEM: NUMBER OF ATOMS\n%d\nITEM: BOX BOUNDS pp pp pp\n"
                     "0 50\n0 50\n0 50\nITEM: ATOMS id type x y z vx\n" % (f, n))
            rows = []
            for i in range(n):
                x, y, z = rng.random(3) * 50
                if i < 300:
                    rows.append("%d 1 %.2f %.2f %.2f 0" % (i + 1, x, y, z))
                else:
                    rows.append("%d\t%d  %.15f %.15e %+.12f   %.9f" % (i + 1, 1 + i % 3, x, y, z,
                                                                     rng.random()))
            body = "\n".join(rows)
            fh.write(body + ("\n" if f < 2 else ""))
    ref = list(read_frames(path))
    for nt in (1, 4, 7):
        got = all_frames(path, nt)
        assert len(got) == len(ref) == 3
        for (ts, nat, bounds, pos, types, ids), fr in zip(got, ref):
            assert ts == fr.timestep and nat == fr.natoms == n
            assert np.array_equal(pos.view(np.uint64), fr.pos.view(np.uint64))
            np.testing.assert_array_equal(types, fr.type_id)
