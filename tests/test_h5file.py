"""The HDF5 writer (sqcalc_b200.h5file) against the published file format.

No HDF5 library or h5py is available here, so the files are parsed back by
tests/h5read.py, a strict reader of the same format subset, and the encodings
the library itself writes for the types sqcalc uses are checked byte for byte.
"""
import struct

import numpy as np
import pytest

from sqcalc_b200 import h5file
import h5read


def test_datatype_encodings_match_the_library_layout():
    # H5T_IEEE_F64LE, H5T_STD_I64LE and H5T_STD_I32LE as stored in a datatype
    # message: class/version byte, three bit-field bytes, size, properties.
    assert h5file._dt_f64() == bytes.fromhex("1120 3f00 0800 0000 0000 4000 340b 0034 ff03 0000")
    assert h5file._dt_int(8) == bytes.fromhex("1008 0000 0800 0000 0000 4000")
    assert h5file._dt_int(4) == bytes.fromhex("1008 0000 0400 0000 0000 2000")
    # fixed-length ASCII string of 18 bytes, space padded (Fortran character)
    assert h5file._dt_str(18, True) == bytes.fromhex("1302 0000 1200 0000")


def test_superblock_fields(tmp_path):
    path = str(tmp_path / "e.h5")
    h5file.write_file(path, h5file.Group())
    b = open(path, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    assert struct.unpack_from("<HHI", b, 16) == (4, 16, 0)
    assert struct.unpack_from("<Q", b, 40)[0] == len(b)
    root = h5read.read(path)
    assert root.kind == "group" and root.children == {} and root.attrs == {}


def _tree():
    root = h5file.Group()
    root.attr("nframes", 7)
    root.attr("qmax", 6.25)
    root.attr("cell", np.arange(9, dtype=np.float64).reshape(3, 3))
    root.attr("weight", "neutron bound coherent scattering lengths")
    root.attr("mapping", "")
    g = root.group("shell")
    g.dataset("q", np.linspace(0.1, 6.0, 50))
    g.dataset("count", np.arange(50, dtype=np.int64) * 3)
    g.attr("partial_normalization", "ovito")
    sp = g.group("S_partial")
    labels = []
    for i in range(13):          # more than one symbol node of 2K = 8 entries
        lab = "%d-%d" % (i + 1, i + 2)
        labels.append(lab)
        sp.dataset(lab, np.full(50, float(i)))
    g.dataset("pairs", labels, strlen=18)
    grid = root.group("grid")
    grid.dataset("h", np.array([-3, 0, 5], dtype=np.int32))
    grid.dataset("S", np.array([1.5, -2.0, 1e300]))
    grid.dataset("empty", np.zeros(0))
    return root, labels


def test_round_trip(tmp_path):
    path = str(tmp_path / "t.h5")
    root, labels = _tree()
    h5file.write_file(path, root)
    r = h5read.read(path)
    assert r.attrs["nframes"] == 7 and r.attrs["nframes"].dtype == np.int64
    assert r.attrs["qmax"] == 6.25
    np.testing.assert_array_equal(r.attrs["cell"], np.arange(9.0).reshape(3, 3))
    assert r.attrs["weight"] == "neutron bound coherent scattering lengths"
    assert r.attrs["mapping"] == ""          # stored as one blank, as the reference does
    np.testing.assert_array_equal(r["shell/q"].value, np.linspace(0.1, 6.0, 50))
    assert r["shell/count"].value.dtype == np.int64
    np.testing.assert_array_equal(r["shell/count"].value, np.arange(50) * 3)
    assert r["shell"].attrs["partial_normalization"] == "ovito"
    assert sorted(r["shell/S_partial"].children) == sorted(labels)
    for i, lab in enumerate(labels):
        np.testing.assert_array_equal(r["shell/S_partial"].children[lab].value, np.full(50, i))
    assert r["shell/pairs"].value == labels
    assert r["shell/pairs"].dtype_info == ("string", 18, 2)
    assert r["grid/h"].value.dtype == np.int32
    np.testing.assert_array_equal(r["grid/h"].value, [-3, 0, 5])
    np.testing.assert_array_equal(r["grid/S"].value, [1.5, -2.0, 1e300])
    assert r["grid/empty"].value.shape == (0,)


def test_large_group_and_limits(tmp_path):
    root = h5file.Group()
    g = root.group("many")
    for i in range(256):         # 32 symbol nodes: a full B-tree leaf
        g.dataset("d%03d" % i, np.array([i], dtype=np.int64))
    path = str(tmp_path / "m.h5")
    h5file.write_file(path, root)
    r = h5read.read(path)
    assert len(r["many"].children) == 256
    assert all(int(r["many"].children["d%03d" % i].value[0]) == i for i in range(256))
    g.dataset("one_more", np.zeros(1))
    with pytest.raises(h5file.H5Error):
        h5file.write_file(str(tmp_path / "n.h5"), root)


@pytest.mark.parametrize("bad", ["", "a/b", ".", "..", "café"])
def test_invalid_names(bad):
    with pytest.raises(h5file.H5Error):
        h5file.Group().dataset(bad, np.zeros(1))


def test_wants_hdf5():
    assert h5file.wants_hdf5("x.h5") and h5file.wants_hdf5("x.hdf5")
    assert not h5file.wants_hdf5("x.h5.txt") and not h5file.wants_hdf5("x.dat")
    assert h5file.wants_hdf5("x.dat", "hdf5") and not h5file.wants_hdf5("x.h5", "text")
    with pytest.raises(h5file.H5Error):
        h5file.wants_hdf5("x", "csv")


def test_reader_rejects_a_damaged_file(tmp_path):
    """The reader is strict: a wrong end-of-file address or a damaged node
    signature is reported, so a passing round trip means the fields agree."""
    path = str(tmp_path / "t.h5")
    h5file.write_file(path, _tree()[0])
    b = bytearray(open(path, "rb").read())
    open(path, "wb").write(bytes(b[:-8]))
    with pytest.raises(h5read.H5FormatError):
        h5read.read(path)
    i = b.find(b"SNOD")
    b[i:i + 4] = b"SNOE"
    open(path, "wb").write(bytes(b))
    with pytest.raises(h5read.H5FormatError):
        h5read.read(path)
