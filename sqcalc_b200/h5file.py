"""HDF5 result files without the HDF5 library.

sqcalc writes its ``--grid x.h5`` and ``--xrd x.h5`` results through libhdf5
(src/sqc_hdf5.f90: hdf5_write_results :46-210, hdf5_write_xrd :1050-1141,
layout :16-23).  The objects involved are few and simple: nested groups, one
dimensional contiguous datasets of float64 / int64 / int32 / fixed-length
strings, and scalar or small array attributes.  This module writes exactly
that subset of the published HDF5 file format, in its oldest layout, which
every HDF5 reader (h5py, h5dump, MATLAB, Julia) accepts:

- superblock version 0 (8-byte offsets and lengths, group K = 4 / 16);
- version 1 object headers;
- groups as symbol tables: a version 1 B-tree leaf of group nodes, symbol
  table nodes (``SNOD``) of up to 2K = 8 entries sorted by name, and a local
  heap (``HEAP``) holding the names;
- datasets with a version 1 dataspace, a version 1 datatype, a version 2 fill
  value (undefined) and a version 3 contiguous layout message;
- version 1 attribute messages in the owning object's header.

Objects are written children first, so every address a parent records is
already known; the superblock is written last at offset 0.  Raw data is
streamed with ``ndarray.tofile`` (a 423^3-mode grid is about 1.6 GB).
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
LEAF_K = 4        # symbol table node holds up to 2 * LEAF_K entries
INTERNAL_K = 16   # B-tree node holds up to 2 * INTERNAL_K children
HEAP_FREE_NULL = 1  # "no free block" in a local heap's free-list head

MSG_DATASPACE = 0x0001
MSG_DATATYPE = 0x0003
MSG_FILL = 0x0005
MSG_LAYOUT = 0x0008
MSG_ATTRIBUTE = 0x000C
MSG_STAB = 0x0011


class H5Error(Exception):
    """A result file that cannot be written (the reference's ``ierr = 1``)."""


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


# --- datatypes -------------------------------------------------------------
def _dt_int(size: int) -> bytes:
    # class 0 (fixed point), version 1; little endian, signed (bit 3)
    return struct.pack("<BBBBIHH", 0x10, 0x08, 0, 0, size, 0, 8 * size)


def _dt_f64() -> bytes:
    # class 1 (floating point), version 1; little endian, implied msb
    # mantissa normalisation (bits 4-5 = 2), sign at bit 63; IEEE binary64
    return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52, 1023)


def _dt_str(size: int, spacepad: bool) -> bytes:
    # class 3 (string), version 1; padding 2 = space pad, 1 = null pad; ASCII
    return struct.pack("<BBBBI", 0x13, 2 if spacepad else 1, 0, 0, size)


def _dataspace(shape) -> bytes:
    # version 1; rank 0 is a scalar dataspace
    out = struct.pack("<BBBBI", 1, len(shape), 0, 0, 0)
    return out + b"".join(struct.pack("<Q", int(d)) for d in shape)


class _Value:
    """A typed array with its HDF5 datatype encoding and raw bytes."""

    def __init__(self, value, strlen=None):
        if isinstance(value, str):
            raw = value.encode("ascii") or b" "
            self.dtype = _dt_str(len(raw), spacepad=True)
            self.shape = ()
            self.array = np.frombuffer(raw, dtype=np.uint8)
            return
        if isinstance(value, (list, tuple)) and value and isinstance(value[0], str):
            n = strlen or max(1, max(len(v) for v in value))
            raw = b"".join(v.encode("ascii")[:n].ljust(n, b" ") for v in value)
            self.dtype = _dt_str(n, spacepad=True)
            self.shape = (len(value),)
            self.array = np.frombuffer(raw, dtype=np.uint8)
            return
        arr = np.asarray(value)
        if arr.dtype.kind == "f":
            arr = np.ascontiguousarray(arr, dtype="<f8")
            self.dtype = _dt_f64()
        elif arr.dtype.kind in "iub":
            if arr.dtype.itemsize <= 4 and arr.dtype.kind != "b" and arr.dtype.kind != "u":
                arr = np.ascontiguousarray(arr, dtype="<i4")
                self.dtype = _dt_int(4)
            else:
                arr = np.ascontiguousarray(arr, dtype="<i8")
                self.dtype = _dt_int(8)
        else:
            raise H5Error("unsupported HDF5 value of dtype %s" % arr.dtype)
        self.shape = arr.shape
        self.array = arr

    @property
    def nbytes(self):
        return self.array.nbytes


class Dataset:
    def __init__(self, value, strlen=None):
        self.value = _Value(value, strlen)
        if self.value.shape == ():
            raise H5Error("datasets are one dimensional or more")


class Group:
    def __init__(self):
        self.children = {}   # name -> Group | Dataset
        self.attrs = {}      # name -> _Value

    def group(self, name: str) -> "Group":
        _check_name(name)
        g = self.children.get(name)
        if g is None:
            g = self.children[name] = Group()
        if not isinstance(g, Group):
            raise H5Error("%s is a dataset, not a group" % name)
        return g

    def dataset(self, name: str, value, strlen=None) -> Dataset:
        _check_name(name)
        if name in self.children:
            raise H5Error("object %s exists" % name)
        d = self.children[name] = Dataset(value, strlen)
        return d

    def attr(self, name: str, value):
        _check_name(name)
        self.attrs[name] = _Value(value)


def _check_name(name: str):
    if not name or "/" in name or name in (".", "..") or not name.isascii() or "\0" in name:
        raise H5Error("invalid HDF5 object name %r" % name)


def _attribute(name: str, v: _Value) -> bytes:
    nm = name.encode("ascii") + b"\0"
    ds = _dataspace(v.shape)
    head = struct.pack("<BBHHH", 1, 0, len(nm), len(v.dtype), len(ds))
    return head + _pad8(nm) + _pad8(v.dtype) + _pad8(ds) + v.array.tobytes()


def _object_header(messages) -> bytes:
    """Version 1 object header: 16-byte prefix, messages padded to 8 bytes."""
    body = b""
    for mtype, data, flags in messages:
        data = _pad8(data)
        if len(data) > 0xFFFF:
            raise H5Error("header message of %d bytes exceeds 64 KiB" % len(data))
        body += struct.pack("<HHB3x", mtype, len(data), flags) + data
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body


class _Out:
    def __init__(self, fh):
        self.fh = fh

    def tell(self):
        return self.fh.tell()

    def put(self, b: bytes) -> int:
        addr = self.fh.tell()
        self.fh.write(b)
        return addr


def _write_dataset(out: _Out, d: Dataset) -> int:
    v = d.value
    data_addr = out.tell() if v.nbytes else UNDEF
    if v.nbytes:
        v.array.tofile(out.fh)
    layout = struct.pack("<BBQQ", 3, 1, data_addr, v.nbytes)
    fill = struct.pack("<BBBB", 2, 2, 2, 0)
    return out.put(_object_header([
        (MSG_DATASPACE, _dataspace(v.shape), 0),
        (MSG_DATATYPE, v.dtype, 1),
        (MSG_FILL, fill, 1),
        (MSG_LAYOUT, layout, 0),
    ]))


def _write_group(out: _Out, g: Group):
    """Write a group's members, then its heap, symbol nodes, B-tree and header.
    Returns (object header address, B-tree address, heap address)."""
    names = sorted(g.children, key=lambda s: s.encode("ascii"))
    if len(names) > 2 * LEAF_K * 2 * INTERNAL_K:
        raise H5Error("a group holds at most %d objects here" % (4 * LEAF_K * INTERNAL_K))
    entries = []
    for name in names:
        child = g.children[name]
        if isinstance(child, Group):
            oh, bt, hp = _write_group(out, child)
            entries.append((name, oh, 1, struct.pack("<QQ", bt, hp)))
        else:
            entries.append((name, _write_dataset(out, child), 0, b"\0" * 16))

    # local heap: offset 0 is the empty name, then every member name
    heap_data = b"\0" * 8
    offsets = {}
    for name in names:
        offsets[name] = len(heap_data)
        heap_data += _pad8(name.encode("ascii") + b"\0")
    heap_addr = out.tell()
    out.put(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), HEAP_FREE_NULL, heap_addr + 32))
    out.put(heap_data)

    # symbol table nodes of up to 2K entries, in name order
    snods, keys = [], [0]
    step = 2 * LEAF_K
    for i in range(0, len(entries), step):
        chunk = entries[i:i + step]
        node = b"SNOD" + struct.pack("<BBH", 1, 0, len(chunk))
        for name, oh, cache, scratch in chunk:
            node += struct.pack("<QQII", offsets[name], oh, cache, 0) + scratch
        node += b"\0" * (40 * (step - len(chunk)))
        snods.append(out.put(node))
        keys.append(offsets[chunk[-1][0]])

    # one B-tree leaf over the symbol nodes, allocated at its full 2K size
    bt = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(snods), UNDEF, UNDEF)
    for i, addr in enumerate(snods):
        bt += struct.pack("<QQ", keys[i], addr)
    bt += struct.pack("<Q", keys[len(snods)])
    full = 24 + 2 * INTERNAL_K * 8 + (2 * INTERNAL_K + 1) * 8
    bt += b"\0" * (full - len(bt))
    bt_addr = out.put(bt)

    msgs = [(MSG_STAB, struct.pack("<QQ", bt_addr, heap_addr), 0)]
    for name, v in g.attrs.items():
        msgs.append((MSG_ATTRIBUTE, _attribute(name, v), 0))
    oh = out.put(_object_header(msgs))
    return oh, bt_addr, heap_addr


def write_file(path: str, root: Group):
    """Write ROOT (its attributes become the file's attributes) to PATH."""
    try:
        fh = open(path, "wb")
    except OSError as e:
        raise H5Error('cannot create HDF5 file "%s"' % path) from e
    with fh:
        out = _Out(fh)
        out.put(b"\0" * 96)
        oh, bt, hp = _write_group(out, root)
        eof = out.tell()
        sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0,
                                     LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQII", 0, oh, 1, 0) + struct.pack("<QQ", bt, hp)
        assert len(sb) == 96
        fh.seek(0)
        fh.write(sb)


def wants_hdf5(path: str, fmt: str | None = None) -> bool:
    """output_wants_hdf5 (src/sqc_output.f90:30-41) with the suffix rule of
    src/sqc_options.f90:816-818: an explicit --format wins, else a name ending
    in .h5 or .hdf5 selects HDF5."""
    if fmt is not None:
        if fmt not in ("text", "hdf5"):
            raise H5Error('unknown format "%s" (use text or hdf5)' % fmt)
        return fmt == "hdf5"
    return path.endswith(".h5") or path.endswith(".hdf5")
