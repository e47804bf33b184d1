"""Strict reader of the HDF5 subset that sqcalc_b200.h5file writes.

Test infrastructure: no HDF5 library or h5py exists in this image, so the
writer is checked by parsing its files back field by field against the
published HDF5 file format (superblock v0, v1 object headers, symbol-table
groups with v1 B-trees, local heaps and symbol nodes, contiguous layouts,
v1 attributes).  Every structural rule the library enforces on read that
this subset touches is asserted: signatures, versions, fixed node sizes,
sorted names, B-tree keys, message sizes and counts, the end-of-file address
and the storage size of each dataset.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class H5FormatError(AssertionError):
    pass


def _req(cond, what):
    if not cond:
        raise H5FormatError(what)


class Node:
    def __init__(self, kind):
        self.kind = kind        # "group" | "dataset"
        self.attrs = {}
        self.children = {}
        self.value = None
        self.dtype_info = None

    def __getitem__(self, path):
        node = self
        for part in path.strip("/").split("/"):
            node = node.children[part]
        return node


class Reader:
    def __init__(self, path):
        with open(path, "rb") as fh:
            self.b = fh.read()
        b = self.b
        _req(b[:8] == b"\x89HDF\r\n\x1a\n", "superblock signature")
        (sbv, fsv, rsv, r0, shv, so, sl, r1, self.leaf_k, self.int_k,
         flags) = struct.unpack_from("<BBBBBBBBHHI", b, 8)
        _req(sbv == 0 and fsv == 0 and rsv == 0 and shv == 0, "superblock version 0")
        _req(so == 8 and sl == 8, "8-byte offsets and lengths")
        _req(self.leaf_k > 0 and self.int_k > 0, "group K values")
        base, fsaddr, eof, drv = struct.unpack_from("<QQQQ", b, 24)
        _req(base == 0, "base address 0")
        _req(fsaddr == UNDEF and drv == UNDEF, "free-space and driver addresses undefined")
        _req(eof == len(b), "end-of-file address %d equals the file size %d" % (eof, len(b)))
        name_off, oh, cache, _ = struct.unpack_from("<QQII", b, 56)
        _req(cache in (0, 1), "root cache type")
        self.root = self._object(oh)
        _req(self.root.kind == "group", "root is a group")
        if cache == 1:
            bt, hp = struct.unpack_from("<QQ", b, 80)
            _req((bt, hp) == self.root._stab, "root symbol table cache matches its header")

    # --- object headers ----------------------------------------------------
    def _messages(self, addr):
        b = self.b
        ver, _, nmsg, refc, size = struct.unpack_from("<BBHII", b, addr)
        _req(ver == 1, "object header version 1")
        _req(refc >= 1, "object reference count")
        _req(size % 8 == 0, "object header chunk size is a multiple of 8")
        p, end = addr + 16, addr + 16 + size
        _req(end <= len(b), "object header inside the file")
        out = []
        while p < end:
            mtype, msize, mflags = struct.unpack_from("<HHB", b, p)
            _req(msize % 8 == 0, "message size is a multiple of 8")
            _req(p + 8 + msize <= end, "message inside its chunk")
            if mtype != 0:
                out.append((mtype, b[p + 8:p + 8 + msize], mflags))
            p += 8 + msize
        _req(p == end, "messages fill the chunk exactly")
        _req(len(out) == nmsg, "message count %d matches %d" % (len(out), nmsg))
        return out

    def _object(self, addr):
        msgs = self._messages(addr)
        types = [m[0] for m in msgs]
        attrs = {}
        for mtype, data, _ in msgs:
            if mtype == 0x000C:
                name, val = self._attribute(data)
                _req(name not in attrs, "unique attribute names")
                attrs[name] = val
        if 0x0011 in types:
            _req(not ({0x0001, 0x0003, 0x0008} & set(types)), "a group has no dataset messages")
            data = msgs[types.index(0x0011)][1]
            bt, hp = struct.unpack_from("<QQ", data, 0)
            node = Node("group")
            node._stab = (bt, hp)
            node.children = self._group(bt, hp)
        else:
            for need in (0x0001, 0x0003, 0x0008):
                _req(need in types, "dataset message %#x present" % need)
            shape = self._dataspace(msgs[types.index(0x0001)][1])
            dt, info = self._datatype(msgs[types.index(0x0003)][1])
            if 0x0005 in types:
                self._fill(msgs[types.index(0x0005)][1])
            lay = msgs[types.index(0x0008)][1]
            ver, cls = lay[0], lay[1]
            _req(ver == 3 and cls == 1, "contiguous layout version 3")
            daddr, dsize = struct.unpack_from("<QQ", lay, 2)
            n = int(np.prod(shape)) if shape else 1
            _req(dsize == n * dt.itemsize, "storage size matches the dataspace")
            if dsize:
                _req(daddr != UNDEF and daddr + dsize <= len(self.b), "data inside the file")
                raw = self.b[daddr:daddr + dsize]
            else:
                raw = b""
            node = Node("dataset")
            node.value = self._decode(raw, dt, info, shape)
            node.dtype_info = info
        for mtype in types:
            _req(mtype in (0x0001, 0x0003, 0x0005, 0x0008, 0x000C, 0x0011),
                 "known message type %#x" % mtype)
        node.attrs = attrs
        return node

    # --- groups ------------------------------------------------------------
    def _heap(self, addr):
        b = self.b
        _req(b[addr:addr + 4] == b"HEAP", "local heap signature")
        _req(b[addr + 4] == 0, "local heap version 0")
        dsize, free, daddr = struct.unpack_from("<QQQ", b, addr + 8)
        _req(dsize % 8 == 0 and dsize >= 8, "heap data size")
        _req(free == 1 or free < dsize, "heap free-list head")
        _req(daddr + dsize <= len(b), "heap data inside the file")
        _req(b[daddr] == 0, "heap offset 0 is the empty name")
        return daddr, dsize

    def _name(self, heap, off):
        daddr, dsize = heap
        _req(off < dsize, "name offset inside the heap")
        end = self.b.index(b"\0", daddr + off)
        _req(end < daddr + dsize, "name terminated inside the heap")
        return self.b[daddr + off:end].decode("ascii")

    def _group(self, bt, hp):
        heap = self._heap(hp)
        entries = []
        self._btree(bt, heap, entries)
        names = [e[0] for e in entries]
        _req(names == sorted(names, key=lambda s: s.encode()), "names in strcmp order")
        _req(len(set(names)) == len(names), "unique names")
        out = {}
        for name, oh, cache, scratch in entries:
            child = self._object(oh)
            if cache == 1:
                _req(child.kind == "group", "cache type 1 only on groups")
                _req(struct.unpack("<QQ", scratch) == child._stab, "cached symbol table")
            out[name] = child
        return out

    def _btree(self, addr, heap, entries):
        b = self.b
        _req(b[addr:addr + 4] == b"TREE", "B-tree signature")
        ntype, level, used = struct.unpack_from("<BBH", b, addr + 4)
        left, right = struct.unpack_from("<QQ", b, addr + 8)
        _req(ntype == 0, "group B-tree node")
        _req(used <= 2 * self.int_k, "B-tree entries within 2K")
        full = 24 + 2 * self.int_k * 8 + (2 * self.int_k + 1) * 8
        _req(addr + full <= len(b), "B-tree node allocated at full size")
        p = addr + 24
        keys, kids = [], []
        for i in range(used):
            keys.append(struct.unpack_from("<Q", b, p)[0])
            kids.append(struct.unpack_from("<Q", b, p + 8)[0])
            p += 16
        keys.append(struct.unpack_from("<Q", b, p)[0])
        knames = [self._name(heap, k) for k in keys]
        for i, kid in enumerate(kids):
            start = len(entries)
            if level == 0:
                self._snod(kid, heap, entries)
            else:
                self._btree(kid, heap, entries)
            got = [e[0] for e in entries[start:]]
            _req(got, "child node not empty")
            _req(all(knames[i].encode() < g.encode() for g in got), "left key below the child")
            _req(got[-1] == knames[i + 1], "right key is the child's last name")

    def _snod(self, addr, heap, entries):
        b = self.b
        _req(b[addr:addr + 4] == b"SNOD", "symbol node signature")
        ver, _, n = struct.unpack_from("<BBH", b, addr + 4)
        _req(ver == 1, "symbol node version 1")
        _req(0 < n <= 2 * self.leaf_k, "symbol node entries within 2K")
        _req(addr + 8 + 2 * self.leaf_k * 40 <= len(b), "symbol node allocated at full size")
        for i in range(n):
            p = addr + 8 + 40 * i
            off, oh, cache, _ = struct.unpack_from("<QQII", b, p)
            entries.append((self._name(heap, off), oh, cache, b[p + 24:p + 40]))

    # --- messages ----------------------------------------------------------
    def _dataspace(self, d):
        ver, rank, flags = d[0], d[1], d[2]
        _req(ver == 1, "dataspace version 1")
        _req(flags & ~1 == 0, "dataspace flags")
        return tuple(struct.unpack_from("<%dQ" % rank, d, 8)) if rank else ()

    def _datatype(self, d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        _req(ver == 1, "datatype version 1")
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = struct.unpack_from("<I", d, 4)[0]
        if cls == 0:
            _req(bits & 1 == 0, "little endian integer")
            off, prec = struct.unpack_from("<HH", d, 8)
            _req(off == 0 and prec == 8 * size, "integer precision")
            signed = bool(bits & 8)
            return np.dtype(("<i" if signed else "<u") + str(size)), ("int", size, signed)
        if cls == 1:
            _req(size == 8, "binary64")
            _req(bits & 1 == 0 and (bits >> 4) & 3 == 2 and (bits >> 8) & 0xFF == 63,
                 "little endian, implied msb, sign bit 63")
            off, prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HHBBBBI", d, 8)
            _req((off, prec, eloc, esz, mloc, msz, bias) == (0, 64, 52, 11, 0, 52, 1023),
                 "IEEE binary64 fields")
            return np.dtype("<f8"), ("float", 8)
        if cls == 3:
            pad, cset = bits & 0xF, (bits >> 4) & 0xF
            _req(pad in (0, 1, 2) and cset == 0, "ASCII string padding")
            _req(size >= 1, "string size")
            return np.dtype("S%d" % size), ("string", size, pad)
        raise H5FormatError("datatype class %d" % cls)

    def _fill(self, d):
        _req(d[0] == 2, "fill value version 2")
        _req(d[1] in (1, 2, 3) and d[2] in (0, 1, 2) and d[3] in (0, 1), "fill value fields")

    def _attribute(self, d):
        ver, _, nlen, tlen, slen = struct.unpack_from("<BBHHH", d, 0)
        _req(ver == 1, "attribute version 1")
        p = 8
        name = d[p:p + nlen]
        _req(name.endswith(b"\0"), "attribute name null-terminated")
        p += (nlen + 7) // 8 * 8
        dt, info = self._datatype(d[p:p + tlen])
        p += (tlen + 7) // 8 * 8
        shape = self._dataspace(d[p:p + slen])
        p += (slen + 7) // 8 * 8
        n = int(np.prod(shape)) if shape else 1
        raw = d[p:p + n * dt.itemsize]
        _req(len(raw) == n * dt.itemsize, "attribute data present")
        return name[:-1].decode("ascii"), self._decode(raw, dt, info, shape)

    @staticmethod
    def _decode(raw, dt, info, shape):
        arr = np.frombuffer(raw, dtype=dt)
        if info[0] == "string":
            pad = info[2]
            vals = [x.decode("ascii") for x in arr]  # numpy strips trailing NULs
            if pad == 2:
                vals = [v.rstrip(" ") for v in vals]
            return vals[0] if shape == () else vals
        arr = arr.reshape(shape) if shape else arr[0]
        return arr


def read(path) -> Node:
    return Reader(path).root
