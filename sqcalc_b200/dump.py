"""LAMMPS text dump reader for the static S(q) path.

Host-side restatement of the parts of thatstar/sqcalc src/sqc_dump.f90 that the
static path needs (lammps_next_frame, :162-313): the ITEM blocks, the box
bounds with optional tilts, and the id / type / x|xu y|yu z|zu columns.  The
static path wraps every coordinate into the cell, so the unwrapping the
reference does for the dynamic subcommand (:325-391) is not needed here.
Reader error codes follow the reference: 1 end of file, 4-8 malformed input.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .cell import Cell


class DumpError(Exception):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


@dataclass
class Frame:
    natoms: int
    timestep: int
    pos: np.ndarray      # (natoms, 3) Cartesian, float64
    type_id: np.ndarray  # (natoms,) int32, 1-based
    id: np.ndarray       # (natoms,) int64
    cell: Cell
    pbc: tuple = (True, True, True)


def _pbc(line):
    toks = line.split()[3:]
    toks = [t for t in toks if t not in ("xy", "xz", "yz")]
    if len(toks) < 3:
        return (True, True, True)
    return tuple(t.startswith("p") for t in toks[:3])


def read_frames(path, max_frames=None):
    """Yield every frame of a default-style LAMMPS dump."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    i, n = 0, len(lines)
    count = 0
    while i < n:
        timestep = natoms = None
        bounds = None
        pbc = (True, True, True)
        while i < n and not lines[i].startswith("ITEM: ATOMS"):
            line = lines[i]
            if line.startswith("ITEM: TIMESTEP"):
                try:
                    timestep = int(lines[i + 1].split()[0])
                except (IndexError, ValueError):
                    raise DumpError(4, "malformed TIMESTEP near line %d" % (i + 1))
                i += 2
            elif line.startswith("ITEM: NUMBER OF ATOMS"):
                try:
                    natoms = int(lines[i + 1].split()[0])
                except (IndexError, ValueError):
                    raise DumpError(5, "malformed NUMBER OF ATOMS near line %d" % (i + 1))
                if natoms <= 0:
                    raise DumpError(5, "non-positive atom count near line %d" % (i + 1))
                i += 2
            elif line.startswith("ITEM: BOX BOUNDS"):
                pbc = _pbc(line)
                rows = []
                for k in range(3):
                    if i + 1 + k >= n:
                        raise DumpError(4, "truncated BOX BOUNDS")
                    vals = lines[i + 1 + k].split()
                    try:
                        v = [float(x) for x in vals[:3]]
                    except ValueError:
                        raise DumpError(6, "malformed BOX BOUNDS near line %d" % (i + 2 + k))
                    if len(v) < 2:
                        raise DumpError(6, "malformed BOX BOUNDS near line %d" % (i + 2 + k))
                    rows.append(v + [0.0] * (3 - len(v)))
                bounds = rows
                i += 4
            else:
                i += 1
        if i >= n:
            if count == 0 and timestep is None:
                raise DumpError(1, "no frame found")
            return
        if natoms is None or bounds is None:
            raise DumpError(7, "ATOMS block before NUMBER OF ATOMS / BOX BOUNDS")
        cols = lines[i].split()[2:]
        need = {}
        for axis, names in (("x", ("x", "xu")), ("y", ("y", "yu")), ("z", ("z", "zu"))):
            hit = [c for c in names if c in cols]
            if not hit:
                raise DumpError(7, "dump has no %s column" % axis)
            need[axis] = cols.index(hit[0])
        if "type" not in cols:
            raise DumpError(7, "dump has no type column")
        body = lines[i + 1:i + 1 + natoms]
        if len(body) < natoms:
            raise DumpError(8, "truncated ATOMS block")
        try:
            data = np.array([list(map(float, row.split())) for row in body], dtype=np.float64)
        except ValueError:
            raise DumpError(8, "malformed atom line in the frame at timestep %s" % timestep)
        if data.ndim != 2 or data.shape[1] < len(cols):
            raise DumpError(8, "short atom line in the frame at timestep %s" % timestep)
        i += 1 + natoms
        lo = [bounds[k][0] for k in range(3)]
        hi = [bounds[k][1] for k in range(3)]
        tilt = [bounds[0][2], bounds[1][2], bounds[2][2]]
        cell = Cell.from_bounds(lo, hi, tilt)
        pos = np.ascontiguousarray(data[:, [need["x"], need["y"], need["z"]]])
        type_id = np.rint(data[:, cols.index("type")]).astype(np.int32)
        ids = (np.rint(data[:, cols.index("id")]).astype(np.int64) if "id" in cols
               else np.arange(1, natoms + 1, dtype=np.int64))
        yield Frame(natoms, int(timestep or 0), pos, type_id, ids, cell, pbc)
        count += 1
        if max_frames is not None and count >= max_frames:
            return
