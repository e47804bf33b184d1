"""``python -m sqcalc_b200 static ...``: the static NUFFT path of sqcalc's CLI.

Mirrors the option surface and exit codes of ``sqcalc static --device gpu``
(app/main.f90:41-259, src/sqc_options.f90:330-600) for the hot path only:
-i -m -w --norm --partials/--no-partials -fz --grid --precision --eps --qmin
--qmax --nq --device --gpu-id --xrd --format, output file (``-`` for stdout).
A --grid or --xrd file named ``.h5``/``.hdf5`` (or any name under
``--format hdf5``) is written as HDF5 (src/sqc_hdf5.f90) by ``h5file``.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time


from . import _lib, h5file
from .cell import Cell
from .dump import Frame
from .static import GpuStructureFactor, SqcalcError
from .weights import MappingError, WeightScheme


def _die(code, msg):
    sys.stderr.write("sqcalc: %s\n" % msg)
    sys.exit(code)


def parse(argv):
    p = argparse.ArgumentParser(prog="sqcalc_b200 static", add_help=True)
    p.add_argument("-i", "--input", required=True)
    p.add_argument("-m", "--mapping", default=None)
    p.add_argument("-w", "--weight", default=None)
    p.add_argument("--norm", default="mean", choices=["mean", "fz", "self", "n", "natom"])
    g = p.add_mutually_exclusive_group()
    g.add_argument("--partials", dest="partials", action="store_true", default=True)
    g.add_argument("--no-partials", dest="partials", action="store_false")
    p.add_argument("-fz", "--faber-ziman", action="store_true")
    p.add_argument("--grid", default=None)
    p.add_argument("--precision", default="double")
    p.add_argument("--eps", type=float, default=None)
    p.add_argument("--qmin", type=float, default=None)
    p.add_argument("--qmax", type=float, default=None)
    p.add_argument("--xrd", default=None, metavar="FILE")
    p.add_argument("--xrd-lambda", type=float, default=None)
    p.add_argument("--xrd-range", type=float, nargs=2, default=None, metavar=("MIN2TH", "MAX2TH"))
    p.add_argument("--xrd-step", type=float, default=None)
    lp = p.add_mutually_exclusive_group()
    lp.add_argument("--lp", dest="lp", action="store_true", default=None)
    lp.add_argument("--no-lp", dest="lp", action="store_false")
    p.add_argument("--nq", type=int, default=500)
    p.add_argument("--format", default=None)
    p.add_argument("--device", default="gpu", choices=["gpu", "cuda"])
    p.add_argument("--gpu-id", type=int, default=0)
    p.add_argument("--method", default="nufft", choices=["nufft", "finufft"])
    p.add_argument("-t", "--threads", type=int, default=0)
    p.add_argument("-q", "--quiet", action="store_true")
    p.add_argument("output", nargs="?", default=None)
    return p.parse_args(argv)


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] != "static":
        _die(2, "usage: python -m sqcalc_b200 static -i DUMP [options] OUTPUT")
    try:
        a = parse(argv[1:])
    except SystemExit as e:
        sys.exit(2 if e.code else 0)
    # --format (src/sqc_options.f90:556-567)
    if a.format is not None:
        fmt = {"text": "text", "txt": "text", "ascii": "text",
               "hdf5": "hdf5", "h5": "hdf5", "hdf": "hdf5"}.get(a.format)
        if fmt is None:
            _die(2, 'unknown format "%s" (use text or hdf5)' % a.format)
        a.format = fmt
    # --xrd and its settings (src/sqc_options.f90:620-658)
    xrd = None
    if a.xrd is not None:
        if a.xrd_lambda is None:
            _die(2, "--xrd needs --xrd-lambda LAMBDA (the incident wavelength)")
        if not a.xrd_lambda > 0.0:
            _die(2, "--xrd-lambda must be a positive wavelength")
        if a.qmin is not None or a.qmax is not None:
            _die(2, "--xrd takes the q range from --xrd-lambda and --xrd-range; "
                    "do not pass --qmin or --qmax with it")
        lo, hi = a.xrd_range if a.xrd_range else (1.0, 179.0)
        if not (lo > 0.0 and hi < 180.0 and hi > lo):
            _die(2, "--xrd-range needs 0 < MIN2TH < MAX2TH < 180 degrees")
        if a.xrd_step is not None and not a.xrd_step > 0.0:
            _die(2, "--xrd-step must be a positive number of degrees")
        xrd = dict(lam=a.xrd_lambda, range=(lo, hi), step=a.xrd_step or 0.0,
                   lp=True if a.lp is None else a.lp)
        if a.weight is None:
            a.weight = "xray"
        a.qmin = 4.0 * math.pi * math.sin(0.5 * math.radians(lo)) / a.xrd_lambda
        a.qmax = 4.0 * math.pi * math.sin(0.5 * math.radians(hi)) / a.xrd_lambda
    elif (a.xrd_lambda is not None or a.xrd_range is not None or a.xrd_step is not None
          or a.lp is not None):
        _die(2, "--xrd-lambda, --xrd-range, --xrd-step and --lp/--no-lp belong to --xrd FILE")
    a.weight = a.weight or "unit"
    a.qmin = 0.0 if a.qmin is None else a.qmin
    a.qmax = 20.0 if a.qmax is None else a.qmax
    try:
        scheme = WeightScheme.from_options(a.weight, a.mapping)
    except MappingError as e:
        _die(2, str(e))
    # The library's multithreaded reader: the first frame configures the
    # method, the rest stream through sqn_accumulate_dump (the parse of one
    # frame overlaps the upload and transform of the previous one).
    if not os.path.exists(a.input):
        _die(4, 'cannot open dump file "%s"' % a.input)
    try:
        reader = _lib.DumpReader(a.input, nthreads=a.threads)
        head = reader.next()
    except _lib.SqnError as e:
        _die(5, 'no complete frame found in "%s" (%s)' % (a.input, e))
    if head is None:
        _die(5, 'no complete frame found in "%s"' % a.input)
    ts, natoms, bounds, pos, types, ids = head
    first = Frame(natoms, ts, pos, types, ids,
                  Cell.from_bounds(bounds[:, 0], bounds[:, 1], bounds[:, 2]))
    method = GpuStructureFactor(norm=a.norm, nq=a.nq, qmin=a.qmin, qmax=a.qmax, eps=a.eps,
                                want_grid=a.grid is not None, partials=a.partials,
                                faber_ziman=a.faber_ziman, precision=a.precision,
                                device=a.gpu_id, xrd=xrd)
    try:
        method.configure(first, scheme)
    except SqcalcError as e:
        _die(6, str(e))
    t0 = time.time()
    method.accumulate_frame(first)
    n = 1
    try:
        n += method.plan.accumulate_dump(reader, ref_bounds=bounds.reshape(-1))
    except _lib.SqnError as e:
        if e.code == _lib.ERR_NUM_NU_PTS_INVALID:
            _die(8, "number of atoms changes between frames")
        code = reader.last_error()
        if code == 10:
            _die(9, "the simulation box changes between frames")
        _die(7, "malformed dump (reader error %d): %s" % (code, e))
    reader.close()
    method.plan.sync()
    if not a.quiet:
        sys.stderr.write("  frames     : %d in %.3f s\n" % (n, time.time() - t0))
    # app/main.f90:390-488: text tables first, then the HDF5 files.
    grid_h5 = a.grid is not None and h5file.wants_hdf5(a.grid, a.format)
    xrd_h5 = a.xrd is not None and h5file.wants_hdf5(a.xrd, a.format)
    try:
        method.write_results(a.output, None if grid_h5 else a.grid)
        if a.xrd is not None and not xrd_h5:
            method.write_xrd(a.xrd)
    except OSError as e:
        _die(11, str(e))
    if xrd_h5:
        try:
            method.write_xrd_hdf5(a.xrd)
        except h5file.H5Error as e:
            _die(21, str(e))
    if grid_h5:
        try:
            method.write_hdf5(a.grid)
        except h5file.H5Error as e:
            _die(18, str(e))
    method.close()


if __name__ == "__main__":
    main()
