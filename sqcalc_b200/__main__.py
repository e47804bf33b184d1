"""``python -m sqcalc_b200 static ...``: the static NUFFT path of sqcalc's CLI.

Mirrors the option surface and exit codes of ``sqcalc static --device gpu``
(app/main.f90:41-259, src/sqc_options.f90:330-600) for the hot path only:
-i -m -w --norm --partials/--no-partials -fz --grid --precision --eps --qmin
--qmax --nq --device --gpu-id, output file (``-`` for stdout).
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np

from .dump import DumpError, read_frames
from .static import GpuStructureFactor, SqcalcError
from .weights import MappingError, WeightScheme


def _die(code, msg):
    sys.stderr.write("sqcalc: %s\n" % msg)
    sys.exit(code)


def parse(argv):
    p = argparse.ArgumentParser(prog="sqcalc_b200 static", add_help=True)
    p.add_argument("-i", "--input", required=True)
    p.add_argument("-m", "--mapping", default=None)
    p.add_argument("-w", "--weight", default="unit")
    p.add_argument("--norm", default="mean", choices=["mean", "fz", "self", "n", "natom"])
    g = p.add_mutually_exclusive_group()
    g.add_argument("--partials", dest="partials", action="store_true", default=True)
    g.add_argument("--no-partials", dest="partials", action="store_false")
    p.add_argument("-fz", "--faber-ziman", action="store_true")
    p.add_argument("--grid", default=None)
    p.add_argument("--precision", default="double")
    p.add_argument("--eps", type=float, default=None)
    p.add_argument("--qmin", type=float, default=0.0)
    p.add_argument("--qmax", type=float, default=20.0)
    p.add_argument("--nq", type=int, default=500)
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
    try:
        scheme = WeightScheme.from_options(a.weight, a.mapping)
    except MappingError as e:
        _die(2, str(e))
    frames = read_frames(a.input)
    try:
        first = next(frames)
    except FileNotFoundError:
        _die(4, 'cannot open dump file "%s"' % a.input)
    except (DumpError, StopIteration) as e:
        _die(5, 'no complete frame found in "%s" (%s)' % (a.input, e))
    method = GpuStructureFactor(norm=a.norm, nq=a.nq, qmin=a.qmin, qmax=a.qmax, eps=a.eps,
                                want_grid=a.grid is not None, partials=a.partials,
                                faber_ziman=a.faber_ziman, precision=a.precision,
                                device=a.gpu_id)
    try:
        method.configure(first, scheme)
    except SqcalcError as e:
        _die(6, str(e))
    ref_a = first.cell.a.copy()
    t0 = time.time()
    frame, n = first, 0
    while True:
        if frame.natoms != first.natoms:
            _die(8, "number of atoms changes between frames")
        if np.max(np.abs(frame.cell.a - ref_a)) > 1e-6 * max(1.0, float(np.max(np.abs(ref_a)))):
            _die(9, "the simulation box changes between frames")
        method.accumulate_frame(frame)
        n += 1
        try:
            frame = next(frames)
        except StopIteration:
            break
        except DumpError as e:
            _die(7, "malformed dump (reader error %d): %s" % (e.code, e))
    method.plan.sync()
    if not a.quiet:
        sys.stderr.write("  frames     : %d in %.3f s\n" % (n, time.time() - t0))
    try:
        method.write_results(a.output, a.grid)
    except OSError as e:
        _die(11, str(e))
    method.close()


if __name__ == "__main__":
    main()
