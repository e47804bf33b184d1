"""Host side of ``sqcalc static --device gpu`` over libsqnufft.so.

Mirrors the reference's GPU method object (cufinufft_structure_factor_t,
src/sqc_gpu.f90:42-71) and the parts of structure_factor_t it relies on
(src/sqc_structure_factor.f90:71-192): ``configure`` from the first frame,
``accumulate_frame`` per frame, ``write_results`` in the reference's table
format (sf_write_results, :771-827).  The per-frame work is one call into the
library; the reciprocal-grid bookkeeping needed for labels and the --grid table
is restated here.
"""
from __future__ import annotations

import math
import sys
from dataclasses import dataclass

import numpy as np

from . import _lib, h5file
from .cell import Cell
from .weights import WEIGHT_NEUTRON, WEIGHT_XRAY, WeightScheme

NORM_NAMES = {"mean": _lib.NORM_MEAN, "fz": _lib.NORM_MEAN, "self": _lib.NORM_SELF,
              "n": _lib.NORM_NATOM, "natom": _lib.NORM_NATOM}
PRECISION_NAMES = {"double": _lib.PREC_DOUBLE, "float64": _lib.PREC_DOUBLE,
                   "f64": _lib.PREC_DOUBLE, "single": _lib.PREC_SINGLE,
                   "float": _lib.PREC_SINGLE, "float32": _lib.PREC_SINGLE,
                   "f32": _lib.PREC_SINGLE}


# scheme_label (src/sqc_weights.f90:176-187)
WEIGHT_LABELS = {WEIGHT_NEUTRON: "neutron bound coherent scattering lengths",
                 WEIGHT_XRAY: "X-ray atomic form factors f(q)"}


class SqcalcError(Exception):
    """A failure the reference reports as ``ierr /= 0`` plus a message."""


def fortran_es(x, width=20, digits=12):
    """Fortran ESw.d edit descriptor (what sf_write_results prints)."""
    if x == 0.0 or not math.isfinite(x):
        if x == 0.0:
            body = "0." + "0" * digits + "E+00"
        else:
            body = "NaN" if math.isnan(x) else ("Infinity" if x > 0 else "-Infinity")
        return body.rjust(width)
    s = "%.*e" % (digits, x)
    mant, exp = s.split("e")
    e = int(exp)
    ex = ("E%+03d" % e) if abs(e) < 100 else ("%+04d" % e)
    return (mant + ex).rjust(width)


@dataclass
class KeptModes:
    """Kept modes in the reference's enumeration order (:352-381)."""
    hkl: np.ndarray
    qvec: np.ndarray
    qlen: np.ndarray
    gidx: np.ndarray


def enumerate_modes(cell: Cell, modes, qmin, qmax):
    """Vectorised restatement of sf_configure's enumeration, plane by plane."""
    b = cell.b  # b[j] = b_j
    m1, m2, m3 = (int(x) for x in modes)
    h1 = np.arange(m1) - (m1 + 1) // 2 + 1
    h2 = np.arange(m2) - (m2 + 1) // 2 + 1
    out_h, out_q, out_l, out_g = [], [], [], []
    H1, H2 = np.meshgrid(h1, h2, indexing="xy")  # H1 fastest
    H1 = H1.reshape(-1).astype(np.float64)
    H2 = H2.reshape(-1).astype(np.float64)
    for p3 in range(1, m3 + 1):
        h3 = p3 - (m3 + 1) // 2
        q = [b[0][r] * H1 + b[1][r] * H2 + b[2][r] * float(h3) for r in range(3)]
        ql = np.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2])
        keep = (ql <= qmax) & (ql >= qmin) & ~((H1 == 0) & (H2 == 0) & (h3 == 0))
        idx = np.nonzero(keep)[0]
        if idx.size == 0:
            continue
        out_h.append(np.stack([H1[idx], H2[idx], np.full(idx.size, float(h3))], 1).astype(np.int32))
        out_q.append(np.stack([q[0][idx], q[1][idx], q[2][idx]], 1))
        out_l.append(ql[idx])
        out_g.append(idx.astype(np.int64) + 1 + (p3 - 1) * m1 * m2)
    if not out_h:
        z = np.zeros((0, 3))
        return KeptModes(z.astype(np.int32), z, np.zeros(0), np.zeros(0, np.int64))
    return KeptModes(np.concatenate(out_h), np.concatenate(out_q), np.concatenate(out_l),
                     np.concatenate(out_g))


class GpuStructureFactor:
    """``sqcalc static --device gpu`` on libsqnufft (cf. cufinufft_structure_factor_t)."""

    def __init__(self, norm="mean", nq=500, qmin=0.0, qmax=20.0, eps=None, want_grid=False,
                 partials=True, faber_ziman=False, precision="double", device=0,
                 upsampfac=0.0, kernel_width=0, max_grid_modes=0, timing=False, xrd=None):
        self.norm = NORM_NAMES[norm] if isinstance(norm, str) else int(norm)
        self.nq = int(nq)
        self.qmin = float(qmin)
        self.qmax = float(qmax)
        self.precision = (PRECISION_NAMES[precision] if isinstance(precision, str)
                          else int(precision))
        # app/main.f90:191-198: float32 without --eps runs at 1e-5.
        if eps is None:
            eps = 1e-5 if self.precision == _lib.PREC_SINGLE else 1e-9
        self.eps = float(eps)
        self.want_grid = bool(want_grid)
        self.partials = bool(partials)
        self.faber_ziman = bool(faber_ziman)
        self.device = int(device)
        self.upsampfac = float(upsampfac)
        self.kernel_width = int(kernel_width)
        self.max_grid_modes = int(max_grid_modes)
        self.timing = bool(timing)
        self.xrd = xrd  # None or dict(lam=..., range=(lo, hi), step=..., lp=...)
        self.plan = None
        self.scheme = None
        self.natoms = 0
        self.ntypes = 0
        self.type_counts = None
        self.kept = None

    # --- sf_configure (:313-422) + gpu_setup (src/sqc_gpu.f90:108-210) -------
    def configure(self, frame, scheme: WeightScheme):
        self.scheme = scheme
        self.natoms = int(frame.natoms)
        self.cell = frame.cell
        maxtype = max(1, int(np.max(frame.type_id)))
        self.ntypes = max(maxtype, scheme.mapped_types())
        if np.any(frame.type_id < 1):
            raise SqcalcError("atom type id %d is outside the range given by -m"
                              % int(np.min(frame.type_id)))
        self.type_counts = np.bincount(frame.type_id, minlength=self.ntypes + 1)[1:]
        amp = xc = None
        if scheme.kind == WEIGHT_NEUTRON:
            amp = scheme.neutron_b(self.ntypes)
        elif scheme.kind == WEIGHT_XRAY:
            xc = scheme.xray_rows(self.ntypes)
        try:
            self.plan = _lib.Plan(frame.cell.flat(), frame.cell.origin, frame.type_id,
                                  ntypes=self.ntypes, weight=scheme.kind, amp_const=amp,
                                  xray_coef=xc, qmin=self.qmin, qmax=self.qmax, nq=self.nq,
                                  norm=self.norm, partials=self.partials,
                                  want_grid=self.want_grid, precision=self.precision,
                                  eps=self.eps, upsampfac=self.upsampfac,
                                  kernel_width=self.kernel_width, device=self.device,
                                  max_grid_modes=self.max_grid_modes, timing=self.timing,
                                  xrd=self.xrd)
        except _lib.SqnError as e:
            if e.code == 42:
                raise SqcalcError("reciprocal grid exceeds the limit of modes; reduce --qmax")
            raise SqcalcError(str(e))
        self.modes = self.plan.modes
        self.gridpoints = self.plan.gridpoints
        self.nmodes = self.plan.nmodes

    def accumulate_frame(self, frame):
        self.plan.accumulate(frame.pos)

    def accumulate_positions(self, pos):
        self.plan.accumulate(pos)

    @property
    def nframes(self):
        return self.plan.accumulators()["nframes"]

    # --- output (:657-827) ---------------------------------------------------
    def q_of_shell(self, s):
        dq = (self.qmax - self.qmin) / self.nq
        return self.qmin + (s + 0.5) * dq

    def results(self):
        S, Sp, Sg, nf = self.plan.finalize(self.faber_ziman, grid=self.want_grid)
        return S, Sp, Sg, nf

    def pair_columns(self):
        cols = []
        for t in range(1, self.ntypes + 1):
            for u in range(t, self.ntypes + 1):
                if self.type_counts[t - 1] == 0 or self.type_counts[u - 1] == 0:
                    continue
                cols.append((t, u, ("A(" if self.faber_ziman else "S(")
                             + self.scheme.pair_label(t, u) + ")"))
        return cols

    def write_results(self, shell_out=None, grid_out=None):
        S, Sp, Sg, _ = self.results()
        if shell_out is not None:
            fh = sys.stdout if shell_out == "-" else open(shell_out, "w")
            try:
                cols = self.pair_columns() if self.partials else []
                head = "# q S(q)" + "".join(" " + c[2] for c in cols)
                fh.write(head + "\n")
                for s in range(self.nq):
                    line = "%14.6f  %s" % (self.q_of_shell(s), fortran_es(S[s]))
                    for t, u, _ in cols:
                        line += "  " + fortran_es(Sp[t - 1, u - 1, s])
                    fh.write(line + "\n")
            finally:
                if fh is not sys.stdout:
                    fh.close()
        if grid_out is not None and self.want_grid:
            kept = enumerate_modes(self.cell, self.modes, self.qmin, self.qmax)
            with open(grid_out, "w") as fh:
                fh.write("# qx qy qz S(q)\n")
                for i in range(len(kept.qlen)):
                    q = kept.qvec[i]
                    fh.write("%14.8f  %14.8f  %14.8f  %s\n" % (q[0], q[1], q[2], fortran_es(Sg[i])))
        return S, Sp, Sg

    # --- HDF5 results (src/sqc_hdf5.f90) ------------------------------------
    def pair_list(self):
        """(a, b, label) of every pair of present types, a <= b, in the order of
        write_shell_partials (src/sqc_hdf5.f90:1322-1352)."""
        out = []
        for t in range(1, self.ntypes + 1):
            for u in range(t, self.ntypes + 1):
                if self.type_counts[t - 1] == 0 or self.type_counts[u - 1] == 0:
                    continue
                out.append((t, u, self.scheme.pair_label(t, u)))
        return out

    def _run_attrs(self, root):
        """The run attributes of hdf5_write_results (src/sqc_hdf5.f90:86-131)."""
        root.attr("nframes", int(self.nframes))
        root.attr("natoms", int(self.natoms))
        root.attr("nmodes", int(self.nmodes))
        root.attr("nq", int(self.nq))
        root.attr("qmin", float(self.qmin))
        root.attr("qmax", float(self.qmax))
        root.attr("eps", float(self.eps))
        root.attr("cell", np.asarray(self.cell.a, dtype=np.float64).reshape(3, 3))
        root.attr("weight", WEIGHT_LABELS.get(self.scheme.kind, "unit weights"))
        root.attr("norm", {_lib.NORM_SELF: "self", _lib.NORM_NATOM: "n"}.get(self.norm, "mean"))
        root.attr("device", "gpu")
        root.attr("precision", "single" if self.precision == _lib.PREC_SINGLE else "double")
        mapping = ",".join("%d:%s" % (t, self.scheme.species[t])
                           for t in range(1, self.scheme.mapped_types() + 1)
                           if self.scheme.species.get(t, ""))
        root.attr("mapping", mapping)

    def write_hdf5(self, path):
        """hdf5_write_results (src/sqc_hdf5.f90:46-210): the run attributes,
        /shell/{q,S,count} (+ /shell/S_partial/<pair>, /shell/pairs and the
        partial_normalization attribute) and, with --grid, /grid/{qx,qy,qz,S,h,k,l}."""
        S, Sp, Sg, _ = self.results()
        acc = self.plan.accumulators()
        root = h5file.Group()
        self._run_attrs(root)
        shell = root.group("shell")
        shell.dataset("q", np.array([self.q_of_shell(s) for s in range(self.nq)]))
        shell.dataset("S", np.asarray(S, dtype=np.float64))
        shell.dataset("count", np.asarray(acc["shell_count"], dtype=np.int64))
        pairs = self.pair_list() if self.partials else []
        if pairs and self.nq > 0:
            sp = shell.group("S_partial")
            for t, u, lab in pairs:
                sp.dataset(lab, np.asarray(Sp[t - 1, u - 1, :], dtype=np.float64))
            shell.dataset("pairs", [lab for _, _, lab in pairs], strlen=18)
            shell.attr("partial_normalization", "faber-ziman" if self.faber_ziman else "ovito")
        if self.want_grid:
            kept = enumerate_modes(self.cell, self.modes, self.qmin, self.qmax)
            grid = root.group("grid")
            for r, name in enumerate(("qx", "qy", "qz")):
                grid.dataset(name, kept.qvec[:, r])
            grid.dataset("S", np.asarray(Sg, dtype=np.float64))
            for r, name in enumerate(("h", "k", "l")):
                grid.dataset(name, kept.hkl[:, r].astype(np.int32))
        h5file.write_file(path, root)

    def write_xrd_hdf5(self, path):
        """hdf5_write_xrd (src/sqc_hdf5.f90:1050-1141) with write_xrd_partials
        (:1144-1200): the pattern's attributes and /xrd/{two_theta,I,count}
        (+ /xrd/I_partial/<pair> and /xrd/pairs)."""
        if not self.xrd:
            return None
        tth, I, Ip, cnt, nf = self.plan.xrd()
        lo, hi = self.xrd.get("range", (1.0, 179.0))
        root = h5file.Group()
        root.attr("lambda", float(self.xrd["lam"]))
        root.attr("two_theta_min", float(lo))
        root.attr("two_theta_max", float(hi))
        root.attr("step", float(self.plan.info.xrd_step))
        root.attr("bins", int(len(tth)))
        root.attr("nframes", int(nf))
        root.attr("natoms", int(self.natoms))
        root.attr("lorentz_polarization", "on" if self.xrd.get("lp", True) else "off")
        root.attr("intensity", "sum of |rho(q)|^2 over the reciprocal lattice points of the "
                  "bin, per atom and per frame")
        g = root.group("xrd")
        g.dataset("two_theta", np.asarray(tth, dtype=np.float64))
        g.dataset("I", np.asarray(I, dtype=np.float64))
        g.dataset("count", np.asarray(cnt, dtype=np.int64))
        pairs = self.pair_list() if (self.partials and len(tth) > 0) else []
        if pairs:
            sub = g.group("I_partial")
            for t, u, lab in pairs:
                sub.dataset(lab, np.asarray(Ip[t - 1, u - 1, :], dtype=np.float64))
            g.dataset("pairs", [lab for _, _, lab in pairs], strlen=18)
            g.attr("partial_normalization", "intensity: I = sum_a I(a-a) + 2 sum_{a<b} I(a-b)")
        h5file.write_file(path, root)
        return tth, I, Ip, cnt

    def write_xrd(self, path):
        """The powder pattern table of sf_write_xrd (src/sqc_structure_factor.f90:964-1031)."""
        if not self.xrd:
            return None
        tth, I, Ip, cnt, nf = self.plan.xrd()
        lo, hi = self.xrd.get("range", (1.0, 179.0))
        step = float(self.plan.info.xrd_step)
        cols = []
        if self.partials:
            for t in range(1, self.ntypes + 1):
                for u in range(t, self.ntypes + 1):
                    if self.type_counts[t - 1] == 0 or self.type_counts[u - 1] == 0:
                        continue
                    cols.append((t, u, "I(" + self.scheme.pair_label(t, u) + ")"))
        with open(path, "w") as fh:
            fh.write("# xrd: lambda %.6f A, 2theta %.4f to %.4f deg, step %.5f deg, %d bins, %s\n"
                     % (self.xrd["lam"], lo, hi, step, len(tth),
                        "1 frame" if nf == 1 else "%d frames" % nf))
            if self.xrd.get("lp", True):
                fh.write("# I(2theta) = sum over the reciprocal lattice points in each bin of "
                         "|rho(q)|^2 times the Lorentz-polarization factor, per atom\n")
            else:
                fh.write("# I(2theta) = sum over the reciprocal lattice points in each bin of "
                         "|rho(q)|^2, without the Lorentz-polarization factor, per atom\n")
            if cols:
                fh.write("# the pair columns add up to the total: "
                         "I = sum_a I(a-a) + 2 sum_{a<b} I(a-b)\n")
            fh.write("# 2theta[deg] I" + "".join(" " + c[2] for c in cols) + "\n")
            for k in range(len(tth)):
                line = "%12.4f  %s" % (tth[k], fortran_es(I[k]))
                for t, u, _ in cols:
                    line += "  " + fortran_es(Ip[t - 1, u - 1, k])
                fh.write(line + "\n")
        return tth, I, Ip, cnt

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None
