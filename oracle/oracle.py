"""CPU oracle for the static S(q) path of sqcalc (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use
this module, and only as the checker.  The product (sqcalc_b200 and
libsqnufft.so) never imports it.

Two oracles live here, both over ``_build/libsqoracle.so`` (see Makefile):

* ``direct_sq`` -- the FP64 direct sum of the reference's ``--method direct``
  (src/sqc_structure_factor.f90:1398-1515) with the shared grid, shell and
  normalisation bookkeeping (:313-451, :595-719).  This is the parity oracle.
* ``nufft_cpu_sq`` -- a CPU restatement of the NUFFT form (ES spreading,
  real-to-complex FFT through scipy's pocketfft, deconvolution, shell sums), the
  stand-in for the reference's FINUFFT CPU path; it is the timed CPU baseline.

Parity of the restatement is pinned by tests/golden (vectors from the
reference's own test/ref_sq.py and the known-answer cases of
test/test_sqcalc.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsqoracle.so")

WEIGHT_UNIT, WEIGHT_NEUTRON, WEIGHT_XRAY = 0, 1, 2
NORM_MEAN, NORM_SELF, NORM_NATOM = 1, 2, 3

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_lib = None


def build():
    """Compile the oracle library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.sqo_cell_setup.argtypes = [_dp, _dp, _dp]
        L.sqo_modes.argtypes = [_dp, ctypes.c_double, _ip]
        L.sqo_modes.restype = ctypes.c_int
        L.sqo_enumerate.argtypes = [_dp, _ip, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p]
        L.sqo_enumerate.restype = ctypes.c_int64
        L.sqo_shell_norms.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int32,
                                      ctypes.c_int32, _ip, ctypes.c_int64, _dp, _ip,
                                      ctypes.c_int32, _dp, _lp]
        L.sqo_direct_frame.argtypes = [ctypes.c_int64, _dp, _dp, _dp, _ip, ctypes.c_int32,
                                       ctypes.c_int, _dp, _dp, ctypes.c_int64, _dp, _dp, _ip,
                                       ctypes.c_int32, ctypes.c_int, _dp, _dp]
        L.sqo_accumulate_values.argtypes = [ctypes.c_int64, _dp, _ip, _lp, _dp, ctypes.c_void_p]
        L.sqo_wrap.argtypes = [ctypes.c_int64, _dp, _dp, _dp, _dp]
        L.sqo_amplitude.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_double]
        L.sqo_amplitude.restype = ctypes.c_double
        L.sqo_next235even.argtypes = [ctypes.c_int64]
        L.sqo_next235even.restype = ctypes.c_int64
        L.sqo_es_params.argtypes = [ctypes.c_double, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_double)]
        L.sqo_kernel_fseries.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
                                         ctypes.c_int32, _dp]
        L.sqo_spread_real.argtypes = [ctypes.c_int64, _dp, _ip, _dp, ctypes.c_int32, _lp,
                                      ctypes.c_int32, ctypes.c_double, _dp]
        L.sqo_bin_halfspace.argtypes = [_dp, ctypes.c_int32, _lp, _ip, _dp, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int32, _dp, _dp, _dp,
                                        ctypes.c_void_p, _dp, _dp]
        L.sqo_direct_grad.argtypes = [ctypes.c_int64, _dp, _dp, _dp, _dp, ctypes.c_int64, _dp,
                                      _ip, _dp, _dp]
        L.sqo_dirft3d1.argtypes = [ctypes.c_int64, _dp, _dp, _dp, _dp, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                   ctypes.c_int64, ctypes.c_int32, _dp]
        _lib = L
    return _lib


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


@dataclass
class Grid:
    """Reciprocal grid of sf_configure (src/sqc_structure_factor.f90:313-422)."""
    cell: np.ndarray
    recip: np.ndarray
    modes: np.ndarray
    hkl: np.ndarray
    qvec: np.ndarray
    qlen: np.ndarray
    gidx: np.ndarray
    shell: np.ndarray
    nq: int
    qmin: float
    qmax: float

    @property
    def nmodes(self):
        return len(self.qlen)

    @property
    def gridpoints(self):
        return int(np.prod(self.modes.astype(np.int64)))


def configure_grid(cell, qmin, qmax, nq):
    """cell: (3, 3) array with the lattice vectors in its ROWS (cell[i] = a_i)."""
    L = lib()
    flat = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    inv = np.zeros(9)
    recip = np.zeros(9)
    L.sqo_cell_setup(flat, inv, recip)
    modes = np.zeros(3, dtype=np.int32)
    if L.sqo_modes(flat, float(qmax), modes) != 0:
        raise ValueError("degenerate simulation cell")
    n = L.sqo_enumerate(recip, modes, float(qmin), float(qmax), int(nq), None, None, None, None,
                        None)
    hkl = np.zeros((n, 3), dtype=np.int32)
    qvec = np.zeros((n, 3))
    qlen = np.zeros(n)
    gidx = np.zeros(n, dtype=np.int64)
    shell = np.zeros(n, dtype=np.int32)
    L.sqo_enumerate(recip, modes, float(qmin), float(qmax), int(nq), hkl.ctypes.data,
                    qvec.ctypes.data, qlen.ctypes.data, gidx.ctypes.data, shell.ctypes.data)
    return Grid(flat.reshape(3, 3), recip.reshape(3, 3), modes, hkl, qvec, qlen, gidx, shell,
                int(nq), float(qmin), float(qmax))


@dataclass
class Weights:
    """Per-type amplitudes: kind, b per type id (neutron) and IT92 rows (x-ray).

    amp_const[t-1] / xray[t-1] belong to LAMMPS type id t.
    """
    kind: int = WEIGHT_UNIT
    amp_const: np.ndarray = field(default_factory=lambda: np.ones(1))
    xray: np.ndarray = field(default_factory=lambda: np.zeros((1, 9)))

    def padded(self, ntypes):
        a = np.ones(ntypes)
        x = np.zeros((ntypes, 9))
        n = min(ntypes, len(self.amp_const))
        a[:n] = self.amp_const[:n]
        m = min(ntypes, len(self.xray))
        x[:m] = self.xray[:m]
        return _c(a, np.float64), _c(x.reshape(-1), np.float64)


@dataclass
class Accumulators:
    """The per-run accumulators of structure_factor_t (:84-137)."""
    num: np.ndarray
    den: np.ndarray
    shell_count: np.ndarray
    partial_num: np.ndarray | None  # (ntypes, ntypes, nq), [ia-1, ib-1, s]
    gnum: np.ndarray | None
    gden: np.ndarray | None
    nframes: int
    natoms: int
    type_counts: np.ndarray

    def shell_value(self):
        """sf_shell_value (:657-665)."""
        f = max(self.nframes, 1)
        out = np.zeros_like(self.num)
        m = self.den > 0
        out[m] = self.num[m] / (f * self.den[m])
        return out

    def partial_value(self, ia, ib, faber_ziman=False):
        """sf_partial_value (:696-719) for type ids ia <= ib (1-based)."""
        f = max(self.nframes, 1)
        cnt = np.maximum(self.shell_count, 1).astype(np.float64)
        v = self.partial_num[ia - 1, ib - 1] / (f * float(self.natoms) * cnt)
        if not faber_ziman:
            return v
        xa = self.type_counts[ia - 1] / self.natoms
        xb = self.type_counts[ib - 1] / self.natoms
        if xa * xb <= 0:
            return np.zeros_like(v)
        return (v - (xa if ia == ib else 0.0)) / (xa * xb) + 1.0

    def grid_value(self, grid: Grid):
        """sf_grid_value (:757-768) of every kept mode."""
        f = max(self.nframes, 1)
        g = grid.gidx - 1
        out = np.zeros(grid.nmodes)
        d = self.gden[g]
        m = d > 0
        out[m] = self.gnum[g][m] / (f * d[m])
        return out


def type_counts_of(type_id, ntypes):
    return np.bincount(np.asarray(type_id, dtype=np.int64), minlength=ntypes + 1)[1:ntypes + 1]


def _norm_tables(grid, weights, type_id, ntypes, norm, want_grid):
    L = lib()
    counts = _c(type_counts_of(type_id, ntypes), np.int32)
    amp, xr = weights.padded(ntypes)
    den = np.zeros(grid.nq)
    cnt = np.zeros(grid.nq, dtype=np.int64)
    L.sqo_shell_norms(int(norm), int(weights.kind), amp, xr, int(len(type_id)), int(ntypes),
                      counts, grid.nmodes, _c(grid.qlen, np.float64), _c(grid.shell, np.int32),
                      grid.nq, den, cnt)
    gden = None
    if want_grid:
        gden = np.zeros(grid.gridpoints)
        for i in range(grid.nmodes):
            gden[grid.gidx[i] - 1] = _mode_den(norm, weights, counts, len(type_id), ntypes,
                                               grid.qlen[i])
    return counts, den, cnt, gden


def _mode_den(norm, weights, counts, natoms, ntypes, q):
    if norm == NORM_NATOM:
        return float(natoms)
    L = lib()
    amp, xr = weights.padded(ntypes)
    sw = sw2 = 0.0
    for t in range(1, ntypes + 1):
        if counts[t - 1] <= 0:
            continue
        w = L.sqo_amplitude(int(weights.kind), amp, xr, t, float(q))
        sw += counts[t - 1] * w
        sw2 += counts[t - 1] * w * w
    return sw * sw / natoms if norm == NORM_MEAN else sw2


def direct_sq(frames, type_id, cell, origin, weights: Weights, qmin, qmax, nq, norm=NORM_MEAN,
              partials=True, want_grid=False, ntypes=None):
    """FP64 direct-sum S(q) over a list of frames (each (N, 3) Cartesian positions)."""
    L = lib()
    type_id = _c(type_id, np.int32)
    ntypes = int(ntypes or max(int(type_id.max()), 1))
    grid = configure_grid(cell, qmin, qmax, nq)
    counts, den, cnt, gden = _norm_tables(grid, weights, type_id, ntypes, norm, want_grid)
    amp, xr = weights.padded(ntypes)
    flat = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    org = _c(origin, np.float64)
    num = np.zeros(nq)
    pnum = np.zeros(ntypes * ntypes * nq) if partials else np.zeros(1)
    gnum = np.zeros(grid.gridpoints) if want_grid else None
    inten = np.zeros(grid.nmodes)
    qvec = _c(grid.qvec, np.float64).reshape(-1)
    for pos in frames:
        pos = _c(pos, np.float64).reshape(-1)
        L.sqo_direct_frame(len(type_id), pos, flat, org, type_id, ntypes, int(weights.kind), amp,
                           xr, grid.nmodes, qvec, _c(grid.qlen, np.float64),
                           _c(grid.shell, np.int32), nq, int(bool(partials)), inten, pnum)
        L.sqo_accumulate_values(grid.nmodes, inten, _c(grid.shell, np.int32),
                                _c(grid.gidx, np.int64), num,
                                gnum.ctypes.data if gnum is not None else None)
    pn = pnum.reshape(nq, ntypes, ntypes).transpose(2, 1, 0) if partials else None
    acc = Accumulators(num, den, cnt, pn, gnum, gden, len(frames), len(type_id), counts)
    return grid, acc


def es_params(eps, sigma):
    w = ctypes.c_int32()
    beta = ctypes.c_double()
    lib().sqo_es_params(float(eps), float(sigma), ctypes.byref(w), ctypes.byref(beta))
    return int(w.value), float(beta.value)


def nufft_cpu_sq(frames, type_id, cell, origin, weights: Weights, qmin, qmax, nq, eps=1e-6,
                 sigma=1.25, norm=NORM_MEAN, partials=True, workers=None, ntypes=None):
    """CPU NUFFT restatement: spread (C/OpenMP) -> rfftn (scipy, ``workers`` threads)
    -> deconvolve + shell sums (C/OpenMP).  Unit and neutron weights only."""
    import scipy.fft

    if weights.kind == WEIGHT_XRAY:
        raise NotImplementedError("the CPU NUFFT baseline covers q-independent weights")
    L = lib()
    type_id = _c(type_id, np.int32)
    ntypes = int(ntypes or max(int(type_id.max()), 1))
    grid_modes = np.zeros(3, dtype=np.int32)
    flat = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    L.sqo_modes(flat, float(qmax), grid_modes)
    inv = np.zeros(9)
    recip = np.zeros(9)
    L.sqo_cell_setup(flat, inv, recip)
    w, beta = es_params(eps, sigma)
    nf = np.array([L.sqo_next235even(max(int(np.ceil(sigma * m)), 2 * w)) for m in grid_modes],
                  dtype=np.int64)
    ph = [np.zeros((m - 1) // 2 + 1) for m in grid_modes]
    for d in range(3):
        L.sqo_kernel_fseries(int(nf[d]), w, beta, int((grid_modes[d] - 1) // 2), ph[d])
    counts = type_counts_of(type_id, ntypes)
    present = [t for t in range(1, ntypes + 1) if counts[t - 1] > 0]
    amp_t, _ = weights.padded(ntypes)
    if partials or len(present) > 1 and weights.kind == WEIGHT_XRAY:
        tr_types = present
        tr_of = np.full(len(type_id), -1, dtype=np.int32)
        for k, t in enumerate(present):
            tr_of[type_id == t] = k
        strength = np.ones(len(type_id))
        tr_amp = np.array([amp_t[t - 1] if weights.kind == WEIGHT_NEUTRON else 1.0
                           for t in tr_types])
    else:
        tr_types = [0]
        tr_of = np.zeros(len(type_id), dtype=np.int32)
        strength = np.array([amp_t[t - 1] if weights.kind == WEIGHT_NEUTRON else 1.0
                             for t in type_id])
        tr_amp = np.ones(1)
    ntr = len(tr_types)
    num = np.zeros(nq)
    npair = ntr * (ntr + 1) // 2
    ppack = np.zeros(npair * nq)
    g = np.zeros(int(ntr * nf[0] * nf[1] * nf[2]))
    frac = np.zeros(3 * len(type_id))
    for pos in frames:
        L.sqo_wrap(len(type_id), _c(pos, np.float64).reshape(-1), flat, _c(origin, np.float64),
                   frac)
        L.sqo_spread_real(len(type_id), frac, tr_of, _c(strength, np.float64), ntr, nf, w, beta, g)
        G = scipy.fft.rfftn(g.reshape(ntr, nf[2], nf[1], nf[0]), axes=(1, 2, 3),
                            workers=workers or os.cpu_count())
        G = np.ascontiguousarray(G).view(np.float64).reshape(-1)
        L.sqo_bin_halfspace(G, ntr, nf, grid_modes, recip, float(qmin), float(qmax), nq, ph[0],
                            ph[1], ph[2], _c(tr_amp, np.float64).ctypes.data, num, ppack)
    grid = configure_grid(cell, qmin, qmax, nq)
    _, den, cnt, _ = _norm_tables(grid, weights, type_id, ntypes, norm, False)
    pn = None
    if partials:
        pn = np.zeros((ntypes, ntypes, nq))
        p = 0
        ppack = ppack.reshape(npair, nq)
        for a in range(ntr):
            for b in range(a, ntr):
                pn[tr_types[a] - 1, tr_types[b] - 1] = ppack[p]
                p += 1
    acc = Accumulators(num, den, cnt, pn, None, None, len(frames), len(type_id), counts)
    return grid, acc, dict(w=w, beta=beta, nf=nf.tolist(), sigma=sigma)


def direct_grad(pos, strength, cell, origin, grid: Grid, wgt):
    """FP64 direct-sum gradient of sum_s wgt[s] * num(s) for one frame."""
    out = np.zeros(3 * len(strength))
    lib().sqo_direct_grad(len(strength), _c(pos, np.float64).reshape(-1),
                          _c(np.asarray(cell).reshape(9), np.float64), _c(origin, np.float64),
                          _c(strength, np.float64), grid.nmodes,
                          _c(grid.qvec, np.float64).reshape(-1), _c(grid.shell, np.int32),
                          _c(wgt, np.float64), out)
    return out.reshape(-1, 3)


def dirft3d1(x, y, z, c, n_modes, iflag=1, modeord=0):
    """Direct type-1 sum; c (ntr, M) complex -> fk (ntr, N3, N2, N1) complex."""
    c = np.atleast_2d(np.asarray(c, dtype=np.complex128))
    ntr, M = c.shape
    N1, N2, N3 = (int(n) for n in n_modes)
    cf = np.ascontiguousarray(c).view(np.float64).reshape(-1)
    out = np.zeros(2 * ntr * N1 * N2 * N3)
    lib().sqo_dirft3d1(M, _c(x, np.float64), _c(y, np.float64), _c(z, np.float64), cf, ntr,
                       int(iflag), N1, N2, N3, int(modeord), out)
    return out.view(np.complex128).reshape(ntr, N3, N2, N1)


def two_theta_deg(q, lam):
    """two_theta_deg (src/sqc_structure_factor.f90:907-914)."""
    st = np.clip(np.asarray(q) * lam / (4.0 * np.pi), -1.0, 1.0)
    return 2.0 * np.arcsin(st) * 180.0 / np.pi


def lorentz_polarization(tth_deg):
    """lorentz_polarization (src/sqc_structure_factor.f90:917-924)."""
    tth = np.radians(tth_deg)
    th = 0.5 * tth
    return (1.0 + np.cos(tth) ** 2) / (np.sin(th) ** 2 * np.cos(th))


def xrd_bins(cell, lam, tmin, tmax, step=0.0):
    """Bin count and width of sf_configure_xrd (:846-890), every direction periodic."""
    a = np.asarray(cell, dtype=np.float64)
    if not step > 0.0:
        vol = abs(np.linalg.det(a))
        widths = [vol / np.linalg.norm(np.cross(a[(i + 1) % 3], a[(i + 2) % 3])) for i in range(3)]
        theta_max = min(0.5 * np.radians(tmax), np.radians(60.0))
        step = (lam / (min(widths) * np.cos(theta_max))) / (np.pi / 180.0)
    nb = max(1, int(np.ceil((tmax - tmin) / step)))
    return nb, (tmax - tmin) / nb


def direct_density(pos, type_id, cell, hkl):
    """rho_a(q_h) = sum_{j of type a} exp(+i q_h . r_j) for the lattice points hkl
    (q_h = h1 b1 + h2 b2 + h3 b3), absolute positions, species in ascending type id:
    the direct sum of dyn_accumulate (src/sqc_dynamics.f90:860-875).  Returns
    complex128 (nspecies, nmodes)."""
    L = lib()
    flat = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    inv = np.zeros(9)
    recip = np.zeros(9)
    L.sqo_cell_setup(flat, inv, recip)
    q = np.asarray(hkl, dtype=np.float64).reshape(-1, 3) @ recip.reshape(3, 3)
    type_id = np.asarray(type_id)
    pos = np.asarray(pos, dtype=np.float64)
    out = []
    for t in np.unique(type_id):
        out.append(np.exp(1j * (pos[type_id == t] @ q.T)).sum(axis=0))
    return np.stack(out)


def direct_xrd(frames, type_id, cell, origin, weights: Weights, lam, tmin, tmax, step=0.0,
               lp=True, ntypes=None):
    """FP64 direct-sum powder pattern over the kept modes of the q range the
    reference derives from the two-theta range (src/sqc_options.f90:650-651):
    I(bin) = sum_frames sum_{q in bin} |sum_a w_a(q) rho_a(q)|^2 LP / (nframes N) and
    I_ab the same with w_a w_b Re(rho_a rho_b*) (sf_accumulate_values :616-619,
    sf_accumulate_xrd_partials :538-588, sf_write_xrd :964-1031).  Small systems
    only (N x kept modes complex exponentials per frame)."""
    type_id = np.asarray(type_id, dtype=np.int32)
    T = int(ntypes or type_id.max())
    qmin = 4.0 * np.pi * np.sin(0.5 * np.radians(tmin)) / lam
    qmax = 4.0 * np.pi * np.sin(0.5 * np.radians(tmax)) / lam
    grid = configure_grid(cell, qmin, qmax, 10)
    nb, step = xrd_bins(cell, lam, tmin, tmax, step)
    tth = two_theta_deg(grid.qlen, lam)
    b = np.clip(((tth - tmin) / step).astype(np.int64), 0, nb - 1)
    wt = lorentz_polarization(tth) if lp else np.ones_like(tth)
    amp, xr = weights.padded(T)
    amp = np.asarray(amp, dtype=np.float64).reshape(-1)
    xr = np.asarray(xr, dtype=np.float64).reshape(-1, 9)
    if weights.kind == WEIGHT_XRAY:
        s = (grid.qlen / (4.0 * np.pi)) ** 2
        w = np.stack([xr[t, 8] + sum(xr[t, i] * np.exp(-xr[t, 4 + i] * s) for i in range(4))
                      for t in range(T)])
    elif weights.kind == WEIGHT_NEUTRON:
        w = np.stack([np.full(grid.nmodes, amp[t]) for t in range(T)])
    else:
        w = np.ones((T, grid.nmodes))
    I = np.zeros(nb)
    Ip = np.zeros((T, T, nb))
    for pos in frames:
        d = np.asarray(pos, dtype=np.float64) - np.asarray(origin)
        rho = np.zeros((T, grid.nmodes), dtype=np.complex128)
        for t in range(T):
            sel = d[type_id == t + 1]
            if len(sel):
                rho[t] = np.exp(1j * (sel @ grid.qvec.T)).sum(axis=0)
        tot = (w * rho).sum(axis=0)
        np.add.at(I, b, np.abs(tot) ** 2 * wt)
        for ta in range(T):
            for tb in range(ta, T):
                v = w[ta] * w[tb] * np.real(rho[ta] * np.conj(rho[tb])) * wt
                np.add.at(Ip[ta, tb], b, v)
    norm = len(frames) * len(type_id)
    cnt = np.bincount(b, minlength=nb)
    return tmin + (np.arange(nb) + 0.5) * step, I / norm, Ip / norm, cnt, qmin, qmax


def direct_sq_separable(frames, type_id, cell, origin, weights: Weights, qmin, qmax, nq,
                        norm=NORM_MEAN, partials=True, ntypes=None, slab_modes=None):
    """The FP64 direct sum of ``direct_sq`` (direct_accumulate,
    src/sqc_structure_factor.f90:1398-1515, on the wrapped positions r = A s of
    :1431-1435) evaluated slab by slab for grids far too large for the per-mode
    loop: with s the wrapped fractional coordinates, q_h . (A s) = 2 pi h . s, so
    exp(i q_h . r_j) = E1[h1, j] E2[h2, j] E3[h3, j] with E_d[h, j] = exp(2 pi i h s_jd)
    and, for one h3 slab, rho_a[h1, h2] = sum_{j of a} E1[h1, j] (E2[h2, j] E3[h3, j])
    is one complex matrix product per type.  The kept test, |q| and the shell of
    every mode use the reference's FP64 operation order (:366-399, as
    ``sqo_enumerate``), so the kept set and the shells are those of ``direct_sq``;
    den and shell_count follow mode_denominator (:425-451).  Only the evaluation
    order of the sum over atoms differs from ``direct_sq`` (agreement ~1e-13).
    Unit and neutron weights (q-independent amplitudes).  Returns (modes, acc)."""
    if weights.kind == WEIGHT_XRAY:
        raise ValueError("direct_sq_separable takes unit or neutron weights")
    L = lib()
    type_id = _c(type_id, np.int32)
    natoms = len(type_id)
    ntypes = int(ntypes or max(int(type_id.max()), 1))
    flat = _c(np.asarray(cell, dtype=np.float64).reshape(9), np.float64)
    inv = np.zeros(9)
    recip = np.zeros(9)
    L.sqo_cell_setup(flat, inv, recip)
    modes = np.zeros(3, dtype=np.int32)
    if L.sqo_modes(flat, float(qmax), modes) != 0:
        raise ValueError("degenerate simulation cell")
    hm = (modes.astype(np.int64) - 1) // 2
    b = recip  # b_j = recip[3 j : 3 j + 3]
    dq = (qmax - qmin) / float(nq)
    counts = type_counts_of(type_id, ntypes)
    amp, _ = weights.padded(ntypes)
    present = [t for t in range(1, ntypes + 1) if counts[t - 1] > 0]
    members = {t: np.nonzero(type_id == t)[0] for t in present}
    # per-mode denominator: q-independent for unit / neutron weights
    mode_den = _mode_den(norm, weights, counts, natoms, ntypes, 0.0)
    h1 = np.arange(-hm[0], hm[0] + 1, dtype=np.float64)[:, None]
    h2 = np.arange(-hm[1], hm[1] + 1, dtype=np.float64)[None, :]
    num = np.zeros(nq)
    cnt = np.zeros(nq, dtype=np.int64)
    pn = np.zeros((ntypes, ntypes, nq))
    frac_all = []
    for pos in frames:
        frac = np.zeros(3 * natoms)
        L.sqo_wrap(natoms, _c(pos, np.float64).reshape(-1), flat, _c(origin, np.float64), frac)
        frac_all.append(frac.reshape(natoms, 3))
    E = [[np.exp(2j * np.pi * np.arange(-hm[d], hm[d] + 1)[:, None] * fr[None, :, d])
          for d in range(3)] for fr in frac_all]
    for k3 in range(-int(hm[2]), int(hm[2]) + 1):
        # |q| in the reference's order: q_r = (b1_r h1 + b2_r h2) + b3_r h3
        q = [(b[r] * h1 + b[3 + r] * h2) + b[6 + r] * float(k3) for r in range(3)]
        ql = np.sqrt((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2])
        keep = (ql <= qmax) & (ql >= qmin)
        if k3 == 0:
            keep[hm[0], hm[1]] = False
        if not keep.any():
            continue
        sh = np.clip(((ql[keep] - qmin) / dq).astype(np.int64), 0, nq - 1)
        cnt += np.bincount(sh, minlength=nq)
        for f in range(len(frames)):
            E1, E2, E3 = E[f]
            rho = {}
            for t in present:
                j = members[t]
                B = E2[:, j] * E3[k3 + hm[2], j][None, :]
                rho[t] = (E1[:, j] @ B.T)[keep]
            tot = sum(amp[t - 1] * rho[t] for t in present)
            num += np.bincount(sh, weights=(tot.real * tot.real + tot.imag * tot.imag),
                               minlength=nq)
            if partials:
                for ia in present:
                    for ib in present:
                        if ib < ia:
                            continue
                        v = rho[ia].real * rho[ib].real + rho[ia].imag * rho[ib].imag
                        pn[ia - 1, ib - 1] += np.bincount(sh, weights=v, minlength=nq)
    den = cnt.astype(np.float64) * mode_den
    acc = Accumulators(num, den, cnt, pn if partials else None, None, None, len(frames), natoms,
                       counts)
    return modes, acc
