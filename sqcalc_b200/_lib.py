"""ctypes binding of libsqnufft.so (the C ABI in include/sqnufft.h).

This is the Python counterpart of sqcalc's iso_c_binding module for the GPU
method (src/sqc_cufinufft.f90): a 1:1 mirror of the C structs and functions,
nothing more.  The library is loaded from this package directory; a missing or
stale build is an error, never a silent fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsqnufft.so")

ABI_VERSION = 2
OK, WARN_EPS_TOO_SMALL = 0, 1
WEIGHT_UNIT, WEIGHT_NEUTRON, WEIGHT_XRAY = 0, 1, 2
NORM_MEAN, NORM_SELF, NORM_NATOM = 1, 2, 3
PREC_DOUBLE, PREC_SINGLE = 0, 1
HOST, DEVICE = 0, 1
FLAG_TIMING = 1
FLAG_GRAD = 2
FLAG_CUFFT = 8
FLAG_AUTOTUNE = 128

# Every symbol include/sqnufft.h declares.
EXPORTS = (
    "sqn_abi_version", "sqn_error_string", "sqn_default_desc", "sqn_plan_create",
    "sqn_plan_info_get", "sqn_accumulate_frames", "sqn_sync", "sqn_get_accumulators",
    "sqn_peek_num_async", "sqn_finalize", "sqn_reset", "sqn_stage_times", "sqn_launch_count",
    "sqn_plan_destroy", "sqn_spread_frame_noalloc", "sqn_sq_grad", "sqn_accumulator_view",
    "sqn_set_frame_count", "sqn_batch_create", "sqn_batch_accumulate", "sqn_batch_sync",
    "sqn_batch_plan", "sqn_batch_graph_launches", "sqn_batch_launch_count",
    "sqn_batch_multi", "sqn_batch_destroy", "sqn_type1_default_opts",
    "sqn_type1_makeplan", "sqn_type1f_makeplan", "sqn_type1_setpts", "sqn_type1f_setpts",
    "sqn_type1_execute", "sqn_type1f_execute", "sqn_type1_destroy", "sqn_dump_open",
    "sqn_dump_next", "sqn_dump_last_error", "sqn_dump_rewind", "sqn_dump_close",
    "sqn_accumulate_dump", "sqn_get_xrd", "sqn_density_modes", "sqn_join",
)
ERR_DUMP = 50
ERR_SCRATCH_LIMIT = 49
ERR_INVALID_ARGUMENT = 21
ERR_NUM_NU_PTS_INVALID = 20
NOALLOC_SCRATCH_BYTES = 32 * 1024 * 1024


class SqnDesc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("cell", ctypes.c_double * 9),
        ("origin", ctypes.c_double * 3),
        ("natoms", ctypes.c_int64),
        ("type_id", ctypes.POINTER(ctypes.c_int32)),
        ("ntypes", ctypes.c_int32),
        ("weight", ctypes.c_int32),
        ("amp_const", ctypes.POINTER(ctypes.c_double)),
        ("xray_coef", ctypes.POINTER(ctypes.c_double)),
        ("qmin", ctypes.c_double),
        ("qmax", ctypes.c_double),
        ("nq", ctypes.c_int32),
        ("norm", ctypes.c_int32),
        ("partials", ctypes.c_int32),
        ("want_grid", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("eps", ctypes.c_double),
        ("upsampfac", ctypes.c_double),
        ("kernel_width", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("max_grid_modes", ctypes.c_int64),
        ("stream", ctypes.c_void_p),
        ("xrd_lambda", ctypes.c_double),
        ("xrd_2theta_min", ctypes.c_double),
        ("xrd_2theta_max", ctypes.c_double),
        ("xrd_step", ctypes.c_double),
        ("xrd_lp", ctypes.c_int32),
        ("reserved2", ctypes.c_int32),
    ]


class SqnInfo(ctypes.Structure):
    _fields_ = [
        ("modes", ctypes.c_int32 * 3),
        ("kernel_width", ctypes.c_int32),
        ("nf", ctypes.c_int64 * 3),
        ("gridpoints", ctypes.c_int64),
        ("nmodes", ctypes.c_int64),
        ("upsampfac", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("eps_used", ctypes.c_double),
        ("ntransforms", ctypes.c_int32),
        ("nspecies", ctypes.c_int32),
        ("device_bytes", ctypes.c_int64),
        ("tile", ctypes.c_int64 * 3),
        ("natoms", ctypes.c_int64),
        ("xrd_bins", ctypes.c_int32),
        ("pruned_fft512", ctypes.c_int32),
        ("xrd_step", ctypes.c_double),
        ("autotuned", ctypes.c_int32),
        ("tune_candidates", ctypes.c_int32),
        ("tune_ms", ctypes.c_double),
    ]


class Type1Opts(ctypes.Structure):
    _fields_ = [
        ("gpu_device_id", ctypes.c_int32),
        ("modeord", ctypes.c_int32),
        ("upsampfac", ctypes.c_double),
        ("gpu_stream", ctypes.c_void_p),
    ]


class SqnError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = int(code)
        super().__init__("%s%s (status %d)" % (where + ": " if where else "",
                                               error_string(code), self.code))


_lib = None


def load():
    """Load libsqnufft.so from the package directory (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libsqnufft.so is not built; run `python -m sqcalc_b200.build` "
                          "(expected at %s)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, i64 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64
    L.sqn_abi_version.restype = ctypes.c_int
    L.sqn_error_string.argtypes = [ctypes.c_int]
    L.sqn_error_string.restype = ctypes.c_char_p
    L.sqn_default_desc.argtypes = [ctypes.POINTER(SqnDesc)]
    L.sqn_plan_create.argtypes = [ctypes.POINTER(SqnDesc), ctypes.POINTER(vp)]
    L.sqn_plan_info_get.argtypes = [vp, ctypes.POINTER(SqnInfo)]
    L.sqn_accumulate_frames.argtypes = [vp, vp, i64, ctypes.c_int32]
    L.sqn_sync.argtypes = [vp]
    L.sqn_get_accumulators.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.sqn_peek_num_async.argtypes = [vp, vp]
    L.sqn_finalize.argtypes = [vp, ctypes.c_int32, vp, vp, vp, vp]
    L.sqn_reset.argtypes = [vp]
    L.sqn_stage_times.argtypes = [vp, dp, ctypes.c_int32]
    L.sqn_launch_count.argtypes = [vp]
    L.sqn_launch_count.restype = i64
    L.sqn_plan_destroy.argtypes = [vp]
    L.sqn_sq_grad.argtypes = [vp, vp, ctypes.c_int32, vp, vp, vp]
    L.sqn_accumulator_view.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(i64),
                                       ctypes.POINTER(i64)]
    L.sqn_set_frame_count.argtypes = [vp, i64]
    L.sqn_batch_create.argtypes = [ctypes.POINTER(SqnDesc), ctypes.c_int32, vp, ctypes.POINTER(vp)]
    L.sqn_batch_accumulate.argtypes = [vp, ctypes.POINTER(vp), i64, ctypes.c_int32]
    L.sqn_batch_sync.argtypes = [vp]
    L.sqn_batch_plan.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(vp)]
    L.sqn_batch_graph_launches.argtypes = [vp]
    L.sqn_batch_graph_launches.restype = i64
    L.sqn_batch_launch_count.argtypes = [vp]
    L.sqn_batch_launch_count.restype = i64
    L.sqn_batch_multi.argtypes = [vp]
    L.sqn_batch_multi.restype = ctypes.c_int32
    L.sqn_batch_destroy.argtypes = [vp]
    L.sqn_type1_default_opts.argtypes = [ctypes.POINTER(Type1Opts)]
    L.sqn_type1_default_opts.restype = None
    L.sqn_type1_makeplan.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(i64),
                                     ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                     ctypes.POINTER(vp), ctypes.POINTER(Type1Opts)]
    L.sqn_type1f_makeplan.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(i64),
                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                      ctypes.POINTER(vp), ctypes.POINTER(Type1Opts)]
    for name in ("sqn_type1_setpts", "sqn_type1f_setpts"):
        getattr(L, name).argtypes = [vp, i64, vp, vp, vp]
    for name in ("sqn_type1_execute", "sqn_type1f_execute"):
        getattr(L, name).argtypes = [vp, vp, vp]
    L.sqn_type1_destroy.argtypes = [vp]
    L.sqn_dump_open.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(vp)]
    L.sqn_dump_next.argtypes = [vp, i64, ctypes.POINTER(i64), ctypes.POINTER(i64), vp, vp, vp,
                                vp]
    L.sqn_dump_last_error.argtypes = [vp]
    L.sqn_dump_rewind.argtypes = [vp]
    L.sqn_dump_close.argtypes = [vp]
    L.sqn_accumulate_dump.argtypes = [vp, vp, i64, vp, ctypes.POINTER(i64)]
    L.sqn_get_xrd.argtypes = [vp, vp, vp, vp, vp, vp]
    L.sqn_density_modes.argtypes = [vp, vp, ctypes.c_int32, vp, i64, vp]
    L.sqn_join.argtypes = [vp]
    L.sqn_spread_frame_noalloc.argtypes = [vp, i64, vp, ctypes.c_int32, vp, vp, vp, vp,
                                           ctypes.c_int32, ctypes.c_double, vp, vp]
    if L.sqn_abi_version() != ABI_VERSION:
        raise ImportError("libsqnufft.so ABI %d, binding expects %d"
                          % (L.sqn_abi_version(), ABI_VERSION))
    _lib = L
    return L


def error_string(code):
    try:
        return load().sqn_error_string(int(code)).decode()
    except ImportError:
        return "status %d" % code


def check(code, where=""):
    if code > WARN_EPS_TOO_SMALL:
        raise SqnError(code, where)
    return code


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Plan:
    """One sqn_plan: configure once, accumulate frames, read accumulators."""

    def __init__(self, cell, origin, type_id, ntypes=None, weight=WEIGHT_UNIT, amp_const=None,
                 xray_coef=None, qmin=0.0, qmax=20.0, nq=500, norm=NORM_MEAN, partials=True,
                 want_grid=False, precision=PREC_DOUBLE, eps=1e-9, upsampfac=0.0,
                 kernel_width=0, device=0, max_grid_modes=0, timing=False, stream=None,
                 grad=False, cufft=False, xrd=None, autotune=False):
        L = load()
        self._L = L
        d = self._describe(cell, origin, type_id, ntypes, weight, amp_const, xray_coef, qmin,
                           qmax, nq, norm, partials, want_grid, precision, eps, upsampfac,
                           kernel_width, device, max_grid_modes, timing, stream, grad, cufft,
                           xrd, autotune)
        h = ctypes.c_void_p()
        self.status = check(L.sqn_plan_create(ctypes.byref(d), ctypes.byref(h)), "sqn_plan_create")
        self._attach(h, owned=True)

    def _describe(self, cell, origin, type_id, ntypes=None, weight=WEIGHT_UNIT, amp_const=None,
                  xray_coef=None, qmin=0.0, qmax=20.0, nq=500, norm=NORM_MEAN, partials=True,
                  want_grid=False, precision=PREC_DOUBLE, eps=1e-9, upsampfac=0.0,
                  kernel_width=0, device=0, max_grid_modes=0, timing=False, stream=None,
                  grad=False, cufft=False, xrd=None, autotune=False):
        """Fill an SqnDesc; the arrays it points to are kept on self.  xrd: None, or a
        dict(lam=..., range=(min, max), step=0.0, lp=True) for the powder pattern.
        cufft: cuFFT R2C instead of the pruned 512-point passes on 512^3 grids.
        autotune: fine grid and kernel width chosen by timing (SQN_FLAG_AUTOTUNE)."""
        L = self._L
        self.type_id = np.ascontiguousarray(type_id, dtype=np.int32)
        self.natoms = int(self.type_id.size)
        self.ntypes = int(ntypes if ntypes is not None else max(int(self.type_id.max()), 1))
        self.nq = int(nq)
        self.partials = bool(partials)
        self.want_grid = bool(want_grid)
        d = SqnDesc()
        L.sqn_default_desc(ctypes.byref(d))
        d.device = int(device)
        cell = np.ascontiguousarray(np.asarray(cell, dtype=np.float64).reshape(9))
        for k in range(9):
            d.cell[k] = float(cell[k])
        for k in range(3):
            d.origin[k] = float(origin[k])
        d.natoms = self.natoms
        d.type_id = self.type_id.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        d.ntypes = self.ntypes
        d.weight = int(weight)
        self._amp = None if amp_const is None else np.ascontiguousarray(amp_const, dtype=np.float64)
        self._xc = None if xray_coef is None else np.ascontiguousarray(xray_coef, dtype=np.float64)
        if self._amp is not None:
            d.amp_const = self._amp.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if self._xc is not None:
            d.xray_coef = self._xc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.qmin, d.qmax, d.nq = float(qmin), float(qmax), self.nq
        d.norm = int(norm)
        d.partials = int(bool(partials))
        d.want_grid = int(bool(want_grid))
        d.precision = int(precision)
        d.flags = ((FLAG_TIMING if timing else 0) | (FLAG_GRAD if grad else 0)
                   | (FLAG_CUFFT if cufft else 0)
                   | (FLAG_AUTOTUNE if autotune else 0))
        d.eps = float(eps)
        d.upsampfac = float(upsampfac)
        d.kernel_width = int(kernel_width)
        d.max_grid_modes = int(max_grid_modes)
        d.stream = stream
        if xrd:
            d.xrd_lambda = float(xrd["lam"])
            lo, hi = xrd.get("range", (1.0, 179.0))
            d.xrd_2theta_min, d.xrd_2theta_max = float(lo), float(hi)
            d.xrd_step = float(xrd.get("step", 0.0) or 0.0)
            d.xrd_lp = 1 if xrd.get("lp", True) else 0
        return d

    def _attach(self, h, owned):
        self._h = h
        self._owned = owned
        info = SqnInfo()
        check(self._L.sqn_plan_info_get(h, ctypes.byref(info)), "sqn_plan_info_get")
        self.info = info
        self.modes = tuple(info.modes)
        self.nmodes = int(info.nmodes)
        self.gridpoints = int(info.gridpoints)

    @property
    def handle(self):
        return self._h

    def accumulate(self, pos, where=HOST):
        """pos: (nframes, natoms, 3) or (natoms, 3) float64 host array, or a device
        pointer (int) with where=DEVICE and an explicit frame count in pos=(ptr, n)."""
        if where == DEVICE:
            ptr, n = pos
            check(self._L.sqn_accumulate_frames(self._h, ctypes.c_void_p(ptr), int(n), DEVICE),
                  "sqn_accumulate_frames")
            return
        a = np.ascontiguousarray(pos, dtype=np.float64)
        n = 1 if a.ndim == 2 else a.shape[0]
        if a.size != n * self.natoms * 3:
            raise ValueError("positions must hold %d atoms per frame" % self.natoms)
        check(self._L.sqn_accumulate_frames(self._h, _ptr(a), n, HOST), "sqn_accumulate_frames")

    def sync(self):
        check(self._L.sqn_sync(self._h), "sqn_sync")

    def accumulators(self, grid=False):
        nq, T = self.nq, self.ntypes
        num, den = np.zeros(nq), np.zeros(nq)
        cnt = np.zeros(nq, dtype=np.int64)
        pn = np.zeros(T * T * nq)
        gnum = np.zeros(self.gridpoints) if grid else None
        gden = np.zeros(self.gridpoints) if grid else None
        nf = ctypes.c_int64()
        check(self._L.sqn_get_accumulators(self._h, _ptr(num), _ptr(den), _ptr(cnt), _ptr(pn),
                                           _ptr(gnum), _ptr(gden),
                                           ctypes.cast(ctypes.byref(nf), ctypes.c_void_p)),
              "sqn_get_accumulators")
        return dict(num=num, den=den, shell_count=cnt,
                    partial_num=pn.reshape(nq, T, T).transpose(2, 1, 0), gnum=gnum, gden=gden,
                    nframes=int(nf.value))

    def finalize(self, faber_ziman=False, grid=False):
        nq, T = self.nq, self.ntypes
        s, sp = np.zeros(nq), np.zeros(T * T * nq)
        sg = np.zeros(self.nmodes) if grid else None
        nf = ctypes.c_int64()
        check(self._L.sqn_finalize(self._h, int(bool(faber_ziman)), _ptr(s), _ptr(sp), _ptr(sg),
                                   ctypes.cast(ctypes.byref(nf), ctypes.c_void_p)),
              "sqn_finalize")
        return s, sp.reshape(nq, T, T).transpose(2, 1, 0), sg, int(nf.value)

    def sq_grad(self, pos, dLdS=None):
        """One frame: S(q) of that frame and, with dLdS, dL/dr for L = sum dLdS * S.

        pos: (natoms, 3) float64 numpy array (host) or a torch CUDA tensor
        (device; the gradient is then a torch CUDA tensor too)."""
        nq = self.nq
        S = np.zeros(nq)
        g = None if dLdS is None else np.ascontiguousarray(dLdS, dtype=np.float64)
        if hasattr(pos, "data_ptr"):  # torch tensor on the device
            import torch
            pos = pos.contiguous()
            grad = torch.empty_like(pos) if g is not None else None
            torch.cuda.current_stream().synchronize()
            check(self._L.sqn_sq_grad(self._h, ctypes.c_void_p(pos.data_ptr()), DEVICE, _ptr(g),
                                      _ptr(S), ctypes.c_void_p(grad.data_ptr()) if grad is not None
                                      else None), "sqn_sq_grad")
            return S, grad
        a = np.ascontiguousarray(pos, dtype=np.float64)
        grad = np.zeros((self.natoms, 3)) if g is not None else None
        check(self._L.sqn_sq_grad(self._h, _ptr(a), HOST, _ptr(g), _ptr(S), _ptr(grad)),
              "sqn_sq_grad")
        return S, grad

    def density_modes(self, pos, hkl):
        """rho_a(q_h) = sum_{j of type a} exp(i q_h . r_j) of one frame at the lattice
        points hkl (nmodes, 3) int; returns complex128 (nspecies, nmodes), species in
        ascending type id.  pos: (natoms, 3) float64 host array or torch CUDA tensor."""
        h = np.ascontiguousarray(hkl, dtype=np.int32).reshape(-1, 3)
        nsp = int(self.info.nspecies)
        rho = np.zeros((nsp, h.shape[0], 2))
        if hasattr(pos, "data_ptr"):
            import torch
            pos = pos.contiguous()
            torch.cuda.current_stream().synchronize()
            check(self._L.sqn_density_modes(self._h, ctypes.c_void_p(pos.data_ptr()), DEVICE,
                                            _ptr(h), h.shape[0], _ptr(rho)), "sqn_density_modes")
        else:
            a = np.ascontiguousarray(pos, dtype=np.float64)
            check(self._L.sqn_density_modes(self._h, _ptr(a), HOST, _ptr(h), h.shape[0],
                                            _ptr(rho)), "sqn_density_modes")
        return rho[..., 0] + 1j * rho[..., 1]

    def xrd(self):
        """Powder pattern per atom and frame: (two_theta, I, I_partial (T, T, bins),
        count, nframes); the pair array is indexed [a-1, b-1, bin] (a <= b) like partial_num."""
        nb, T = int(self.info.xrd_bins), self.ntypes
        tth, I = np.zeros(nb), np.zeros(nb)
        Ip, cnt = np.zeros(T * T * nb), np.zeros(nb, dtype=np.int64)
        nf = ctypes.c_int64()
        check(self._L.sqn_get_xrd(self._h, _ptr(tth), _ptr(I), _ptr(Ip), _ptr(cnt),
                                  ctypes.cast(ctypes.byref(nf), ctypes.c_void_p)), "sqn_get_xrd")
        return tth, I, Ip.reshape(nb, T, T).transpose(2, 1, 0), cnt, int(nf.value)

    def accumulate_dump(self, reader, max_frames=-1, ref_bounds=None):
        """Frames of a DumpReader into the plan (parse of frame f + 1 overlapped
        with the upload and transform of frame f); returns the frame count."""
        done = ctypes.c_int64()
        rb = None if ref_bounds is None else np.ascontiguousarray(ref_bounds, dtype=np.float64)
        check(self._L.sqn_accumulate_dump(self._h, reader.handle, int(max_frames), _ptr(rb),
                                          ctypes.byref(done)), "sqn_accumulate_dump")
        return int(done.value)

    def accumulator_view(self):
        """(device pointer, number of doubles, frames so far) of the plan's FP64 sums."""
        ptr, count, nf = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int64()
        check(self._L.sqn_accumulator_view(self._h, ctypes.byref(ptr), ctypes.byref(count),
                                           ctypes.byref(nf)), "sqn_accumulator_view")
        return int(ptr.value or 0), int(count.value), int(nf.value)

    def set_frame_count(self, nframes):
        check(self._L.sqn_set_frame_count(self._h, int(nframes)), "sqn_set_frame_count")

    def peek_num_async(self, host_buf_ptr):
        check(self._L.sqn_peek_num_async(self._h, ctypes.c_void_p(host_buf_ptr)), "sqn_peek")

    def join(self):
        """The plan's stream waits for its FFT stream (events recorded on the plan's
        stream afterwards cover every queued frame)."""
        check(self._L.sqn_join(self._h), "sqn_join")

    def reset(self):
        check(self._L.sqn_reset(self._h), "sqn_reset")

    def stage_times(self):
        out = (ctypes.c_double * 5)()
        check(self._L.sqn_stage_times(self._h, out, 5), "sqn_stage_times")
        return dict(sort_ms=out[0], spread_ms=out[1], fft_ms=out[2], bin_ms=out[3],
                    frames=int(out[4]))

    def launch_count(self):
        return int(self._L.sqn_launch_count(self._h))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            if getattr(self, "_owned", True):
                self._L.sqn_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """sqn_batch: many independent systems, one CUDA graph launch per frame of all.

    systems: list of dicts of Plan keyword arguments (cell, origin, type_id, ...).
    plans[k] is a non-owning Plan view of system k for results."""

    def __init__(self, systems, stream=None):
        L = load()
        self._L = L
        n = len(systems)
        descs = (SqnDesc * max(n, 1))()
        views = []
        for k, kw in enumerate(systems):
            v = Plan.__new__(Plan)
            v._L = L
            descs[k] = v._describe(**kw)
            views.append(v)
        h = ctypes.c_void_p()
        self.status = check(L.sqn_batch_create(descs, n, stream, ctypes.byref(h)),
                            "sqn_batch_create")
        self._h = h
        for k, v in enumerate(views):
            ph = ctypes.c_void_p()
            check(L.sqn_batch_plan(h, k, ctypes.byref(ph)), "sqn_batch_plan")
            v._attach(ph, owned=False)
        self.plans = views

    def accumulate(self, pos, where=HOST, nframes=None):
        """pos[k]: (nframes, natoms_k, 3) float64 numpy arrays (host), or device
        pointers (ints) with where=DEVICE and nframes given."""
        n = len(self.plans)
        ptrs = (ctypes.c_void_p * n)()
        if where == DEVICE:
            for k in range(n):
                ptrs[k] = int(pos[k])
            nf = int(nframes)
        else:
            self._hold = [np.ascontiguousarray(a, dtype=np.float64) for a in pos]
            nf = 1 if self._hold[0].ndim == 2 else self._hold[0].shape[0]
            for k, (a, v) in enumerate(zip(self._hold, self.plans)):
                if a.size != nf * v.natoms * 3:
                    raise ValueError("system %d: positions must hold %d frames of %d atoms"
                                     % (k, nf, v.natoms))
                ptrs[k] = a.ctypes.data
        check(self._L.sqn_batch_accumulate(self._h, ptrs, nf, where), "sqn_batch_accumulate")

    def sync(self):
        check(self._L.sqn_batch_sync(self._h), "sqn_batch_sync")

    def graph_launches(self):
        return int(self._L.sqn_batch_graph_launches(self._h))

    def launch_count(self):
        """Kernels of this library launched by the graph replays so far."""
        return int(self._L.sqn_batch_launch_count(self._h))

    @property
    def multi(self):
        """True when every frame stage runs for all systems in one launch."""
        return bool(self._L.sqn_batch_multi(self._h))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            for v in self.plans:
                v._h = ctypes.c_void_p()
            self._L.sqn_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Type1Plan:
    """sqn_type1_*: cuFINUFFT-shaped type-1 3D NUFFT on torch CUDA tensors.

    fk[t, k3, k2, k1] = sum_j c[t, j] exp(iflag i (k1 x_j + k2 y_j + k3 z_j)); the
    plan runs on torch's current CUDA stream unless a stream handle is given."""

    def __init__(self, n_modes, iflag=1, ntransf=1, eps=1e-6, precision=PREC_DOUBLE,
                 modeord=0, upsampfac=0.0, device=0, stream=None, nufft_type=1, dim=3):
        import torch
        L = load()
        self._L = L
        self.fp64 = precision == PREC_DOUBLE
        self.n_modes = tuple(int(n) for n in n_modes)
        self.ntransf = int(ntransf)
        o = Type1Opts()
        L.sqn_type1_default_opts(ctypes.byref(o))
        o.gpu_device_id = int(device)
        o.modeord = int(modeord)
        o.upsampfac = float(upsampfac)
        o.gpu_stream = (stream if stream is not None
                        else torch.cuda.current_stream(device).cuda_stream)
        nm = (ctypes.c_int64 * 3)(*self.n_modes)
        h = ctypes.c_void_p()
        make = L.sqn_type1_makeplan if self.fp64 else L.sqn_type1f_makeplan
        self.status = check(make(int(nufft_type), int(dim), nm, int(iflag), self.ntransf,
                                 float(eps), ctypes.byref(h), ctypes.byref(o)),
                            "sqn_type1_makeplan")
        self._h = h
        self._pts = None

    def setpts(self, x, y, z):
        import torch
        dt = torch.float64 if self.fp64 else torch.float32
        pts = [t.to(dtype=dt).contiguous() for t in (x, y, z)]
        self._pts = pts  # kept alive until the next setpts
        f = self._L.sqn_type1_setpts if self.fp64 else self._L.sqn_type1f_setpts
        check(f(self._h, int(pts[0].numel()), *(ctypes.c_void_p(t.data_ptr()) for t in pts)),
              "sqn_type1_setpts")

    def execute(self, c):
        import torch
        ct = torch.complex128 if self.fp64 else torch.complex64
        c = c.to(dtype=ct).contiguous()
        N1, N2, N3 = self.n_modes
        fk = torch.empty((self.ntransf, N3, N2, N1), dtype=ct, device=c.device)
        f = self._L.sqn_type1_execute if self.fp64 else self._L.sqn_type1f_execute
        check(f(self._h, ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(fk.data_ptr())),
              "sqn_type1_execute")
        return fk

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.sqn_type1_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DumpReader:
    """sqn_dump_*: multithreaded LAMMPS text dump reader (memory-mapped)."""

    def __init__(self, path, nthreads=0):
        L = load()
        self._L = L
        h = ctypes.c_void_p()
        check(L.sqn_dump_open(os.fsencode(path), int(nthreads), ctypes.byref(h)), "sqn_dump_open")
        self._h = h
        self._cap = 0

    @property
    def handle(self):
        return self._h

    def next(self, capacity=None):
        """The next frame as (timestep, natoms, bounds (3, 3), pos (N, 3), type_id (N,),
        ids (N,)), or None at the end of the file."""
        cap = int(capacity or max(self._cap, 1024))
        while True:
            pos = np.empty((cap, 3))
            types = np.empty(cap, dtype=np.int32)
            ids = np.empty(cap, dtype=np.int64)
            bounds = np.zeros(9)
            n, ts = ctypes.c_int64(), ctypes.c_int64()
            rc = self._L.sqn_dump_next(self._h, cap, ctypes.byref(n), ctypes.byref(ts), _ptr(bounds),
                                       _ptr(pos), _ptr(types), _ptr(ids))
            if rc == ERR_INVALID_ARGUMENT and n.value > cap:
                cap = int(n.value)
                continue
            if rc == ERR_DUMP:
                raise SqnError(rc, "sqn_dump_next: reader error %d"
                               % self._L.sqn_dump_last_error(self._h))
            check(rc, "sqn_dump_next")
            break
        natoms = int(n.value)
        if natoms == 0:
            return None
        self._cap = max(self._cap, natoms)
        return (int(ts.value), natoms, bounds.reshape(3, 3), pos[:natoms], types[:natoms],
                ids[:natoms])

    def last_error(self):
        return int(self._L.sqn_dump_last_error(self._h))

    def rewind(self):
        check(self._L.sqn_dump_rewind(self._h), "sqn_dump_rewind")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.sqn_dump_close(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
