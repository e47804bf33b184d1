"""The reference's own cuFINUFFT, built from thatstar/sqcalc's vendored sources
(external/finufft/src/cuda) for sm_100a by oracle/cufinufft.mk into
oracle/_ref/libcufinufft.so.  Test and baseline infrastructure only: the GPU
tests compare this library's type-1 transforms and S(q) with it, and the
benchmark times it as the reference's GPU bar; the product never loads it.

The bindings mirror sqcalc's own iso_c_binding module (src/sqc_cufinufft.f90:
183-259) and the C header external/finufft/include/cufinufft.h:16-38; the opts
struct is external/finufft/include/cufinufft_opts.h:7-41.  sqcalc's call
(src/sqc_gpu.f90:185-204): cufinufft_default_opts, modeord 0 (CMCL), type 1,
dim 3, iflag +1, ntransf = species (partials or x-ray) else 1, eps.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcufinufft.so")


class Opts(ctypes.Structure):
    """cufinufft_opts (external/finufft/include/cufinufft_opts.h:7-41)."""
    _fields_ = [
        ("upsampfac", ctypes.c_double),
        ("gpu_method", ctypes.c_int),
        ("gpu_sort", ctypes.c_int),
        ("gpu_binsizex", ctypes.c_int),
        ("gpu_binsizey", ctypes.c_int),
        ("gpu_binsizez", ctypes.c_int),
        ("gpu_obinsizex", ctypes.c_int),
        ("gpu_obinsizey", ctypes.c_int),
        ("gpu_obinsizez", ctypes.c_int),
        ("gpu_maxsubprobsize", ctypes.c_int),
        ("gpu_kerevalmeth", ctypes.c_int),
        ("gpu_spreadinterponly", ctypes.c_int),
        ("gpu_maxbatchsize", ctypes.c_int),
        ("gpu_device_id", ctypes.c_int),
        ("gpu_stream", ctypes.c_void_p),
        ("modeord", ctypes.c_int),
        ("gpu_np", ctypes.c_int),
        ("debug", ctypes.c_int),
    ]


_lib = None


def available():
    return os.path.exists(LIB_PATH)


def build(ref_root):
    """make -C oracle -f cufinufft.mk REF=<sqcalc checkout> (several minutes)."""
    jobs = str(max(1, min(8, os.cpu_count() or 1)))
    subprocess.run(["make", "-s", "-C", HERE, "-f", "cufinufft.mk", "REF=" + ref_root,
                    "-j" + jobs], check=True)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
        L.cufinufft_default_opts.argtypes = [ctypes.POINTER(Opts)]
        for pre, real in (("cufinufft", ctypes.c_double), ("cufinufftf", ctypes.c_float)):
            mk = getattr(L, pre + "_makeplan")
            mk.argtypes = [ctypes.c_int, ctypes.c_int, i64p, ctypes.c_int, ctypes.c_int, real,
                           ctypes.POINTER(vp), ctypes.POINTER(Opts)]
            mk.restype = ctypes.c_int
            sp = getattr(L, pre + "_setpts")
            sp.argtypes = [vp, ctypes.c_int64, vp, vp, vp, ctypes.c_int, vp, vp, vp]
            sp.restype = ctypes.c_int
            ex = getattr(L, pre + "_execute")
            ex.argtypes = [vp, vp, vp]
            ex.restype = ctypes.c_int
            de = getattr(L, pre + "_destroy")
            de.argtypes = [vp]
            de.restype = ctypes.c_int
        _lib = L
    return _lib


class Type1Plan:
    """A 3D type-1 cuFINUFFT plan with sqcalc's options (modeord 0, iflag +1)."""

    def __init__(self, modes, ntransf, eps, fp64, device=0, stream=None, modeord=0, iflag=1):
        L = lib()
        self.fp64 = bool(fp64)
        self._pre = "cufinufft" if fp64 else "cufinufftf"
        o = Opts()
        L.cufinufft_default_opts(ctypes.byref(o))
        o.modeord = int(modeord)
        o.gpu_device_id = int(device)
        o.gpu_stream = stream
        self.opts = o
        n = (ctypes.c_int64 * 3)(*[int(m) for m in modes])
        h = ctypes.c_void_p()
        rc = getattr(L, self._pre + "_makeplan")(1, 3, n, int(iflag), int(ntransf), eps,
                                                 ctypes.byref(h), ctypes.byref(o))
        if rc > 1:
            raise RuntimeError("cufinufft makeplan failed: %d" % rc)
        self.h = h

    def setpts(self, M, x, y, z):
        """x, y, z: device pointers (ints) to M coordinates in [-pi, pi)."""
        rc = getattr(lib(), self._pre + "_setpts")(self.h, int(M), x, y, z, 0, None, None, None)
        if rc > 1:
            raise RuntimeError("cufinufft setpts failed: %d" % rc)

    def execute(self, c, fk):
        """c: device pointer to ntransf x M complex strengths; fk: ntransf x prod(modes)."""
        rc = getattr(lib(), self._pre + "_execute")(self.h, c, fk)
        if rc > 1:
            raise RuntimeError("cufinufft execute failed: %d" % rc)

    def close(self):
        if self.h:
            getattr(lib(), self._pre + "_destroy")(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
