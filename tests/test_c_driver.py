"""include/sqnufft.h from plain C: tests/c/abi_driver.c (the call sequence of
sqcalc's GPU method: default descriptor, plan, host frames, finalize, destroy)
compiles as strict C99 against the header and links against libsqnufft.so; on
a GPU it runs and prints the S(q) and S(1-2) of the same plan that Python
builds through ctypes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "abi_driver.c")


def build_driver(tmp_path):
    from sqcalc_b200 import build
    lib = build.build()
    cc = shutil.which("gcc") or "cc"
    exe = str(tmp_path / "abi_driver")
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I" + os.path.join(ROOT, "include"), "-o", exe, SRC,
                    "-L" + os.path.dirname(lib), "-lsqnufft",
                    "-Wl,-rpath," + os.path.dirname(lib)], check=True)
    return exe


def test_header_compiles_as_c99_and_links(tmp_path):
    exe = build_driver(tmp_path)
    assert os.access(exe, os.X_OK)


def lcg_system(n=1500, nframes=2, box=16.0):
    """The driver's positions: the same 64-bit LCG, top 53 bits / 2^53."""
    state = 88172645463325252
    out = np.empty(nframes * n * 3)
    for i in range(out.size):
        state = (state * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        out[i] = box * ((state >> 11) * (1.0 / 9007199254740992.0))
    types = (1 + (np.arange(n) & 1)).astype(np.int32)
    return types, out.reshape(nframes, n, 3)


@pytest.mark.gpu
def test_c_driver_matches_python_plan(tmp_path):
    from sqcalc_b200 import _lib
    exe = build_driver(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    vals = np.array([float(x) for x in r.stdout.split()])
    S_c, S12_c = vals[:50], vals[50:100]
    types, frames = lcg_system()
    with _lib.Plan(np.eye(3).reshape(9) * 16.0, np.zeros(3), types, qmin=0.0, qmax=5.0, nq=50,
                   norm=_lib.NORM_MEAN, partials=True, precision=_lib.PREC_DOUBLE,
                   eps=1e-10) as p:
        p.accumulate(frames)
        S, Sp, _, n = p.finalize()
    assert n == 2
    np.testing.assert_allclose(S_c, S, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(S12_c, Sp[0, 1], rtol=1e-12, atol=1e-12)
