"""Parity with the reference's own GPU code: the cuFINUFFT that thatstar/sqcalc
vendors (external/finufft/src/cuda), built for sm_100a by oracle/cufinufft.mk
into oracle/_ref/libcufinufft.so (skipped when that library was not built).

* This library's cuFINUFFT-shaped type-1 entry points against the reference's
  cufinufft[f]_makeplan / setpts / execute on the same points and strengths
  (external/finufft/include/cufinufft.h:16-38), relative l2 within a few eps.
* S(q) and the partials of a plan against the reference's GPU frame flow
  restated on the host: cuFINUFFT modes of every species with sqcalc's options
  (src/sqc_gpu.f90:185-204: modeord 0, iflag +1, one transform per species,
  coordinates 2 pi s - pi, :230-236), downloaded, then the pair sums and the
  shell binning of src/sqc_structure_factor.f90:481-521 and :595-643.
"""
import numpy as np
import pytest

from oracle import cufinufft_ref as REF
from oracle import oracle as O
from sqcalc_b200 import _lib

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF.available(), reason="oracle/_ref/libcufinufft.so not built")]


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("fp64,eps", [(True, 1e-9), (False, 1e-5)])
def test_type1_matches_reference_cufinufft(fp64, eps):
    """Both transforms against the direct type-1 sum (oracle.dirft3d1, FINUFFT's
    own check, external/finufft/test/utils/dirft3d.hpp:13-20): ours within 20 eps
    (measured 1.0e-4 relative l2 in FP32 at eps 1e-5 on these 33 x 40 x 28 modes,
    upsampling ~1.2; the reference, at upsampling 2, 1.2e-5; FP64 within 10 eps),
    and their difference no larger than the sum of the two errors."""
    import torch
    rng = np.random.default_rng(12)
    M, nm, ntr = 4000, (33, 40, 28), 2
    dt = torch.float64 if fp64 else torch.float32
    ct = torch.complex128 if fp64 else torch.complex64
    xh = [(rng.random(M) * 2 - 1) * np.pi for _ in range(3)]
    ch = rng.standard_normal((ntr, M)) + 1j * rng.standard_normal((ntr, M))
    xyz = [torch.from_numpy(x).to("cuda", dt) for x in xh]
    c = torch.from_numpy(ch).to("cuda", ct).contiguous()
    fk_ref = torch.zeros((ntr, nm[2], nm[1], nm[0]), dtype=ct, device="cuda")
    with REF.Type1Plan(nm, ntr, eps, fp64) as rp:
        rp.setpts(M, xyz[0].data_ptr(), xyz[1].data_ptr(), xyz[2].data_ptr())
        rp.execute(c.data_ptr(), fk_ref.data_ptr())
    torch.cuda.synchronize()
    prec = _lib.PREC_DOUBLE if fp64 else _lib.PREC_SINGLE
    with _lib.Type1Plan(nm, iflag=1, ntransf=ntr, eps=eps, precision=prec) as p:
        p.setpts(*xyz)
        fk = p.execute(c).cpu().numpy()
    ref = fk_ref.cpu().numpy()
    assert fk.shape == ref.shape
    exact = O.dirft3d1(xh[0], xh[1], xh[2], ch, nm, iflag=1)
    e_ours, e_ref = rel_l2(fk, exact), rel_l2(ref, exact)
    assert e_ours < (10 if fp64 else 20) * eps, (e_ours, e_ref)
    assert rel_l2(fk, ref) <= 1.01 * (e_ours + e_ref) + 1e-15, (e_ours, e_ref)


def reference_gpu_frame_sq(frames, tid, box, qmax, nq, eps):
    """S(q) and partials through the reference's GPU flow on one device: per
    frame cuFINUFFT (FP64) of every species' one-hot strengths, the full mode
    cube downloaded, pair products and shell sums on the host."""
    import torch
    grid = O.configure_grid(np.eye(3) * box, 0.0, qmax, nq)
    m = [int(v) for v in grid.modes]
    species = sorted(set(int(t) for t in tid))
    T = len(species)
    n = len(tid)
    onehot = np.zeros((T, n), dtype=np.complex128)
    for a, t in enumerate(species):
        onehot[a, tid == t] = 1.0
    c = torch.from_numpy(onehot).cuda()
    # kept modes in the CMCL cube [T][m3][m2][m1], h = p - (m + 1)/2 (1-based p)
    h = grid.hkl.astype(np.int64)
    idx = ((h[:, 2] + (m[2] - 1) // 2) * m[1] + (h[:, 1] + (m[1] - 1) // 2)) * m[0] + \
        (h[:, 0] + (m[0] - 1) // 2)
    sh = grid.shell.astype(np.int64) - 1
    num = np.zeros(nq)
    pn = np.zeros((T, T, nq))
    with REF.Type1Plan(m, T, eps, True) as rp:
        for pos in frames:
            frac = np.zeros(3 * n)
            O.lib().sqo_wrap(n, np.ascontiguousarray(pos, dtype=np.float64).reshape(-1),
                             np.ascontiguousarray((np.eye(3) * box).reshape(9)), np.zeros(3), frac)
            x = [torch.from_numpy(2 * np.pi * frac.reshape(n, 3)[:, d] - np.pi).cuda()
                 for d in range(3)]
            fk = torch.zeros((T, m[2], m[1], m[0]), dtype=torch.complex128, device="cuda")
            rp.setpts(n, x[0].data_ptr(), x[1].data_ptr(), x[2].data_ptr())
            rp.execute(c.data_ptr(), fk.data_ptr())
            rho = fk.cpu().numpy().reshape(T, -1)[:, idx]
            tot = rho.sum(axis=0)
            num += np.bincount(sh, weights=np.abs(tot) ** 2, minlength=nq)
            for a in range(T):
                for b in range(a, T):
                    v = (rho[a] * np.conj(rho[b])).real
                    pn[a, b] += np.bincount(sh, weights=v, minlength=nq)
    counts = O.type_counts_of(tid, max(species))
    den = np.bincount(sh, minlength=nq) * (float(n))  # norm mean, unit weights: (sum n_t)^2 / N
    cnt = np.bincount(sh, minlength=nq)
    S = np.where(den > 0, num / (len(frames) * np.where(den > 0, den, 1)), 0.0)
    Sp = pn / (len(frames) * n * np.maximum(cnt, 1))
    return S, Sp, counts


def test_plan_matches_reference_gpu_flow():
    rng = np.random.default_rng(21)
    box, n, qmax, nq = 20.0, 3000, 8.0, 200
    tid = rng.integers(1, 3, size=n).astype(np.int32)
    frames = [rng.random((n, 3)) * box for _ in range(2)]
    S_ref, Sp_ref, _ = reference_gpu_frame_sq(frames, tid, box, qmax, nq, 1e-10)
    with _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), tid, qmin=0.0, qmax=qmax, nq=nq,
                   norm=_lib.NORM_MEAN, partials=True, precision=_lib.PREC_DOUBLE,
                   eps=1e-10) as p:
        for f in frames:
            p.accumulate(f)
        S, Sp, _, _ = p.finalize()
    assert np.max(np.abs(S - S_ref)) / max(1.0, np.max(np.abs(S_ref))) < 1e-8
    for a in (1, 2):
        for b in range(a, 3):
            assert np.max(np.abs(Sp[a - 1, b - 1] - Sp_ref[a - 1, b - 1])) < 1e-8
