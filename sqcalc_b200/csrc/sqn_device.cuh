// Device helpers shared by the per-frame kernels (sqn_kernels.cu) and the
// adjoint kernels (sqn_adjoint.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sqn_internal.h"

namespace sqn {
namespace dev {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// Atom -> fine grid
// ---------------------------------------------------------------------------

struct AtomCell {
  int ix0[3];     // first support cell, wrapped into [0, nf)
  double off[3];  // (X - ix0) - (w/2 - 1/2), in (-1/2, 1/2]
};

// s = A^-1 (r - origin), s -= floor(s)  (cell_fractional, src/sqc_cell.f90:143-152,
// and the wrap of src/sqc_gpu.f90:230-236); X = nf * s is the fine-grid coordinate.
__device__ __forceinline__ void atom_cell(const double *__restrict__ pos, int64_t i,
                                          const FrameGeom &g, AtomCell &c) {
  const double d0 = __dsub_rn(pos[3 * i + 0], g.origin[0]);
  const double d1 = __dsub_rn(pos[3 * i + 1], g.origin[1]);
  const double d2 = __dsub_rn(pos[3 * i + 2], g.origin[2]);
  const double halfw = 0.5 * (double)g.w;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    double s = __dadd_rn(__dadd_rn(__dmul_rn(g.inv[r], d0), __dmul_rn(g.inv[3 + r], d1)),
                         __dmul_rn(g.inv[6 + r], d2));
    s = __dsub_rn(s, floor(s));
    // A non-finite coordinate must not index outside the grid: park it at 0.
    if (!(s >= 0.0 && s <= 1.0)) s = 0.0;
    const double X = __dmul_rn((double)g.nf[r], s);
    const double start = ceil(__dsub_rn(X, halfw));
    c.off[r] = __dsub_rn(__dsub_rn(X, start), halfw - 0.5);
    int ix0 = (int)start;
    if (ix0 < 0) ix0 += g.nf[r];
    if (ix0 >= g.nf[r]) ix0 -= g.nf[r];
    c.ix0[r] = ix0;
  }
}

// Home tile of the support start (one bin per tile holds every transform) and
// the start cell relative to the tile origin.
__device__ __forceinline__ uint32_t home_key(const AtomCell &c, const FrameGeom &g, int &l0,
                                             int &l1, int &l2) {
  const int t0 = c.ix0[0] / g.tile[0], t1 = c.ix0[1] / g.tile[1], t2 = c.ix0[2] / g.tile[2];
  l0 = c.ix0[0] - t0 * g.tile[0];
  l1 = c.ix0[1] - t1 * g.tile[1];
  l2 = c.ix0[2] - t2 * g.tile[2];
  return (uint32_t)((t2 * g.ntile[1] + t1) * g.ntile[0] + t0);
}

// ES kernel: phi(t) = exp(beta (sqrt(1 - (2t/w)^2) - 1)) on |t| < w/2, else 0
// (external/finufft/include/cufinufft/spreadinterp.h:84-98).
// FP32: the hardware approximations of sqrt and 2^x, exp(u) = 2^(u log2 e)
// (relative errors near 2^-22 on the kernel values, below the FP32 plans'
// smallest eps, FLT_EPSILON; the error of a value far out in the tail is
// relative to that small value).  Both in their flush-to-zero forms: the
// arguments are 1 - z2 in (0, 1] and beta (r - 1) log2 e in [-beta log2 e, 0]
// (beta < 40), and the results sqrt in (0, 1] and 2^x >= 2^-58, all normal.
__device__ __forceinline__ float es_phi(float t, float c2, float beta) {
  constexpr float kLog2e = 1.44269504088896340736f;
  const float z2 = c2 * t * t;
  float r, e;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(fmaxf(1.0f - z2, 0.0f)));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(beta * (r - 1.0f) * kLog2e));
  return z2 < 1.0f ? e : 0.0f;
}
__device__ __forceinline__ double es_phi(double t, double c2, double beta) {
  const double z2 = c2 * t * t;
  return z2 < 1.0 ? exp(beta * (sqrt(1.0 - z2) - 1.0)) : 0.0;
}

// ---------------------------------------------------------------------------
// Modes
// ---------------------------------------------------------------------------

// |q| of mode h in the reference's operation order, without contraction
// (src/sqc_structure_factor.f90:366-368), so that shells match bit for bit.
__device__ __forceinline__ double qlen_exact(const BinGeom &b, int h1, int h2, int h3) {
  double q[3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
    q[r] = __dadd_rn(__dadd_rn(__dmul_rn(b.recip[r], (double)h1), __dmul_rn(b.recip[3 + r], (double)h2)),
                     __dmul_rn(b.recip[6 + r], (double)h3));
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])),
                              __dmul_rn(q[2], q[2])));
}

// shell = int((|q| - qmin)/dq) clamped to [0, nq)   (:396-399, zero based)
__device__ __forceinline__ int shell_of(const BinGeom &b, double ql) {
  int s = (int)__ddiv_rn(__dsub_rn(ql, b.qmin), b.dq);
  return min(max(s, 0), b.nq - 1);
}

// Kept test and zero-based shell of mode h, identical to the reference's FP64
// evaluation (:366-399).  A fast estimate (q from the row constant, |q| in
// FP32) decides whenever |q| is clear of qmin, qmax and every shell edge by a
// margin well above its error; otherwise the exact FP64 path runs.  ql returns
// |q| (FP64, for the x-ray form factors).
__device__ __forceinline__ bool classify_mode(const BinGeom &b, const double *crow, int h1,
                                              int h2, int h3, int &s, double &ql) {
  if (h1 == 0 && h2 == 0 && h3 == 0) return false;
  const double q0 = fma((double)h1, b.recip[0], crow[0]);
  const double q1 = fma((double)h1, b.recip[1], crow[1]);
  const double q2 = fma((double)h1, b.recip[2], crow[2]);
  const double ql2 = fma(q0, q0, fma(q1, q1, q2 * q2));
  const float qf = sqrtf((float)ql2);
  const float tol_q = 4e-7f * qf + 1e-30f;
  const float t = (qf - b.qminf) * b.invdqf;
  const float tol_t = 4e-7f * (qf * b.invdqf + 1.0f) + 1e-6f;
  const bool near = fabsf(qf - b.qmaxf) <= tol_q || fabsf(qf - b.qminf) <= tol_q ||
                    fabsf(t - rintf(t)) <= tol_t;
  if (b.xray) ql = sqrt(ql2);
  if (!near) {
    if (qf > b.qmaxf || qf < b.qminf) return false;
    s = min(max((int)t, 0), b.nq - 1);
    return true;
  }
  ql = qlen_exact(b, h1, h2, h3);
  if (ql > b.qmax || ql < b.qmin) return false;
  s = shell_of(b, ql);
  return true;
}

// Row constant h2 b2 + h3 b3 of the fast |q| estimate.
__device__ __forceinline__ void row_const(const BinGeom &b, int h2, int h3, double *crow) {
#pragma unroll
  for (int k = 0; k < 3; ++k)
    crow[k] = fma((double)h2, b.recip[3 + k], (double)h3 * b.recip[6 + k]);
}

// IT92 form factor f(q) = sum_i a_i exp(-b_i (q/4pi)^2) + c (src/sqc_elements.f90:226-239).
__device__ __forceinline__ double xray_f(const double *__restrict__ c, double q) {
  double st = q / (4.0 * 3.14159265358979323846);
  st = st * st;
  double f = c[8];
#pragma unroll
  for (int i = 0; i < 4; ++i) f = f + c[i] * exp(-c[4 + i] * st);
  return f;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Add v to hist[s]: one atomic per warp when every active lane has the same shell.
__device__ __forceinline__ void hist_add(double *hist, int s, double v, bool keep, bool uni,
                                         int s0, int lane) {
  if (uni) {
    v = warp_sum(keep ? v : 0.0);
    if (lane == 0) atomicAdd(&hist[s0], v);
  } else if (keep) {
    atomicAdd(&hist[s], v);
  }
}

template <typename R> struct Cplx;
template <> struct Cplx<float> { using T = float2; };
template <> struct Cplx<double> { using T = double2; };

// The packed word of a point record lives in the low 32 bits of slot 0.
template <typename R> __device__ __forceinline__ R pack_rec(uint32_t w);
template <> __device__ __forceinline__ float pack_rec<float>(uint32_t w) {
  return __uint_as_float(w);
}
template <> __device__ __forceinline__ double pack_rec<double>(uint32_t w) {
  return __longlong_as_double((long long)w);
}
template <typename R> __device__ __forceinline__ uint32_t unpack_rec(R v);
template <> __device__ __forceinline__ uint32_t unpack_rec<float>(float v) {
  return __float_as_uint(v);
}
template <> __device__ __forceinline__ uint32_t unpack_rec<double>(double v) {
  return (uint32_t)__double_as_longlong(v);
}

// Whole point records (REC_SLOTS = 4 values, 16- or 32-byte aligned).
__device__ __forceinline__ void store_rec(float *r, float a, float b, float c, float d) {
  *reinterpret_cast<float4 *>(r) = make_float4(a, b, c, d);
}
__device__ __forceinline__ void store_rec(double *r, double a, double b, double c, double d) {
  reinterpret_cast<double2 *>(r)[0] = make_double2(a, b);
  reinterpret_cast<double2 *>(r)[1] = make_double2(c, d);
}
__device__ __forceinline__ void load_rec(const float *r, float (&v)[4]) {
  const float4 a = *reinterpret_cast<const float4 *>(r);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void load_rec(const double *r, double (&v)[4]) {
  const double2 a = reinterpret_cast<const double2 *>(r)[0];
  const double2 b = reinterpret_cast<const double2 *>(r)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// ES kernel value at support cell k (0 <= k < w) of an atom whose record
// offset along the axis is off.
template <typename R>
__device__ __forceinline__ R es_at(int k, R off, R halfw, R c2, R beta) {
  return es_phi(((R)k - halfw) - off, c2, beta);
}

// Two-theta bin and weight of a mode of length q (two_theta_deg, lorentz_polarization
// and the bin rule of sf_configure_xrd, src/sqc_structure_factor.f90:894-924).
__device__ __forceinline__ void xrd_bin_weight(const BinGeom &b, double q, int &xb, double &wt) {
  constexpr double kPi = 3.14159265358979323846;
  double st = q * b.xlambda / (4.0 * kPi);
  st = fmax(-1.0, fmin(1.0, st));
  const double tth = 2.0 * asin(st) * 180.0 / kPi;
  xb = (int)((tth - b.xmin) / b.xstep);
  xb = min(max(xb, 0), b.xbins - 1);
  wt = 1.0;
  if (b.xlp) {
    const double t2 = tth * (kPi / 180.0), th = 0.5 * t2;
    const double c2 = cos(t2), sth = sin(th);
    wt = (1.0 + c2 * c2) / (sth * sth * cos(th));
  }
}

// One mode per lane, called by all 32 lanes of a warp: classify the mode
// (kept test and shell, identical to the reference's FP64 evaluation),
// deconvolve the transforms' values v[t] by dec = 1 / (phihat1 phihat2
// phihat3), form the weighted total (x-ray f_a(|q|) or constant amplitudes)
// and, with partials, the pair products Re(rho_a rho_b*) in FP64, and add
// them with multiplicity 2 for h1 > 0 (the mirror mode -h) to the shell
// histograms hist[quantity * nq + shell]; with want_grid add |total|^2 to
// gnum[gidx] (each mode is visited once per frame).  The reference's
// counterpart is the host loops of src/sqc_structure_factor.f90:481-521
// and :595-643.
template <typename R, int TM, bool XR, bool XD = false>
__device__ __forceinline__ void bin_mode(const BinGeom &b, int ntr, bool inrange, int h1, int h2,
                                         int h3, const double *crow,
                                         const typename Cplx<R>::T (&v)[TM], R dec,
                                         const double *__restrict__ amp,
                                         const double *__restrict__ xcoef, double *hist,
                                         double *__restrict__ gnum, int64_t gidx, int lane,
                                         double *xhist = nullptr, int hq = -1, int hs = 1) {
  // sum p of shell s at hist[p hq + s hs] (hq < 0: hq = nq, the accumulators' layout)
  if (hq < 0) hq = b.nq;
  double ql = 0.0;
  int s = 0;
  const bool keep = inrange && classify_mode(b, crow, h1, h2, h3, s, ql);
  const unsigned act = __ballot_sync(FULL, keep);
  if (act == 0u) return;
  double re[TM], im[TM], am[TM];
  double tre = 0.0, tim = 0.0;
  const double mult = h1 > 0 ? 2.0 : 1.0;
#pragma unroll
  for (int t = 0; t < TM; ++t) {
    re[t] = 0.0;
    im[t] = 0.0;
    am[t] = 0.0;
  }
  if (keep) {
#pragma unroll
    for (int t = 0; t < TM; ++t) {
      if (t < ntr) {
        re[t] = (double)(v[t].x * dec);
        im[t] = (double)(v[t].y * dec);
        am[t] = XR ? xray_f(xcoef + 9 * t, ql) : amp[t];
        tre += am[t] * re[t];
        tim += am[t] * im[t];
      }
    }
  }
  const double I = tre * tre + tim * tim;
  if (b.want_grid && keep) gnum[gidx] += I;
  const int s0 = __shfl_sync(FULL, s, __ffs(act) - 1);
  const bool uni = __all_sync(FULL, !keep || s == s0);
  hist_add(hist, s * hs, mult * I, keep, uni, s0 * hs, lane);
  if (b.partials) {
    int p = 1;
#pragma unroll
    for (int a = 0; a < TM; ++a) {
#pragma unroll
      for (int c = a; c < TM; ++c) {
        if (c < ntr) {
          hist_add(hist + p * hq, s * hs, mult * (re[a] * re[c] + im[a] * im[c]), keep, uni,
                   s0 * hs, lane);
          ++p;
        }
      }
    }
  }
  if (XD && xhist) {
    // powder pattern: the same per-mode quantities, binned in two-theta with the
    // Lorentz-polarization weight; the pair products carry the amplitudes
    // (sf_accumulate_values :616-619, sf_accumulate_xrd_partials :538-588)
    int xb = 0;
    double wt = 0.0;
    if (keep) xrd_bin_weight(b, qlen_exact(b, h1, h2, h3), xb, wt);
    const int xb0 = __shfl_sync(FULL, xb, __ffs(act) - 1);
    const bool xuni = __all_sync(FULL, !keep || xb == xb0);
    hist_add(xhist, xb, mult * wt * I, keep, xuni, xb0, lane);
    if (b.partials) {
      int p = 1;
#pragma unroll
      for (int a = 0; a < TM; ++a) {
#pragma unroll
        for (int c = a; c < TM; ++c) {
          if (c < ntr) {
            hist_add(xhist + p * b.xbins, xb,
                     mult * wt * am[a] * am[c] * (re[a] * re[c] + im[a] * im[c]), keep, xuni,
                     xb0, lane);
            ++p;
          }
        }
      }
    }
  }
}

}  // namespace dev
}  // namespace sqn
