// Adjoint of the frame S(q): dS(q)/dr_j for q-independent weights.
//
// With T(h) = sum_j c_j exp(i q_h . r_j) and S(s) = sum_{h in s} |T(h)|^2 / den(s),
// the gradient of L = sum_s g_s S(s) (g_s = dL/dS(s)) is
//   dL/dr_j = 2 c_j Re sum_h (g_s/den_s) conj(T(h)) (i q_h) exp(i q_h . r_j)
//           = 2 c_j sum_i b_i U_i(s_j),
//   U_i(s) = sum_h i h_i (g_s/den_s) conj(T(h)) exp(2 pi i h . s),
// with q_h = sum_i h_i b_i and s_j the fractional coordinates.  Each U_i is a
// type-2 NUFFT whose coefficients are Hermitian (T comes from real strengths),
// so it is real: amplify by 1/phihat on the half spectrum, one C2R FFT, then
// interpolate with the same ES kernel.  The forward transform (conj(T) from
// the R2C FFT of the weighted spread) is recomputed rather than stored.
// There is no counterpart in the reference; the FP64 direct-sum gradient in
// the tests differentiates src/sqc_structure_factor.f90:1440-1456.
#include <cstdint>
#include <cuda_runtime.h>

#include "sqn_device.cuh"
#include "sqn_internal.h"

namespace sqn {
namespace {

using namespace dev;

// Half-space pass over the kept modes: |T|^2 into the frame's shell sums and,
// when F is given, F_i(h) = i h_i gsh[shell] conj(T(h)) / phihat(h).
template <typename R, bool SMEM>
__global__ void __launch_bounds__(256, 2)
    k_adj_coef(const int4 *__restrict__ rows, int nrows, const typename Cplx<R>::T *__restrict__ G,
               BinGeom b, const R *__restrict__ inv1, const R *__restrict__ inv2,
               const R *__restrict__ inv3, const double *__restrict__ gsh,
               double *__restrict__ num, typename Cplx<R>::T *__restrict__ F) {
  extern __shared__ double s_num[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  double *hist = SMEM ? s_num : num;
  if (SMEM) {
    for (int i = tid; i < b.nq; i += blockDim.x) s_num[i] = 0.0;
    __syncthreads();
  }
  for (int r = blockIdx.x * nwarps + warp; r < nrows; r += gridDim.x * nwarps) {
    const int4 row = rows[r];
    const int h2 = row.x, h3 = row.y, lo = row.z, hi = row.w;
    const int64_t ky = h2 >= 0 ? h2 : b.nf[1] + h2;
    const int64_t kz = h3 >= 0 ? h3 : b.nf[2] + h3;
    const int64_t rowbase = (kz * b.nf[1] + ky) * b.c1;
    const R dyz = inv2[abs(h2)] * inv3[abs(h3)];
    double crow[3];
    row_const(b, h2, h3, crow);
    for (int h1b = lo; h1b <= hi; h1b += 32) {
      const int h1 = h1b + lane;
      const bool inrow = h1 <= hi;
      typename Cplx<R>::T v;
      if (inrow) v = G[rowbase + h1];
      double ql = 0.0;
      int s = 0;
      const bool keep = inrow && classify_mode(b, crow, h1, h2, h3, s, ql);
      const unsigned act = __ballot_sync(FULL, keep);
      if (act == 0u) continue;
      double I = 0.0;
      if (keep) {
        const R dec = inv1[h1] * dyz;
        const R re = v.x * dec, im = v.y * dec;
        I = (double)re * (double)re + (double)im * (double)im;
        if (F) {
          const R c = (R)gsh[s] * dec;
          typename Cplx<R>::T f;
          f.x = -(R)h1 * c * im;
          f.y = (R)h1 * c * re;
          F[rowbase + h1] = f;
          f.x = -(R)h2 * c * im;
          f.y = (R)h2 * c * re;
          F[b.vol_cplx + rowbase + h1] = f;
          f.x = -(R)h3 * c * im;
          f.y = (R)h3 * c * re;
          F[2 * b.vol_cplx + rowbase + h1] = f;
        }
      }
      const int s0 = __shfl_sync(FULL, s, __ffs(act) - 1);
      const bool uni = __all_sync(FULL, !keep || s == s0);
      hist_add(hist, s, (h1 > 0 ? 2.0 : 1.0) * I, keep, uni, s0, lane);
    }
  }
  if (SMEM) {
    __syncthreads();
    for (int i = tid; i < b.nq; i += blockDim.x)
      if (s_num[i] != 0.0) atomicAdd(&num[i], s_num[i]);
  }
}

// One warp per atom in bin-sorted order: U_i(s_j) by ES interpolation of the
// three real grids, then dL/dr_j = 2 c_j sum_i b_i U_i.  Lanes 0..w-1 evaluate
// the kernel values of the support along each axis (the same expression as
// the spread).  The two half-warps then walk the w^2 (dy, dz) rows of the
// support, alternately, with lane x of a half on cell dx = x of the row, so a
// load instruction reads two contiguous row segments (not 32 scattered
// cells); each lane accumulates its cells' weighted values in FP64 and the
// warp sums them at the end.
template <typename R>
__global__ void __launch_bounds__(256)
    k_interp(const R *__restrict__ recs, const int32_t *__restrict__ orig,
             const double *__restrict__ pos, FrameGeom g, const R *__restrict__ U, Recip rb,
             const double *__restrict__ camp, double *__restrict__ grad) {
  const int lane = threadIdx.x & 31;
  const int half = lane >> 4, x = lane & 15;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int w = g.w;
  const R halfw = R(0.5) * (R)w - R(0.5);
  const R c2 = R(4) / ((R)w * (R)w);
  const R beta = (R)g.beta;
  const bool xin = x < w;  // w <= MAX_W = 16
  for (int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < g.natoms;
       p += nwarps) {
    const int j = orig[p];
    AtomCell c;
    atom_cell(pos, j, g, c);
    R rec[REC_SLOTS];
    load_rec(recs + p * REC_SLOTS, rec);
    const int sp = (int)(unpack_rec<R>(rec[0]) >> 24);
    const int kl = lane < w ? lane : 0;
    const R kxl = es_at(kl, rec[1], halfw, c2, beta);
    const R kyl = es_at(kl, rec[2], halfw, c2, beta);
    const R kzl = es_at(kl, rec[3], halfw, c2, beta);
    const R kx = __shfl_sync(FULL, kxl, x);  // this lane's x weight (lanes x < w)
    int ix = c.ix0[0] + x;
    if (ix >= g.nf[0]) ix -= g.nf[0];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    // rows r = half, half + 2, ...: (dy, dz) = (r mod w, r / w), advanced by two
    int dy = half, dz = 0;
    if (dy >= w) {
      dy -= w;
      ++dz;
    }
    // every lane runs the same iterations (the shuffles are warp-wide); the
    // odd row count leaves the second half one row short on its last step
    const int nrow = w * w, niter = (nrow + 1) >> 1;
    for (int i = 0; i < niter; ++i) {
      const bool rin = half + 2 * i < nrow;
      int iy = c.ix0[1] + dy;
      if (iy >= g.nf[1]) iy -= g.nf[1];
      int iz = c.ix0[2] + dz;
      if (iz >= g.nf[2]) iz -= g.nf[2];
      const R wyz = __shfl_sync(FULL, kyl, dy & 31) * __shfl_sync(FULL, kzl, dz & 31);
      if (xin && rin) {
        const int64_t o = ((int64_t)iz * g.nf[1] + iy) * g.pitch + ix;
        const double k = (double)(wyz * kx);
        a0 = fma(k, (double)U[o], a0);
        a1 = fma(k, (double)U[g.vol_real + o], a1);
        a2 = fma(k, (double)U[2 * g.vol_real + o], a2);
      }
      dy += 2;
      if (dy >= w) {
        dy -= w;
        ++dz;
      }
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    if (lane < 3) {
      const double f = 2.0 * camp[sp];
      grad[3 * (int64_t)j + lane] =
          f * (rb.b[lane] * a0 + rb.b[3 + lane] * a1 + rb.b[6 + lane] * a2);
    }
  }
}

}  // namespace

template <typename R>
cudaError_t launch_adj_coef(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                            const R *inv1, const R *inv2, const R *inv3, const double *gsh,
                            double *num, void *F, int nsm, cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const size_t hist = (size_t)b.nq * sizeof(double);
  if (hist <= 160 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_adj_coef<R, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist);
    if (e != cudaSuccess) return e;
    k_adj_coef<R, true><<<nsm * 4, 256, hist, s>>>(rows, nrows, (const C *)G, b, inv1, inv2,
                                                   inv3, gsh, num, (C *)F);
  } else {
    k_adj_coef<R, false><<<nsm * 4, 256, 0, s>>>(rows, nrows, (const C *)G, b, inv1, inv2, inv3,
                                                 gsh, num, (C *)F);
  }
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_interp(const R *recs, const int32_t *orig, const double *pos,
                          const FrameGeom &g, const R *U, const Recip &rb, const double *camp,
                          double *grad, cudaStream_t s) {
  int64_t blocks = (g.natoms + 7) / 8;
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_interp<R><<<(unsigned)blocks, 256, 0, s>>>(recs, orig, pos, g, U, rb, camp, grad);
  return cudaGetLastError();
}

template cudaError_t launch_adj_coef<float>(const int4 *, int, const void *, const BinGeom &,
                                            const float *, const float *, const float *,
                                            const double *, double *, void *, int, cudaStream_t);
template cudaError_t launch_adj_coef<double>(const int4 *, int, const void *, const BinGeom &,
                                             const double *, const double *, const double *,
                                             const double *, double *, void *, int,
                                             cudaStream_t);
template cudaError_t launch_interp<float>(const float *, const int32_t *, const double *,
                                          const FrameGeom &, const float *, const Recip &,
                                          const double *, double *, cudaStream_t);
template cudaError_t launch_interp<double>(const double *, const int32_t *, const double *,
                                           const FrameGeom &, const double *, const Recip &,
                                           const double *, double *, cudaStream_t);

}  // namespace sqn
