// Pruned three-pass FFT of the spread grids, fused with the deconvolution,
// pair products and shell binning (replaces cuFFT R2C + k_bin on the frame
// path).
//
// The type-1 NUFFT only needs the modes |h_d| <= hm_d of the fine-grid
// spectrum, and S(q) only those with qmin <= |q| <= qmax.  The three passes
// use this:
//   k_fft_x      rows along x: two real rows form one complex row, one FFT of
//                length nf0 per pair; only h1 = 0 .. hm0 of each row's half
//                spectrum is written (A1[t][z][y][h1])
//   k_fft_y      columns along y for PC consecutive h1: FFT of length nf1;
//                only h2 = -hm1 .. hm1 is written (A2[t][z][h2][h1]), and only
//                for (h1, h2) whose line along b3 comes within qmax of the
//                origin
//   k_fft_z_bin  columns along z for PC consecutive h1 at one h2, every
//                transform: FFT of length nf2, then each kept mode (h1, h2, h3)
//                is classified, deconvolved and binned exactly as k_bin does
//                (bin_mode); the spectrum is never written to HBM
// A1 lives in the complex half-spectrum buffer of the plan and A2 in the real
// grid buffer, both free at that point of the frame.
//
// Each column FFT is a mixed-radix (2, 3, 4, 5, 8) Stockham transform in
// shared memory with the forward sign exp(-2 pi i j k / n), as cuFFT's
// forward transform, and a twiddle table computed on the host in FP64.
// Columns are stored padded (one slot every 32 elements) so that the strided
// stage writes do not collide on banks.
#include <cstdint>
#include <cuda_runtime.h>

#include "sqn_device.cuh"
#include "sqn_internal.h"

namespace sqn {
namespace {

using namespace dev;

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}
template <typename C> __device__ __forceinline__ C csub(C a, C b) {
  a.x -= b.x;
  a.y -= b.y;
  return a;
}
// -i * a
template <typename C> __device__ __forceinline__ C cmi(C a) {
  C r;
  r.x = a.y;
  r.y = -a.x;
  return r;
}

// In-register forward DFTs of size R (X_k = sum_j v_j exp(-2 pi i j k / R)).
template <int RR, typename C> struct Dft;
template <typename C> struct Dft<2, C> {
  __device__ __forceinline__ static void run(C *v) {
    const C a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};
template <typename C> struct Dft<4, C> {
  __device__ __forceinline__ static void run(C *v) {
    const C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const C a2 = cadd(v[1], v[3]), a3 = cmi(csub(v[1], v[3]));
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
  }
};
template <typename C> struct Dft<8, C> {
  __device__ __forceinline__ static void run(C *v) {
    using R = decltype(v[0].x);
    C e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, C>::run(e);
    Dft<4, C>::run(o);
    const R s = (R)0.70710678118654752440;  // sqrt(1/2)
    C w1, w3;
    w1.x = (o[1].x + o[1].y) * s;  // exp(-i pi / 4) o1
    w1.y = (o[1].y - o[1].x) * s;
    const C w2 = cmi(o[2]);        // exp(-i pi / 2) o2
    w3.x = (o[3].y - o[3].x) * s;  // exp(-3 i pi / 4) o3
    w3.y = -(o[3].x + o[3].y) * s;
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], w1);
    v[5] = csub(e[1], w1);
    v[2] = cadd(e[2], w2);
    v[6] = csub(e[2], w2);
    v[3] = cadd(e[3], w3);
    v[7] = csub(e[3], w3);
  }
};
template <typename C> struct Dft<3, C> {
  __device__ __forceinline__ static void run(C *v) {
    using R = decltype(v[0].x);
    const R h = (R)0.86602540378443864676;  // sin(2 pi / 3)
    const C t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    C m = v[0];
    m.x -= (R)0.5 * t1.x;
    m.y -= (R)0.5 * t1.y;
    v[0] = cadd(v[0], t1);
    C b;
    b.x = h * t2.x;
    b.y = h * t2.y;
    v[1] = cadd(m, cmi(b));
    v[2] = csub(m, cmi(b));
  }
};
template <typename C> struct Dft<5, C> {
  __device__ __forceinline__ static void run(C *v) {
    using R = decltype(v[0].x);
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;  // cos 2pi/5, 4pi/5
    const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;   // sin 2pi/5, 4pi/5
    const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    C a1, a2, b1, b2;
    a1.x = v[0].x + c1 * t1.x + c2 * t2.x;
    a1.y = v[0].y + c1 * t1.y + c2 * t2.y;
    a2.x = v[0].x + c2 * t1.x + c1 * t2.x;
    a2.y = v[0].y + c2 * t1.y + c1 * t2.y;
    b1.x = s1 * t3.x + s2 * t4.x;
    b1.y = s1 * t3.y + s2 * t4.y;
    b2.x = s2 * t3.x - s1 * t4.x;
    b2.y = s2 * t3.y - s1 * t4.y;
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, cmi(b1));
    v[4] = csub(a1, cmi(b1));
    v[2] = cadd(a2, cmi(b2));
    v[3] = csub(a2, cmi(b2));
  }
};

// Padded position of element i of a column.
__device__ __forceinline__ int padi(int i) { return i + (i >> 5); }

__device__ __forceinline__ int fdiv(int x, const FastDiv &f) {
  return f.d == 1 ? x : (int)__umulhi((uint32_t)x, f.m);
}

// One radix-RR stage for butterfly j of column col: Stockham, Ns = product
// of the earlier radices, tw[m] = exp(-2 pi i m / n).
template <int RR, typename C>
__device__ __forceinline__ void stage(const C *src, C *dst, int ld, int col, int j, int k, int nr,
                                      int Ns, int tstep, const C *tw) {
  C v[RR];
  const C *s = src + col * ld;
#pragma unroll
  for (int r = 0; r < RR; ++r) v[r] = s[padi(j + r * nr)];
  // tw[0] = 1 exactly, so k = 0 needs no branch
#pragma unroll
  for (int r = 1; r < RR; ++r) v[r] = cmul(v[r], tw[k * r * tstep]);
  Dft<RR, C>::run(v);
  C *d = dst + col * ld;
  const int o = (j - k) * RR + k;
#pragma unroll
  for (int r = 0; r < RR; ++r) d[padi(o + r * Ns)] = v[r];
}

// All butterflies of one radix-RR stage over ncol columns.
template <int RR, typename C>
__device__ __forceinline__ void stage_all(const C *a, C *b, int ld, int ncol, const FastDiv &fnr,
                                          const FastDiv &fns, int Ns, const C *tw) {
  const int nr = (int)fnr.d;
  const int tstep = nr / Ns;  // n / (Ns RR)
  const int tasks = nr * ncol;
  for (int e = threadIdx.x; e < tasks; e += blockDim.x) {
    const int col = fdiv(e, fnr), j = e - col * nr;
    const int k = j - Ns * fdiv(j, fns);  // j mod Ns
    stage<RR>(a, b, ld, col, j, k, nr, Ns, tstep, tw);
  }
}

// Power-of-two lengths: the same stages with every size a compile-time
// constant (shifts and masks for the index arithmetic).  Radix 8 while three
// or more factors of two remain, then 4 and/or 2.
template <int LOGR, int LOGN, int LOGNS, typename C>
__device__ __forceinline__ void stage_pow2(const C *a, C *b, int ld, int ncol, const C *tw) {
  constexpr int RR = 1 << LOGR, NR = (1 << LOGN) / RR, NS = 1 << LOGNS;
  constexpr int TSTEP = NR / NS;
  const int tasks = NR * ncol;
  for (int e = threadIdx.x; e < tasks; e += blockDim.x) {
    const int col = e / NR, j = e & (NR - 1);
    stage<RR>(a, b, ld, col, j, j & (NS - 1), NR, NS, TSTEP, tw);
  }
}

template <int LOGN, int LOGNS, typename C>
__device__ C *fft_pow2(C *a, C *b, int ld, int ncol, const C *tw) {
  if constexpr (LOGNS >= LOGN) {
    return a;
  } else {
    constexpr int REM = LOGN - LOGNS;
    constexpr int LOGR = REM == 4 ? 2 : (REM >= 3 ? 3 : REM);
    stage_pow2<LOGR, LOGN, LOGNS>(a, b, ld, ncol, tw);
    __syncthreads();
    return fft_pow2<LOGN, LOGNS + LOGR>(b, a, ld, ncol, tw);
  }
}

// FFT of ncol padded columns (leading dimension ld) in shared memory; a holds
// the input, b is scratch; returns the buffer with the result.  Ends with a
// barrier.
template <typename C>
__device__ C *fft_cols(C *a, C *b, const FftAxis &ax, int ncol, int ld, const C *tw) {
  switch (ax.n) {
    case 64: return fft_pow2<6, 0>(a, b, ld, ncol, tw);
    case 128: return fft_pow2<7, 0>(a, b, ld, ncol, tw);
    case 256: return fft_pow2<8, 0>(a, b, ld, ncol, tw);
    case 512: return fft_pow2<9, 0>(a, b, ld, ncol, tw);
    case 1024: return fft_pow2<10, 0>(a, b, ld, ncol, tw);
    case 2048: return fft_pow2<11, 0>(a, b, ld, ncol, tw);
    default: break;
  }
  int Ns = 1;
  for (int st = 0; st < ax.nst; ++st) {
    const int RR = ax.radix[st];
    switch (RR) {
      case 8: stage_all<8>(a, b, ld, ncol, ax.nr[st], ax.ns[st], Ns, tw); break;
      case 4: stage_all<4>(a, b, ld, ncol, ax.nr[st], ax.ns[st], Ns, tw); break;
      case 2: stage_all<2>(a, b, ld, ncol, ax.nr[st], ax.ns[st], Ns, tw); break;
      case 3: stage_all<3>(a, b, ld, ncol, ax.nr[st], ax.ns[st], Ns, tw); break;
      default: stage_all<5>(a, b, ld, ncol, ax.nr[st], ax.ns[st], Ns, tw); break;
    }
    __syncthreads();
    C *t = a;
    a = b;
    b = t;
    Ns *= RR;
  }
  return a;
}

template <typename C> __device__ void load_twiddles(C *s_tw, const C *tw, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_tw[i] = tw[i];
}

// h3 interval [lo, hi] (indices h3 + hm2) of column (h1, h2) that can hold
// modes with |q| <= qmax: |v + h3 b3|^2 <= qmax^2 for v = h1 b1 + h2 b2, widened
// by one on each side against rounding; lo > hi when empty.
__device__ __forceinline__ int2 h3_span(const BinGeom &b, int h1, int h2) {
  double v[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = (double)h1 * b.recip[k] + (double)h2 * b.recip[3 + k];
  const double *b3 = b.recip + 6;
  const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const double vb = v[0] * b3[0] + v[1] * b3[1] + v[2] * b3[2];
  const double bb = b3[0] * b3[0] + b3[1] * b3[1] + b3[2] * b3[2];
  const double q2 = b.qmax * b.qmax * (1.0 + 1e-9) + 1e-12;
  const double disc = vb * vb - bb * (vv - q2);
  if (disc < 0.0) return make_int2(1, 0);
  const double r = sqrt(disc);
  const int hm2 = b.hm[2];
  const int lo = max(-hm2, (int)floor((-vb - r) / bb) - 1);
  const int hi = min(hm2, (int)ceil((-vb + r) / bb) + 1);
  return make_int2(lo + hm2, hi + hm2);
}

// ---------------------------------------------------------------------------
// Pass 1: rows along x
// ---------------------------------------------------------------------------
template <typename R, int PC>
__global__ void __launch_bounds__(256)
    k_fft_x(const R *__restrict__ grid, typename Cplx<R>::T *__restrict__ A1, FftAxis ax,
            int64_t npairs, int64_t pitch, int H1, const typename Cplx<R>::T *__restrict__ tw) {
  using C = typename Cplx<R>::T;
  using V2 = typename Cplx<R>::T;  // two consecutive reals of a row
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = ax.n, ld = padi(n) + 1, nh = n >> 1;
  C *s_tw = reinterpret_cast<C *>(smem);
  C *a = s_tw + n;
  C *b = a + PC * ld;
  load_twiddles(s_tw, tw, n);
  const int64_t pair0 = (int64_t)blockIdx.x * PC;
#pragma unroll
  for (int p = 0; p < PC; ++p) {
    const int64_t pr = pair0 + p;
    const bool ok = pr < npairs;
    const V2 *r0 = reinterpret_cast<const V2 *>(grid + (2 * pr) * pitch);
    const V2 *r1 = reinterpret_cast<const V2 *>(grid + (2 * pr + 1) * pitch);
    C *col = a + p * ld;
    for (int i2 = threadIdx.x; i2 < nh; i2 += blockDim.x) {
      V2 u, w;
      u.x = u.y = w.x = w.y = R(0);
      if (ok) {
        u = r0[i2];
        w = r1[i2];
      }
      C v0, v1;
      v0.x = u.x;
      v0.y = w.x;
      v1.x = u.y;
      v1.y = w.y;
      col[padi(2 * i2)] = v0;
      col[padi(2 * i2 + 1)] = v1;
    }
  }
  __syncthreads();
  const C *z = fft_cols(a, b, ax, PC, ld, s_tw);
  // X1[h] = (Z[h] + conj Z[n-h]) / 2, X2[h] = (Z[h] - conj Z[n-h]) / (2i)
#pragma unroll
  for (int p = 0; p < PC; ++p) {
    const int64_t pr = pair0 + p;
    if (pr >= npairs) break;
    const C *zc = z + p * ld;
    C *o0 = A1 + (2 * pr) * H1, *o1 = A1 + (2 * pr + 1) * H1;
    for (int h = threadIdx.x; h < H1; h += blockDim.x) {
      const C zh = zc[padi(h)];
      const C zm = zc[padi(h == 0 ? 0 : n - h)];
      C x1, x2;
      x1.x = R(0.5) * (zh.x + zm.x);
      x1.y = R(0.5) * (zh.y - zm.y);
      x2.x = R(0.5) * (zh.y + zm.y);
      x2.y = R(0.5) * (zm.x - zh.x);
      o0[h] = x1;
      o1[h] = x2;
    }
  }
}

// ---------------------------------------------------------------------------
// Pass 2: columns along y
// ---------------------------------------------------------------------------
template <typename R, int PC>
__global__ void __launch_bounds__(256)
    k_fft_y(const typename Cplx<R>::T *__restrict__ A1, typename Cplx<R>::T *__restrict__ A2,
            FftAxis ax, BinGeom bg, int H1, int M1, const int2 *__restrict__ h2span,
            const typename Cplx<R>::T *__restrict__ tw) {
  using C = typename Cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = ax.n, ld = padi(n) + 1;
  C *s_tw = reinterpret_cast<C *>(smem);
  C *a = s_tw + n;
  C *b = a + PC * ld;
  const int nblk = (H1 + PC - 1) / PC;
  const int plane = blockIdx.x / nblk;
  const int h1b = (blockIdx.x - plane * nblk) * PC;
  load_twiddles(s_tw, tw, n);
  // rows h2 outside every column's span of the block are never read
  int jlo = M1, jhi = -1;
#pragma unroll
  for (int c = 0; c < PC; ++c)
    if (h1b + c < H1) {
      const int2 sp = h2span[h1b + c];
      jlo = min(jlo, sp.x);
      jhi = max(jhi, sp.y);
    }
  const C *src = A1 + (int64_t)plane * n * H1 + h1b;
  for (int e = threadIdx.x; e < PC * n; e += blockDim.x) {
    const int y = e / PC, c = e - y * PC;
    C v;
    v.x = R(0);
    v.y = R(0);
    if (h1b + c < H1) v = src[(int64_t)y * H1 + c];
    a[c * ld + padi(y)] = v;
  }
  __syncthreads();
  const C *yv = fft_cols(a, b, ax, PC, ld, s_tw);
  const int hm1 = bg.hm[1];
  C *dst = A2 + (int64_t)plane * M1 * H1 + h1b;
  const int rows = jhi - jlo + 1;
  for (int e = threadIdx.x; e < PC * rows; e += blockDim.x) {
    const int jj = e / PC, c = e - jj * PC;
    if (h1b + c >= H1) continue;
    const int j = jlo + jj, h2 = j - hm1;
    dst[(int64_t)j * H1 + c] = yv[c * ld + padi(h2 >= 0 ? h2 : n + h2)];
  }
}

// ---------------------------------------------------------------------------
// Pass 3: columns along z, every transform, then the fused binning
// ---------------------------------------------------------------------------
template <typename R, int PC, int NT, bool SMEM, bool XR>
__global__ void __launch_bounds__(FFT_Z_THREADS, 2)
    k_fft_z_bin(const typename Cplx<R>::T *__restrict__ A2, FftAxis ax, BinGeom b, int H1,
                int M1, FastDiv M2_div, const int2 *__restrict__ h2span,
                const typename Cplx<R>::T *__restrict__ tw, const R *__restrict__ inv1,
                const R *__restrict__ inv2, const R *__restrict__ inv3,
                const double *__restrict__ amp, const double *__restrict__ xcoef,
                double *__restrict__ acc, double *__restrict__ gnum) {
  using C = typename Cplx<R>::T;
  constexpr int TM = NT > 0 ? NT : MAX_FAST_T;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int2 s_span[PC];
  const int n = ax.n, ld = padi(n) + 1;
  const int ntr = NT > 0 ? NT : b.ntr;
  const int hm2 = b.hm[2], M2 = 2 * hm2 + 1;
  const int nhist = hist_len(b);
  C *s_tw = reinterpret_cast<C *>(smem);
  C *a = s_tw + n;
  C *bb = a + PC * ld;
  C *res = bb + PC * ld;  // [ntr][PC][M2]
  double *s_hist = reinterpret_cast<double *>(res + ntr * PC * M2);
  double *hist = SMEM ? s_hist : acc;
  double *xhist = b.xrd ? hist + b.nquant * b.nq : nullptr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  load_twiddles(s_tw, tw, n);
  if (SMEM)
    for (int i = tid; i < nhist; i += blockDim.x) s_hist[i] = 0.0;
  __syncthreads();
  const int nblk = (H1 + PC - 1) / PC;
  const int items = M1 * nblk;
  const int64_t tstride = (int64_t)n * M1 * H1;  // one transform of A2
  const int64_t zstride = (int64_t)M1 * H1;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int j = it / nblk, h1b = (it - j * nblk) * PC;
    const int h2 = j - b.hm[1];
    bool need = false;  // the same test as the y pass: uniform across the CTA
#pragma unroll
    for (int c = 0; c < PC; ++c)
      if (h1b + c < H1) {
        const int2 sp = h2span[h1b + c];
        need = need || (j >= sp.x && j <= sp.y);
      }
    if (!need) continue;
    if (tid < PC) s_span[tid] = h1b + tid < H1 ? h3_span(b, h1b + tid, h2) : make_int2(1, 0);
    for (int t = 0; t < ntr; ++t) {
      const C *src = A2 + t * tstride + (int64_t)j * H1 + h1b;
      for (int e = tid; e < PC * n; e += blockDim.x) {
        const int z = e / PC, c = e - z * PC;
        C v;
        v.x = R(0);
        v.y = R(0);
        if (h1b + c < H1) v = src[(int64_t)z * zstride + c];
        a[c * ld + padi(z)] = v;
      }
      __syncthreads();
      const C *zv = fft_cols(a, bb, ax, PC, ld, s_tw);
      C *r = res + t * PC * M2;
      for (int e = tid; e < PC * M2; e += blockDim.x) {
        const int c = fdiv(e, M2_div), i = e - c * M2;
        const int h3 = i - hm2;
        r[e] = zv[c * ld + padi(h3 >= 0 ? h3 : n + h3)];
      }
      __syncthreads();
    }
    // modes (h1b + c, h2, h3) inside the column's span: lanes along h3
    const R d2 = inv2[abs(h2)];
    const int total = PC * M2;
    for (int e0 = warp * 32; e0 < total; e0 += nwarps * 32) {
      const int e = e0 + lane;
      const int c = fdiv(min(e, total - 1), M2_div), i = e - c * M2;
      const int h1 = h1b + c, h3 = i - hm2;
      const int2 sp = s_span[c];
      const bool inr = e < total && h1 < H1 && i >= sp.x && i <= sp.y;
      if (__ballot_sync(FULL, inr) == 0u) continue;
      C v[TM];
#pragma unroll
      for (int t = 0; t < TM; ++t)
        if (t < ntr && inr) v[t] = res[t * PC * M2 + e];
      double crow[3];
      row_const(b, h2, h3, crow);
      const R dec = inr ? inv1[h1] * (d2 * inv3[abs(h3)]) : R(0);
      const int64_t gidx =
          ((int64_t)(h3 + hm2) * b.m2 + (int64_t)(h2 + b.hm[1])) * (int64_t)(b.hm[0] + 1) + h1;
      bin_mode<R, TM, XR, true>(b, ntr, inr, h1, h2, h3, crow, v, dec, amp, xcoef, hist, gnum,
                                gidx, lane, xhist);
    }
    __syncthreads();  // res and s_span are rewritten by the next item
  }
  if (SMEM) {
    __syncthreads();
    for (int i = tid; i < nhist; i += blockDim.x) {
      const double v = s_hist[i];
      if (v != 0.0) atomicAdd(&acc[i], v);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
size_t col_ld(int n) { return (size_t)(n + (n >> 5) + 1); }

template <typename R> size_t pass12_smem(int n, int pc) {
  const size_t cs = 2 * sizeof(R);
  return cs * ((size_t)n + 2 * (size_t)pc * col_ld(n));
}

template <typename R> size_t pass3_smem(int n, int pc, int ntr, int M2, size_t hist_bytes) {
  const size_t cs = 2 * sizeof(R);
  return cs * ((size_t)n + 2 * (size_t)pc * col_ld(n) + (size_t)ntr * pc * M2) + hist_bytes;
}

template <typename K> cudaError_t allow_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename R, int PC, int NT, bool SMEM>
cudaError_t launch_z_xr(const FftPlan3 &f, const void *A2, const BinGeom &b, const R *i1,
                        const R *i2, const R *i3, const double *amp, const double *xc,
                        double *acc, double *gnum, cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const size_t hist = SMEM ? (size_t)hist_len(b) * sizeof(double) : 0;
  const size_t sm = pass3_smem<R>(f.ax[2].n, PC, b.ntr, 2 * b.hm[2] + 1, hist);
  cudaError_t e;
  if (b.xray) {
    e = allow_smem(k_fft_z_bin<R, PC, NT, SMEM, true>, sm);
    if (e != cudaSuccess) return e;
    k_fft_z_bin<R, PC, NT, SMEM, true><<<f.grid3, FFT_Z_THREADS, sm, s>>>(
        (const C *)A2, f.ax[2], b, f.H1, f.M1, f.M2_div, f.h2span, (const C *)f.tw[2], i1, i2,
        i3, amp, xc, acc, gnum);
  } else {
    e = allow_smem(k_fft_z_bin<R, PC, NT, SMEM, false>, sm);
    if (e != cudaSuccess) return e;
    k_fft_z_bin<R, PC, NT, SMEM, false><<<f.grid3, FFT_Z_THREADS, sm, s>>>(
        (const C *)A2, f.ax[2], b, f.H1, f.M1, f.M2_div, f.h2span, (const C *)f.tw[2], i1, i2,
        i3, amp, xc, acc, gnum);
  }
  return cudaGetLastError();
}

template <typename R, int PC, int NT>
cudaError_t launch_z_nt(const FftPlan3 &f, const void *A2, const BinGeom &b, const R *i1,
                        const R *i2, const R *i3, const double *amp, const double *xc,
                        double *acc, double *gnum, cudaStream_t s) {
  if (f.hist_smem)
    return launch_z_xr<R, PC, NT, true>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
  return launch_z_xr<R, PC, NT, false>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
}

template <typename R, int PC>
cudaError_t launch_z_pc(const FftPlan3 &f, const void *A2, const BinGeom &b, const R *i1,
                        const R *i2, const R *i3, const double *amp, const double *xc,
                        double *acc, double *gnum, cudaStream_t s) {
  switch (b.ntr) {
    case 1: return launch_z_nt<R, PC, 1>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
    case 2: return launch_z_nt<R, PC, 2>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
    case 3: return launch_z_nt<R, PC, 3>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
    case 4: return launch_z_nt<R, PC, 4>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
    default: return launch_z_nt<R, PC, 0>(f, A2, b, i1, i2, i3, amp, xc, acc, gnum, s);
  }
}

template <typename R, int PC>
cudaError_t launch_xy_pc(const FftPlan3 &f, const void *grid, void *A1, void *A2,
                         const BinGeom &b, int64_t pitch, cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const int64_t npairs = (int64_t)b.ntr * b.nf[2] * b.nf[1] / 2;
  size_t sm = pass12_smem<R>(f.ax[0].n, PC);
  cudaError_t e = allow_smem(k_fft_x<R, PC>, sm);
  if (e != cudaSuccess) return e;
  const int64_t g1 = (npairs + PC - 1) / PC;
  k_fft_x<R, PC><<<(unsigned)g1, 256, sm, s>>>((const R *)grid, (C *)A1, f.ax[0], npairs, pitch,
                                                f.H1, (const C *)f.tw[0]);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sm = pass12_smem<R>(f.ax[1].n, PC);
  e = allow_smem(k_fft_y<R, PC>, sm);
  if (e != cudaSuccess) return e;
  const int64_t g2 = (int64_t)b.ntr * b.nf[2] * ((f.H1 + PC - 1) / PC);
  k_fft_y<R, PC><<<(unsigned)g2, 256, sm, s>>>((const C *)A1, (C *)A2, f.ax[1], b, f.H1, f.M1,
                                                f.h2span, (const C *)f.tw[1]);
  return cudaGetLastError();
}

}  // namespace

int fft_columns_per_cta(bool fp64) { return fp64 ? 2 : 4; }
int fft_z_columns_per_cta(bool fp64) { return fp64 ? 2 : 4; }

size_t fft_pass_smem(const FftPlan3 &f, int pass, bool fp64, int ntr, int nhist) {
  const int pc = fft_columns_per_cta(fp64);
  if (pass < 2)
    return fp64 ? pass12_smem<double>(f.ax[pass].n, pc) : pass12_smem<float>(f.ax[pass].n, pc);
  const size_t hist = f.hist_smem ? (size_t)nhist * sizeof(double) : 0;
  return fp64 ? pass3_smem<double>(f.ax[2].n, fft_z_columns_per_cta(fp64), ntr, f.M2, hist)
              : pass3_smem<float>(f.ax[2].n, fft_z_columns_per_cta(fp64), ntr, f.M2, hist);
}

template <typename R>
cudaError_t launch_fft_xy(const FftPlan3 &f, const void *grid, void *A1, void *A2,
                          const BinGeom &b, int64_t pitch, cudaStream_t s) {
  return launch_xy_pc<R, sizeof(R) == 8 ? 2 : 4>(f, grid, A1, A2, b, pitch, s);
}

template <typename R>
cudaError_t launch_fft_z_bin(const FftPlan3 &f, const void *A2, const BinGeom &b, const R *inv1,
                             const R *inv2, const R *inv3, const double *amp,
                             const double *xcoef, double *acc, double *gnum, cudaStream_t s) {
  return launch_z_pc<R, sizeof(R) == 8 ? 2 : 4>(f, A2, b, inv1, inv2, inv3, amp, xcoef, acc,
                                                 gnum, s);
}

template cudaError_t launch_fft_xy<float>(const FftPlan3 &, const void *, void *, void *,
                                          const BinGeom &, int64_t, cudaStream_t);
template cudaError_t launch_fft_xy<double>(const FftPlan3 &, const void *, void *, void *,
                                           const BinGeom &, int64_t, cudaStream_t);
template cudaError_t launch_fft_z_bin<float>(const FftPlan3 &, const void *, const BinGeom &,
                                             const float *, const float *, const float *,
                                             const double *, const double *, double *, double *,
                                             cudaStream_t);
template cudaError_t launch_fft_z_bin<double>(const FftPlan3 &, const void *, const BinGeom &,
                                              const double *, const double *, const double *,
                                              const double *, const double *, double *, double *,
                                              cudaStream_t);

}  // namespace sqn
