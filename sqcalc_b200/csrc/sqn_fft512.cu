// Pruned three-pass FFT for 512-point axes, one warp per 512-point line with
// the line held in registers (replaces cuFFT R2C on the frame path when every
// fine-grid axis is 512).
//
// A line of 512 complex values is split n = n1 + 32 n2 (n1 = lane): each lane
// runs a 16-point DFT over n2 in registers, multiplies by exp(-2 pi i n1 k2 /
// 512), the warp transposes through a 512-slot scratch line in shared memory
// (skewed so that neither the writes nor the reads collide on banks), each
// lane runs a second 16-point DFT, and a radix-2 step across lanes L and
// L ^ 16 (shuffles) finishes the 32-point DFT.  Lane L = k2 + 16 b then holds
// X[k2 + 16 a + 256 b], a = 0 .. 15.  Forward sign exp(-2 pi i j k / n), as
// cuFFT's forward transform; twiddles from an FP64 host table.
//
// Passes (only the modes |h_d| <= hm_d of the type-1 NUFFT are kept):
//   k_fft512_x     two real rows along x form one complex line; the half
//                  spectrum h1 = 0 .. H1-1 of each row is written (A1[t][z][y][h1])
//   k_fft512_cols  lines along a strided axis for 16 consecutive h1 of one
//                  plane, staged in shared memory (coalesced 128-byte rows in
//                  and out); only the band h = -hm .. hm is written, in FFT
//                  order (h >= 0 at h, h < 0 at 2 hm + 1 + h).  The y pass
//                  (A1 -> A2[t][z][h2][h1]) and the z pass
//                  (A2 -> G[t][h3][h2][h1]) are the same kernel with other strides.
// The result is the compact half spectrum that k_bin reads with nf1 = 2 hm1 + 1,
// nf2 = 2 hm2 + 1 and a row pitch of P1 >= H1.
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "sqn_device.cuh"
#include "sqn_internal.h"

namespace sqn {
namespace {

using namespace dev;

template <typename C> __device__ __forceinline__ C c_add(C a, C b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}
template <typename C> __device__ __forceinline__ C c_sub(C a, C b) {
  a.x -= b.x;
  a.y -= b.y;
  return a;
}
template <typename C> __device__ __forceinline__ C c_mul(C a, C w) {
  C r;
  r.x = a.x * w.x - a.y * w.y;
  r.y = a.x * w.y + a.y * w.x;
  return r;
}
// FP32: one packed instruction (add/sub.rn.f32x2, sm_100) per complex add.
__device__ __forceinline__ float2 c_add(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb;\n\t"
      "mov.b64 pa, {%2, %3};\n\t"
      "mov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pa, pa, pb;\n\t"
      "mov.b64 {%0, %1}, pa;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb;\n\t"
      "mov.b64 pa, {%2, %3};\n\t"
      "mov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pa, pa, pb;\n\t"
      "mov.b64 {%0, %1}, pa;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
// o + s a for s = +-1 (one rounding, as o + a or o - a)
template <typename C, typename R> __device__ __forceinline__ C c_sfma(R s, C a, C o) {
  C r;
  r.x = fma(s, a.x, o.x);
  r.y = fma(s, a.y, o.y);
  return r;
}
__device__ __forceinline__ float2 c_sfma(float s, float2 a, float2 o) {
  float2 r;
  asm("{\n\t.reg .b64 ps, pa, po;\n\t"
      "mov.b64 ps, {%2, %2};\n\t"
      "mov.b64 pa, {%3, %4};\n\t"
      "mov.b64 po, {%5, %6};\n\t"
      "fma.rn.f32x2 po, ps, pa, po;\n\t"
      "mov.b64 {%0, %1}, po;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(s), "f"(a.x), "f"(a.y), "f"(o.x), "f"(o.y));
  return r;
}
// a * exp(-i theta) for cos theta = c, sin theta = s
template <typename C, typename R> __device__ __forceinline__ C c_rot(C a, R c, R s) {
  C r;
  r.x = a.x * c + a.y * s;
  r.y = a.y * c - a.x * s;
  return r;
}

// 4-point forward DFT in place.
template <typename C> __device__ __forceinline__ void dft4(C &v0, C &v1, C &v2, C &v3) {
  const C a0 = c_add(v0, v2), a1 = c_sub(v0, v2);
  const C a2 = c_add(v1, v3), a3 = c_sub(v1, v3);
  v0 = c_add(a0, a2);
  v2 = c_sub(a0, a2);
  // v1 = a1 - i a3, v3 = a1 + i a3
  v1.x = a1.x + a3.y;
  v1.y = a1.y - a3.x;
  v3.x = a1.x - a3.y;
  v3.y = a1.y + a3.x;
}

// 16-point forward DFT in registers, natural order in and out:
// n = n1 + 4 n2, k = k2 + 4 k1, twiddle exp(-2 pi i n1 k2 / 16).
template <typename C> __device__ __forceinline__ void dft16(C (&v)[16]) {
  using R = decltype(v[0].x);
  const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;  // cos, sin pi/8
  const R r2 = (R)0.70710678118654752440;                                  // cos pi/4
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) dft4(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
  // v[n1 + 4 k2] now holds A[n1][k2]; multiply by exp(-i pi n1 k2 / 8)
  v[5] = c_rot(v[5], c1, s1);    // n1 1 k2 1: m 1
  v[9] = c_rot(v[9], r2, r2);    // n1 1 k2 2: m 2
  v[13] = c_rot(v[13], s1, c1);  // n1 1 k2 3: m 3
  v[6] = c_rot(v[6], r2, r2);    // n1 2 k2 1: m 2
  {                              // n1 2 k2 2: m 4, exp(-i pi / 2) = -i
    const R t = v[10].x;
    v[10].x = v[10].y;
    v[10].y = -t;
  }
  v[14] = c_rot(v[14], -r2, r2);   // n1 2 k2 3: m 6
  v[7] = c_rot(v[7], s1, c1);      // n1 3 k2 1: m 3
  v[11] = c_rot(v[11], -r2, r2);   // n1 3 k2 2: m 6
  v[15] = c_rot(v[15], -c1, -s1);  // n1 3 k2 3: m 9
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) dft4(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
  // v[4 k2 + k1] holds X[k2 + 4 k1]; reorder to natural order
  C o[16];
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) o[k2 + 4 * k1] = v[4 * k2 + k1];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = o[k];
}

template <typename C> __device__ __forceinline__ C shfl_xor16(C v) {
  C r;
  r.x = __shfl_xor_sync(FULL, v.x, 16);
  r.y = __shfl_xor_sync(FULL, v.y, 16);
  return r;
}

// Skewed slot of element (k2, n1) of the transpose (512 slots): the writes
// (fixed k2, lanes over n1) and the reads (fixed m2, lanes over k2 and m1 with
// n1 = m1 + 2 m2) both touch every 8-byte bank pair exactly twice (slot mod 16
// is (n1 ^ k2) mod 16, a bijection of n1 mod 16 for fixed k2 and of k2 for
// fixed n1).
__device__ __forceinline__ int tslot(int k2, int n1) { return k2 * 32 + (n1 ^ k2); }

// Twiddle table (TW_LEN entries): tw[m] = exp(-2 pi i m / 512) for m < 512,
// then tw[512 + 32 k2 + n1] = exp(-2 pi i n1 k2 / 512), the per-lane factors
// laid out so that a warp reads 32 consecutive entries (no bank conflicts).
constexpr int TW_LEN = 1024;

// Forward 512-point DFT of the line whose element lane + 32 j is v[j].  The
// scratch line has 512 slots; slot i lives at scr[i * sstride].  On return
// lane L = k2 + 16 b holds X[k2 + 16 a + 256 b] in v[a].  The caller
// synchronises the warp before reusing the scratch line.
template <typename C>
__device__ __forceinline__ void warp_fft512(C (&v)[16], C *scr, int sstride, const C *tw,
                                            int lane) {
  dft16(v);  // v[k2] = Y[n1 = lane][k2]
#pragma unroll
  for (int k2 = 1; k2 < 16; ++k2) v[k2] = c_mul(v[k2], tw[512 + 32 * k2 + lane]);
#pragma unroll
  for (int k2 = 0; k2 < 16; ++k2) scr[tslot(k2, lane) * sstride] = v[k2];
  __syncwarp();
  const int k2 = lane & 15, m1 = lane >> 4;
#pragma unroll
  for (int m2 = 0; m2 < 16; ++m2) v[m2] = scr[tslot(k2, m1 + 2 * m2) * sstride];
  __syncwarp();
  dft16(v);  // v[a] = sum_m2 Y[m1 + 2 m2][k2] exp(-2 pi i m2 a / 16)
  if (m1) {
#pragma unroll
    for (int a = 1; a < 16; ++a) v[a] = c_mul(v[a], tw[16 * a]);  // exp(-2 pi i a / 32)
  }
  // lanes m1 = 0 form v + o, lanes m1 = 1 form o - v
  using R = decltype(v[0].x);
  const R sg = m1 ? R(-1) : R(1);
#pragma unroll
  for (int a = 0; a < 16; ++a) v[a] = c_sfma(sg, v[a], shfl_xor16(v[a]));
}

// ---------------------------------------------------------------------------
// Pass 1: rows along x.  Warps take row pairs (2 pr, 2 pr + 1); rows are
// pitch reals apart, nrows in all.
// ---------------------------------------------------------------------------
template <typename R> __host__ __device__ constexpr int x_warps() {
  return sizeof(R) == 4 ? 8 : 4;
}

template <typename R>
__global__ void __launch_bounds__(32 * x_warps<R>())
    k_fft512_x(const R *__restrict__ grid, typename Cplx<R>::T *__restrict__ A1, int64_t nrows,
               int64_t pitch, int H1, int P1, const typename Cplx<R>::T *__restrict__ tw) {
  using C = typename Cplx<R>::T;
  constexpr int X_WARPS = x_warps<R>();
  __shared__ C s_tw[TW_LEN];
  __shared__ C s_line[X_WARPS][512];
  for (int i = threadIdx.x; i < TW_LEN; i += blockDim.x) s_tw[i] = tw[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  C *line = s_line[warp];
  const int64_t npairs = (nrows + 1) >> 1;
  for (int64_t pr = (int64_t)blockIdx.x * X_WARPS + warp; pr < npairs;
       pr += (int64_t)gridDim.x * X_WARPS) {
    const R *r0 = grid + (2 * pr) * pitch;
    const bool two = 2 * pr + 1 < nrows;
    C v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      v[j].x = r0[lane + 32 * j];
      v[j].y = two ? r0[pitch + lane + 32 * j] : R(0);
    }
    warp_fft512(v, line, 1, s_tw, lane);
    // natural order into the scratch line for the split of the two rows
    const int k2 = lane & 15, b = lane >> 4;
#pragma unroll
    for (int a = 0; a < 16; ++a) line[k2 + 16 * a + 256 * b] = v[a];
    __syncwarp();
    // X1[h] = (Z[h] + conj Z[512-h]) / 2, X2[h] = (Z[h] - conj Z[512-h]) / (2i)
    C *o0 = A1 + (2 * pr) * P1;
    for (int h = lane; h < H1; h += 32) {
      const C zh = line[h];
      const C zm = line[(512 - h) & 511];
      C x1, x2;
      x1.x = R(0.5) * (zh.x + zm.x);
      x1.y = R(0.5) * (zh.y - zm.y);
      x2.x = R(0.5) * (zh.y + zm.y);
      x2.y = R(0.5) * (zm.x - zh.x);
      o0[h] = x1;
      if (two) o0[P1 + h] = x2;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Column passes: 512-point lines along a strided axis, 16 consecutive columns
// (h1) of one plane per CTA step, 16 warps (one column each).
// Plane o = t * planes_per_t + p starts at t * tstride + p * pstride; row r of
// the plane is rstride elements further.
// ---------------------------------------------------------------------------
constexpr int COLS = 16;
constexpr int COL_LD = COLS + 1;  // staged row pitch (complex)

struct ColPass {
  int64_t in_t, in_p, in_r;     // input strides (complex elements)
  int64_t out_t, out_p, out_r;  // output strides
  int planes_per_t;
  int64_t nplanes;
  int ncols;  // columns per plane (H1)
  int hm;     // kept band -hm .. hm
  // optional, per plane p of a transform: columns >= col_end[p] are neither
  // transformed nor written (nothing reads them)
  const int *col_end;
  // optional, per 16-column block of a plane: the band of output rows h in
  // [lo, hi] that is read later (h < 0 at row 2 hm + 1 + h); other rows of the
  // block are not written
  const short2 *blk_rows;
};

template <typename R>
__global__ void __launch_bounds__(32 * COLS, sizeof(R) == 4 ? 2 : 1)
    k_fft512_cols(const typename Cplx<R>::T *__restrict__ in, typename Cplx<R>::T *__restrict__ out,
                  ColPass cp, const typename Cplx<R>::T *__restrict__ tw) {
  using C = typename Cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s_tw = reinterpret_cast<C *>(smem_raw);
  C *tile = s_tw + TW_LEN;  // [512][COL_LD]
  for (int i = threadIdx.x; i < TW_LEN; i += blockDim.x) s_tw[i] = tw[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int M = 2 * cp.hm + 1;
  // Steps: the full 16-column blocks of every plane, then the partial last
  // blocks (rem columns) of G = 16 / rem planes at a time, so that no step
  // leaves most of its warps idle.  32-bit step indices (the host keeps the
  // step count below 2^31): the divisions are a few instructions.
  const int nfull = cp.ncols / COLS, rem = cp.ncols - nfull * COLS;
  const int G = rem > 0 ? COLS / rem : 1;
  const unsigned nfs = (unsigned)cp.nplanes * (unsigned)nfull;
  const unsigned nsteps =
      nfs + (rem > 0 ? (unsigned)((cp.nplanes + G - 1) / G) : 0u);
  // thread -> (tile column c, rows r0 + 32 k)
  const int c = threadIdx.x & (COLS - 1), r0 = threadIdx.x >> 4;
  for (unsigned st = blockIdx.x; st < nsteps; st += gridDim.x) {
    // the plane and column of tile column cc of this step (false: no column)
    auto where = [&](int cc, unsigned &plane, int &col) {
      if (st < nfs) {
        plane = st / (unsigned)nfull;
        col = (int)(st - plane * (unsigned)nfull) * COLS + cc;
        return true;
      }
      const int sub = cc / rem;
      plane = (st - nfs) * (unsigned)G + (unsigned)sub;
      col = nfull * COLS + (cc - sub * rem);
      return sub < G && plane < (unsigned)cp.nplanes;
    };
    auto used = [&](int cc, unsigned &plane, int &col) {
      if (!where(cc, plane, col)) return false;
      return !cp.col_end || col < __ldg(cp.col_end + plane % (unsigned)cp.planes_per_t);
    };
    unsigned plane;
    int col;
    const bool mine = used(c, plane, col);
    const unsigned t = plane / (unsigned)cp.planes_per_t, p = plane - t * cp.planes_per_t;
    __syncthreads();  // the previous step's stores have read the tile
    if (mine) {
      // a thread's loads (rows r0 + 32 k) go out eight at a time
      const C *src = in + t * cp.in_t + p * cp.in_p + col + (int64_t)r0 * cp.in_r;
      const int64_t step = 32 * cp.in_r;
#pragma unroll
      for (int k0 = 0; k0 < 512 / 32; k0 += 8) {
        C ld[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          ld[k] = src[0];
          src += step;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) tile[(r0 + 32 * (k0 + k)) * COL_LD + c] = ld[k];
      }
    }
    __syncthreads();
    unsigned wplane;
    int wcol;
    if (used(warp, wplane, wcol)) {
      C *colp = tile + warp;
      C v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = colp[(lane + 32 * j) * COL_LD];
      __syncwarp();
      // the column itself is the scratch line (slot i at row i)
      warp_fft512(v, colp, COL_LD, s_tw, lane);
      const int k2 = lane & 15, b = lane >> 4;
#pragma unroll
      for (int a = 0; a < 16; ++a) colp[(k2 + 16 * a + 256 * b) * COL_LD] = v[a];
    }
    __syncthreads();
    // output rows hw = 0 .. hm come from tile rows hw, rows hm + 1 .. M - 1
    // (h = hw - M < 0) from tile rows 512 + hw - M
    if (mine) {
      const int64_t ostep = 32 * cp.out_r;
      C *dst = out + t * cp.out_t + p * cp.out_p + col + (int64_t)r0 * cp.out_r;
      const C *tp = tile + r0 * COL_LD + c;
      int hw = r0;
      if (cp.blk_rows) {
        // rows h in [lo, hi] only (positive h at row h, negative at row M + h of
        // the output and 512 + h of the tile), as per-thread loop bounds
        const short2 rr = __ldg(cp.blk_rows + col / COLS);
        const int lo = rr.x, hi = rr.y;
        C *obase = out + t * cp.out_t + p * cp.out_p + col;
        const int pl = max(lo, 0), ph = min(hi, cp.hm);
        for (int h = pl + (((r0 - pl) % 32) + 32) % 32; h <= ph; h += 32)
          obase[(int64_t)h * cp.out_r] = tile[h * COL_LD + c];
        const int nl = max(lo, -cp.hm), nh = min(hi, -1);
        for (int h = nl + (((r0 - (M + nl)) % 32) + 32) % 32; h <= nh; h += 32)
          obase[(int64_t)(M + h) * cp.out_r] = tile[(512 + h) * COL_LD + c];
      } else {
        for (; hw <= cp.hm; hw += 32, tp += 32 * COL_LD, dst += ostep) *dst = *tp;
        tp += (512 - M) * COL_LD;
        for (; hw < M; hw += 32, tp += 32 * COL_LD, dst += ostep) *dst = *tp;
      }
    }
  }
}

template <typename R> size_t cols_smem() {
  return sizeof(typename Cplx<R>::T) * (TW_LEN + 512 * COL_LD);
}

}  // namespace

template <typename R> cudaError_t fft512_set_attributes() {
  return cudaFuncSetAttribute(k_fft512_cols<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)cols_smem<R>());
}
template cudaError_t fft512_set_attributes<float>();
template cudaError_t fft512_set_attributes<double>();

// Twiddle table of the passes (TW_LEN complex values, FP64 on the host).
void fft512_twiddles(std::vector<double> &tw) {
  tw.assign(2 * TW_LEN, 0.0);
  for (int m = 0; m < TW_LEN; ++m) {
    const int e = m < 512 ? m : ((m - 512) & 31) * ((m - 512) >> 5);  // n1 k2
    const double a = -2.0 * M_PI * (double)e / 512.0;
    tw[2 * m] = std::cos(a);
    tw[2 * m + 1] = std::sin(a);
  }
}

// grid [ntr][nf2][nf1][pitch] real -> A1 [ntr][nf2][nf1][P1] -> A2 [ntr][nf2][M2][P1]
// -> G [ntr][M3][M2][P1] with h1 = 0 .. H1 - 1 of each P1-long row used (A2 may share
// the grid's storage; A1 and G share one buffer).  h1_end (optional, [M2] in FFT
// order of h2): the z pass skips the columns (h1, h2) with h1 >= h1_end[h2], which
// hold no kept mode for any h3; h2_band (optional, short2 per 16-column block of
// h1): the y pass writes only the h2 rows [lo, hi] of a block that some of its
// columns need.  A2's and G's entries elsewhere are left unwritten.  A row pitch P1 of 16 complex
// values makes every 16-column segment the column passes move start on a 128-byte
// boundary.
template <typename R>
cudaError_t launch_fft512(const R *grid, void *A1, void *A2, void *G, int ntr, int64_t pitch,
                          int H1, int P1, int hm1, int hm2, const void *tw,
                          const int *h1_end, const void *h2_band, int nsm, cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const int n = 512;
  const int M2 = 2 * hm1 + 1, M3 = 2 * hm2 + 1;
  const int64_t nrows = (int64_t)ntr * n * n;
  if (P1 < H1 || (int64_t)ntr * n * (H1 / COLS + 1) >= ((int64_t)1 << 31))
    return cudaErrorInvalidValue;
  k_fft512_x<R><<<nsm * 8, 32 * x_warps<R>(), 0, s>>>(grid, (C *)A1, nrows, pitch, H1, P1,
                                                      (const C *)tw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t sm = cols_smem<R>();
  const int cta = sizeof(R) == 4 ? 2 : 1;
  ColPass y;
  y.in_t = (int64_t)n * n * P1;
  y.in_p = (int64_t)n * P1;
  y.in_r = P1;
  y.out_t = (int64_t)n * M2 * P1;
  y.out_p = (int64_t)M2 * P1;
  y.out_r = P1;
  y.planes_per_t = n;
  y.nplanes = (int64_t)ntr * n;
  y.ncols = H1;
  y.hm = hm1;
  y.col_end = nullptr;
  y.blk_rows = static_cast<const short2 *>(h2_band);  // per 16-column block of h1
  auto cols = [&](const void *src, void *dst, const ColPass &cp) {
    k_fft512_cols<R><<<nsm * cta, 32 * COLS, sm, s>>>((const C *)src, (C *)dst, cp,
                                                      (const C *)tw);
  };
  cols(A1, A2, y);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  ColPass z;
  z.in_t = (int64_t)n * M2 * P1;
  z.in_p = P1;
  z.in_r = (int64_t)M2 * P1;
  z.out_t = (int64_t)M3 * M2 * P1;
  z.out_p = P1;
  z.out_r = (int64_t)M2 * P1;
  z.planes_per_t = M2;
  z.nplanes = (int64_t)ntr * M2;
  z.ncols = H1;
  z.hm = hm2;
  z.col_end = h1_end;  // plane p = h2 in FFT order
  z.blk_rows = nullptr;
  cols(A2, G, z);
  return cudaGetLastError();
}
template cudaError_t launch_fft512<float>(const float *, void *, void *, void *, int, int64_t,
                                          int, int, int, int, const void *, const int *,
                                          const void *, int, cudaStream_t);
template cudaError_t launch_fft512<double>(const double *, void *, void *, void *, int, int64_t,
                                           int, int, int, int, const void *, const int *,
                                           const void *, int, cudaStream_t);

}  // namespace sqn
