// Internal types shared by the host side (sqn_api.cu) and the kernels
// (sqn_kernels.cu) of libsqnufft.so.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sqn {

// Spread tile in fine-grid cells: 32 x-cells (one per lane, so every row store
// is a 128-byte coalesced write), 8 y-rows (one per warp), 8 z-cells held in
// registers by each thread.
constexpr int TILE_X = 32;
constexpr int TILE_Y = 8;
constexpr int TILE_Z = 8;
constexpr int SPREAD_THREADS = TILE_X * TILE_Y;  // 256
constexpr int ROW = TILE_X + TILE_Y + TILE_Z;    // kernel row entries per staged point
constexpr int CHUNK = SPREAD_THREADS;            // candidate points per pass
constexpr int MAX_W = 16;
constexpr int MAX_BINS_DIM = 4;                  // bins per dim a tile may need (w <= 16)
constexpr int MAX_NB = 64;                       // neighbour bins of a tile
constexpr int MAX_FAST_T = 8;                    // species held in registers by the bin kernel

// Point record written by the bin sort and read by the spread kernel.
// packed: bits 0-7 / 8-15 / 16-23 start cell of the kernel support relative to
// the origin of the home tile in x / y / z; bits 24-31 species index.
// f[d]: (X_d - ix0_d) - (w/2 - 1/2) in (-1/2, 1/2], X_d the fine-grid coordinate
// and ix0_d = ceil(X_d - w/2) the first cell of the support.
template <typename R> struct alignas(16) PointRec;
template <> struct alignas(16) PointRec<float> {
  float f[3];
  uint32_t packed;
};
template <> struct alignas(16) PointRec<double> {
  double f[3];
  uint32_t packed;
  uint32_t pad;
};

// Geometry and kernel parameters, passed by value to the per-frame kernels.
struct FrameGeom {
  double inv[9];      // A^-1, inv[3*c + r] = (A^-1)(r, c)
  double origin[3];
  int nf[3];          // fine grid
  int tile[3];        // tile extent per dim
  int ntile[3];       // tiles per dim
  int w;              // ES kernel width
  double beta;        // ES shape
  int ntr;            // fine grids per frame
  int ntiles;         // ntile[0]*ntile[1]*ntile[2]
  int64_t pitch;      // real row pitch of the spread grid (elements)
  int64_t vol_real;   // real elements per fine grid
  int64_t natoms;
};

// Parameters of the fused deconvolve / pair-product / shell-binning pass.
struct BinGeom {
  double recip[9];    // b_j = recip[3*j + r]
  double qmin, qmax, dq;
  int nq;
  int hm[3];          // (modes - 1) / 2
  int nf[3];
  int64_t c1;         // complex row length nf1/2 + 1
  int64_t vol_cplx;   // complex elements per transform
  int ntr;            // transforms
  int nquant;         // 1 + number of accumulated pair sums
  int partials;
  int xray;           // q-dependent amplitudes
  int want_grid;
  int m2;             // modes[1]
  int norm;
  int64_t natoms;
};

// Launch wrappers (sqn_kernels.cu).  Each returns cudaGetLastError().
template <typename R>
cudaError_t launch_prep(const double *pos, const uint8_t *species, const FrameGeom &g,
                        int *counts, uint32_t *key, uint32_t *slot, cudaStream_t s);
cudaError_t launch_scan(int *counts, int *starts, int n, cudaStream_t s);
template <typename R>
cudaError_t launch_scatter(const double *pos, const uint8_t *species, const FrameGeom &g,
                           const uint32_t *key, const uint32_t *slot, const int *starts,
                           PointRec<R> *recs, cudaStream_t s);
template <typename R>
cudaError_t launch_spread(const PointRec<R> *recs, const int *starts, const FrameGeom &g,
                          const R *strength, R *grid, cudaStream_t s);
template <typename R>
cudaError_t launch_bin(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                       const R *inv1, const R *inv2, const R *inv3, const double *amp,
                       const double *xcoef, double *acc, double *gnum, int nsm,
                       cudaStream_t s);
cudaError_t launch_norms(const int4 *rows, int nrows, const BinGeom &b, const double *amp,
                         const double *xcoef, const double *counts_t, double *den,
                         double *cnt, int nsm, cudaStream_t s);
size_t spread_smem_bytes(bool fp64);
cudaError_t spread_set_attributes();

}  // namespace sqn
