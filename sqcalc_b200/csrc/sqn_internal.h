// Internal types shared by the host side (sqn_api.cu, sqn_noalloc.cu) and the
// kernels (sqn_kernels.cu) of libsqnufft.so.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace sqn {

// Spread tile in fine-grid cells (x fastest).  A CTA of 16 warps owns one
// 32 x 16 x 32 tile of ONE transform (grid y index = transform); warp k owns
// the 8 x 4 (x, y) patch ((k % 4) * 8, (k / 4) * 4) of it and each lane keeps
// 16 z-cells of its (x, y) column in registers, in two passes over the tile.
// The bin sort keys points by (transform, tile), so a CTA reads only the bins
// of its own transform.
constexpr int TILE_X = 32;
constexpr int TILE_Y = 16;
constexpr int TILE_Z = 32;
constexpr int PATCH_X = 8;
constexpr int PATCH_Y = 4;
constexpr int SPREAD_WARPS = (TILE_X / PATCH_X) * (TILE_Y / PATCH_Y);  // 16
constexpr int SPREAD_THREADS = 32 * SPREAD_WARPS;                       // 512
// staged values per point: x row, y row, z row, 4 of padding (row pitch 84
// values: consecutive rows start 20 banks apart)
constexpr int SPREAD_ROW = TILE_X + TILE_Y + TILE_Z + 4;
static_assert((TILE_X & (TILE_X - 1)) == 0 && (TILE_Y & (TILE_Y - 1)) == 0 &&
                  (TILE_Z & (TILE_Z - 1)) == 0,
              "tile extents are powers of two");
constexpr int MAX_W = 16;
// A bin is one tile, so a tile's start cells X0 - (w - 1) .. X0 + T - 1 (cyclic)
// span fewer than 2T cells for w - 1 < T: its own bin, the one before and, when
// the axis ends in a tile shorter than w - 1 that the range wraps across, the
// one before that -- at most 3 bins per dimension.
constexpr int MAX_BINS_DIM = 3;
constexpr int MAX_NB = MAX_BINS_DIM * MAX_BINS_DIM * MAX_BINS_DIM;  // neighbour bins of a tile
constexpr int MAX_FAST_T = 8;                  // species held in registers (k_bin)
// Shape facts k_spread hard-codes (lane -> cell map, patch masks, 8-cell z
// groups, 16-byte aligned staged rows).
static_assert(TILE_X / PATCH_X == 4 && PATCH_X == 8 && PATCH_Y == 4,
              "k_spread maps warp & 3 / lane & 7 / lane >> 3 onto the patches");
static_assert(4 + TILE_Y / PATCH_Y <= 8, "patch mask bits 0-7, z-group bits 8-11");
static_assert(TILE_Z == 32, "two passes of two 8-cell z groups per lane");
static_assert((TILE_X + TILE_Y) % 4 == 0 && SPREAD_ROW % 4 == 0,
              "staged rows and their z part are 16-byte aligned");
static_assert(MAX_W - 1 < TILE_X && MAX_W - 1 < TILE_Y && MAX_W - 1 < TILE_Z,
              "a tile's bin list per dimension fits MAX_BINS_DIM for every w <= MAX_W");
static_assert(MAX_NB <= 32, "one bin per lane in the bin-list prefix");
static_assert(MAX_W - 1 < TILE_Z / 2, "the half-depth tiles of small grids keep <= 3 bins too");

// z extent of the spread tiles of a fine grid: TILE_Z (two accumulation passes
// over one staging of the points) when the grids still give at least 4 CTAs
// per SM, else TILE_Z / 2 (one pass; small grids keep twice the CTAs).
inline int spread_tile_z(const int64_t *nf, int ngrids, int nsm) {
  const int64_t nxy = ((nf[0] + TILE_X - 1) / TILE_X) * ((nf[1] + TILE_Y - 1) / TILE_Y);
  const int64_t ctas = nxy * ((nf[2] + TILE_Z - 1) / TILE_Z) * (int64_t)ngrids;
  return ctas >= 4 * (int64_t)nsm ? TILE_Z : TILE_Z / 2;
}

// Point records written by the bin sort and read by the spread and
// interpolation kernels: four R-sized slots per atom,
//   slot 0     packed word: bits 0-7 / 8-15 / 16-23 first support cell relative
//              to the home tile origin in x / y / z, bits 24-31 species index
//              (stored in the slot's low 32 bits)
//   slots 1-3  off_d = (X_d - ix0_d) - (w/2 - 1/2), the offset of the atom from
//              the centre of its support along each axis, in R precision; the ES
//              kernel value at support cell k is phi((k - (w/2 - 1/2)) - off_d)
// 16 bytes per atom in FP32, 32 in FP64 (one vector load each).
constexpr int REC_SLOTS = 4;
inline int rec_stride(int, bool) { return REC_SLOTS; }

// Geometry and kernel parameters, passed by value to the per-frame kernels.
struct FrameGeom {
  double inv[9];      // A^-1, inv[3*c + r] = (A^-1)(r, c)
  double origin[3];
  int nf[3];          // fine grid
  int tile[3];        // tile extent per dim
  int ntile[3];       // tiles per dim
  int w;              // ES kernel width
  double beta;        // ES shape
  int ntr;            // fine grids per frame (bins are keyed by transform when > 1)
  int ntiles;         // ntile[0]*ntile[1]*ntile[2]
  int rec_stride;     // R-sized slots per point record
  int chunk;          // points the spread stages in shared memory per pass
  int64_t pitch;     // real row pitch of the spread grid (elements)
  int64_t vol_real;   // real elements per fine grid
  int64_t natoms;
};

// Parameters of the fused deconvolve / pair-product / shell-binning pass.
struct BinGeom {
  double recip[9];    // b_j = recip[3*j + r]
  double qmin, qmax, dq;
  float qminf, qmaxf, invdqf;  // FP32 copies for the fast shell estimate
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
  // powder XRD pattern: xquant * xbins sums right after the nquant * nq shell
  // sums in the accumulator buffer
  int xrd, xbins, xquant, xlp;
  double xlambda, xmin, xstep;  // Angstrom, degrees, degrees
};

// FP64 sums of one frame pass: shell sums, then the powder-pattern sums.
__host__ __device__ inline int hist_len(const BinGeom &b) {
  return b.nquant * b.nq + (b.xrd ? b.xquant * b.xbins : 0);
}

// Launch wrappers (sqn_kernels.cu).  Each returns cudaGetLastError().
template <typename R>
cudaError_t launch_prep(const double *pos, const uint8_t *species, const FrameGeom &g,
                        int *counts, uint32_t *key, uint32_t *slot, cudaStream_t s);
cudaError_t launch_scan(int *counts, int *starts, int n, cudaStream_t s);
template <typename R>
cudaError_t launch_scatter(const double *pos, const uint8_t *species, const FrameGeom &g,
                           const uint32_t *key, const uint32_t *slot, const int *starts,
                           R *recs, int32_t *orig, cudaStream_t s);
template <typename R>
cudaError_t launch_spread(const R *recs, const int *starts, const FrameGeom &g,
                          const R *strength, R *grid, cudaStream_t s);
template <typename R>
cudaError_t launch_bin(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                       const R *inv1, const R *inv2, const R *inv3, const double *amp,
                       const double *xcoef, double *acc, double *gnum, int nsm,
                       cudaStream_t s);
cudaError_t launch_norms(const int4 *rows, int nrows, const BinGeom &b, const double *amp,
                         const double *xcoef, const double *counts_t, double *den,
                         double *cnt, double *xcnt, int nsm, cudaStream_t s);
size_t spread_smem_bytes(int chunk, bool fp64);
int spread_chunk(bool fp64);
cudaError_t spread_set_attributes();

// Host math (sqn_api.cu).
namespace hostmath {
int64_t next235even(int64_t n);
int es_width(double eps, double sigma);
double es_beta(int w, double sigma);
bool choose_fine_grid(const int *modes, double eps, double sigma_req, int w_req, int wcap,
                      int64_t *nf, int *w_out, double *sigma_out);
// phihat(k) of the ES kernel on an nf-point grid for k = 0 .. kmax
std::vector<double> kernel_ft(int64_t nf, int w, double beta, int kmax);
}  // namespace hostmath

// Pruned 512-point FFT passes (sqn_fft512.cu): grid -> A1 (x) -> A2 (y) -> G
// (z), G the compact half spectrum [ntr][2 hm2 + 1][2 hm1 + 1][P1] (rows of P1 >= H1
// complex values, h1 < H1 used; with h1_end, only h1 < h1_end[h2] written).
template <typename R> cudaError_t fft512_set_attributes();
void fft512_twiddles(std::vector<double> &tw);  // the passes' table, interleaved re, im
template <typename R>
cudaError_t launch_fft512(const R *grid, void *A1, void *A2, void *G, int ntr, int64_t pitch,
                          int H1, int P1, int hm1, int hm2, const void *tw, const int *h1_end,
                          const void *h2_band, int nsm, cudaStream_t s);

// Density amplitudes of requested lattice points from the half spectra.
template <typename R>
cudaError_t launch_gather_modes(const void *G, const BinGeom &b, const int *hkl, int64_t nm,
                                const R *inv1, const R *inv2, const R *inv3,
                                const double *origin, double *rho, cudaStream_t s);

// Spread with a weight per point instead of per species (g.ntr == 1): grid k
// of the ngrids takes the weights wsorted[k * natoms ..] (bin-sorted record
// order) and is written at grid + k * vol_real.
template <typename R>
cudaError_t launch_spread_pw(const R *recs, const int *starts, const FrameGeom &g,
                             const R *wsorted, R *grid, int ngrids, cudaStream_t s);
// Bin keys of a frame geometry: one per (transform, tile).
inline int64_t spread_nkeys(const FrameGeom &g) {
  return (int64_t)g.ntiles * (g.ntr > 1 ? g.ntr : 1);
}

// One system of a batch for the multi-system kernels: its geometry and the
// device buffers of its plan.  The batch keeps an array of these in device
// memory and runs each frame stage for all systems in one launch.
struct BatchSys {
  FrameGeom g;
  BinGeom b;
  const double *pos;
  const uint8_t *species;
  int *counts, *starts;
  uint32_t *key, *slot;
  void *recs;
  const void *strength;
  void *grid;
  const void *G;
  const int4 *rows;
  const void *inv[3];
  const double *amp, *xcoef;
  double *acc, *gnum;
  int nkeys, nrows;
};
// Block and atom offsets of the systems in the multi-system launches
// (prefix sums, nsys + 1 entries each, device memory).
struct BatchPrefix {
  const int64_t *atoms;  // atoms of systems < s
  const int *spread;     // spread CTAs (tiles x transforms) of systems < s
  const int *bin;        // bin CTAs of systems < s
};
constexpr int MAX_BATCH_SYSTEMS = 1024;
template <typename R>
cudaError_t launch_batch_sort(const BatchSys *sys, int nsys, const BatchPrefix &pre,
                              int64_t natoms, cudaStream_t s);
template <typename R>
cudaError_t launch_batch_spread(const BatchSys *sys, int nsys, const BatchPrefix &pre,
                                int nblocks, int chunk, cudaStream_t s);
// All systems share ntr, the x-ray flag and no powder pattern; hist_max is the
// largest nquant * nq.
template <typename R>
cudaError_t launch_batch_bin(const BatchSys *sys, int nsys, const BatchPrefix &pre, int nblocks,
                             int ntr, bool xray, int hist_max, cudaStream_t s);
// Shared-memory limits of the multi-system spread and bin kernels (call once,
// before any stream capture).
template <typename R> cudaError_t batch_set_attributes(int ntr, bool xray, int hist_max);

// Adjoint (sqn_adjoint.cu).
struct Recip {
  double b[9];  // b_j = b[3*j + r]
};
template <typename R>
cudaError_t launch_adj_coef(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                            const R *inv1, const R *inv2, const R *inv3, const double *gsh,
                            double *num, void *F, int nsm, cudaStream_t s);
template <typename R>
cudaError_t launch_interp(const R *recs, const int32_t *orig, const double *pos,
                          const FrameGeom &g, const R *U, const Recip &rb, const double *camp,
                          double *grad, cudaStream_t s);

}  // namespace sqn
