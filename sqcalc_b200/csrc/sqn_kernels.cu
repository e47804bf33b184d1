// Device kernels of the static S(q) hot path (sm_100a).
//
// Per frame:
//   k_prep     wrap each atom into the cell, find the first cell of its ES
//              kernel support on the fine grid and its home tile; count the
//              bin of (transform, tile)                          [HBM: positions]
//   k_scan     exclusive scan of the bin counts (one CTA) and reset the counts
//   k_scatter  write each atom's 16-byte record into its bin slot: packed start
//              cell + species and its three offsets from the support centre
//   k_spread   gather spreading: one CTA owns one 32 x 16 x 16 fine-grid tile
//              of one transform, stages the ES kernel values of the points of
//              that transform's bins that can reach it, already shifted onto
//              the tile's cells, in shared memory, and each warp accumulates
//              its 8 x 4 patch (16 z-cells per lane) in registers from the
//              points that reach the patch; every cell is written exactly
//              once, so the grid needs no zeroing and no atomics
//                                                              [HBM: grid write]
//   (cuFFT R2C / D2Z, out of place)
//   k_bin      deconvolve the half-space modes, form the weighted total and the
//              pair products Re(rho_a rho_b*) and add them, in FP64, to
//              per-CTA shared-memory shell histograms flushed once per CTA
//                                                  [HBM: kept modes read once]
//
// The reference does the same math as cuFINUFFT spread + cuFFT + deconvolve
// (external/finufft/src/cuda/3d/spreadinterp3d.cuh:276-383,
//  external/finufft/src/cuda/deconvolve_wrapper.cu:76-118) followed by the host
// loops of src/sqc_structure_factor.f90:457-643.
#include <cstdint>
#include <cuda_runtime.h>

#include "sqn_device.cuh"
#include "sqn_internal.h"

namespace sqn {

namespace {

using namespace dev;

// Bin key of atom i and its slot in the bin.
__device__ __forceinline__ void prep_atom(const double *__restrict__ pos,
                                          const uint8_t *__restrict__ species,
                                          const FrameGeom &g, int *__restrict__ counts,
                                          uint32_t *__restrict__ key, uint32_t *__restrict__ slot,
                                          int64_t i) {
  AtomCell c;
  atom_cell(pos, i, g, c);
  int l0, l1, l2;
  // bins of transform t follow those of transform t - 1 (one transform per species)
  const uint32_t k = home_key(c, g, l0, l1, l2) +
                     (g.ntr > 1 ? (uint32_t)species[i] * (uint32_t)g.ntiles : 0u);
  key[i] = k;
  slot[i] = (uint32_t)atomicAdd(&counts[k], 1);
}

__global__ void k_prep(const double *__restrict__ pos, const uint8_t *__restrict__ species,
                       FrameGeom g, int *__restrict__ counts, uint32_t *__restrict__ key,
                       uint32_t *__restrict__ slot) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.natoms;
       i += (int64_t)gridDim.x * blockDim.x)
    prep_atom(pos, species, g, counts, key, slot, i);
}

// Exclusive scan of counts[0..n) into starts[0..n], then zero counts for the
// next frame.  One CTA of 1024 threads walks the array in chunks of 4096
// (four consecutive counts per thread, vector loads and stores), carrying the
// running total from chunk to chunk.
__device__ __forceinline__ void scan_counts(int *__restrict__ counts, int *__restrict__ starts,
                                            int n) {
  __shared__ int wsum[32];
  __shared__ int s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 4096) {
    const int i0 = base + 4 * tid;
    int c[4] = {0, 0, 0, 0};
    const bool full = i0 + 3 < n;
    if (full) {
      const int4 v = *reinterpret_cast<const int4 *>(counts + i0);
      c[0] = v.x;
      c[1] = v.y;
      c[2] = v.z;
      c[3] = v.w;
    } else {
      for (int k = 0; k < 4; ++k)
        if (i0 + k < n) c[k] = counts[i0 + k];
    }
    const int s = c[0] + c[1] + c[2] + c[3];
    int v = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) wsum[warp] = v;
    __syncthreads();
    if (warp == 0) {
      int x = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += t;
      }
      wsum[lane] = x;
    }
    __syncthreads();
    const int excl = s_carry + v - s + (warp > 0 ? wsum[warp - 1] : 0);
    const int o0 = excl, o1 = o0 + c[0], o2 = o1 + c[1], o3 = o2 + c[2];
    if (full) {
      *reinterpret_cast<int4 *>(starts + i0) = make_int4(o0, o1, o2, o3);
      *reinterpret_cast<int4 *>(counts + i0) = make_int4(0, 0, 0, 0);
    } else {
      const int o[4] = {o0, o1, o2, o3};
      for (int k = 0; k < 4; ++k)
        if (i0 + k < n) {
          starts[i0 + k] = o[k];
          counts[i0 + k] = 0;
        }
    }
    __syncthreads();  // every thread has read s_carry and wsum
    if (tid == 1023) s_carry = excl + s;
    __syncthreads();
  }
  if (tid == 0) starts[n] = s_carry;
}

__global__ void __launch_bounds__(1024) k_scan(int *__restrict__ counts, int *__restrict__ starts,
                                               int n) {
  scan_counts(counts, starts, n);
}

// The 16-byte (FP32) / 32-byte (FP64) record of atom i at its sorted position.
template <typename R>
__device__ __forceinline__ void scatter_atom(const double *__restrict__ pos,
                                             const uint8_t *__restrict__ species,
                                             const FrameGeom &g, const uint32_t *__restrict__ key,
                                             const uint32_t *__restrict__ slot,
                                             const int *__restrict__ starts, R *__restrict__ recs,
                                             int32_t *__restrict__ orig, int64_t i) {
  AtomCell c;
  atom_cell(pos, i, g, c);
  const int sp = species[i];
  int l0, l1, l2;
  (void)home_key(c, g, l0, l1, l2);
  const int64_t dst = (int64_t)starts[key[i]] + slot[i];
  if (orig) orig[dst] = (int32_t)i;
  store_rec(recs + dst * REC_SLOTS,
            pack_rec<R>((uint32_t)l0 | ((uint32_t)l1 << 8) | ((uint32_t)l2 << 16) |
                        ((uint32_t)sp << 24)),
            (R)c.off[0], (R)c.off[1], (R)c.off[2]);
}

template <typename R>
__global__ void k_scatter(const double *__restrict__ pos, const uint8_t *__restrict__ species,
                          FrameGeom g, const uint32_t *__restrict__ key,
                          const uint32_t *__restrict__ slot, const int *__restrict__ starts,
                          R *__restrict__ recs, int32_t *__restrict__ orig) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.natoms;
       i += (int64_t)gridDim.x * blockDim.x)
    scatter_atom<R>(pos, species, g, key, slot, starts, recs, orig, i);
}

// Eight z values of a staged row (16-byte aligned) with vector loads.
__device__ __forceinline__ void load_z8(const float *src, float (&z)[8]) {
  const float4 a = reinterpret_cast<const float4 *>(src)[0];
  const float4 b = reinterpret_cast<const float4 *>(src)[1];
  z[0] = a.x; z[1] = a.y; z[2] = a.z; z[3] = a.w;
  z[4] = b.x; z[5] = b.y; z[6] = b.z; z[7] = b.w;
}
__device__ __forceinline__ void load_z8(const double *src, double (&z)[8]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double2 v = reinterpret_cast<const double2 *>(src)[k];
    z[2 * k] = v.x;
    z[2 * k + 1] = v.y;
  }
}

// c0 += a z0, c1 += a z1: one packed FP32 FMA (the sm_100 builtin, which the
// register allocator sees through) in FP32, two FMAs in FP64.
__device__ __forceinline__ void fma2(float a, float z0, float z1, float &c0, float &c1) {
  const float2 r = __ffma2_rn(make_float2(a, a), make_float2(z0, z1), make_float2(c0, c1));
  c0 = r.x;
  c1 = r.y;
}
__device__ __forceinline__ void fma2(double a, double z0, double z1, double &c0, double &c1) {
  c0 = fma(a, z0, c0);
  c1 = fma(a, z1, c1);
}

// Bits lo .. hi of a mask (0 <= lo <= hi < 32).
__device__ __forceinline__ unsigned bit_range(int lo, int hi) {
  return (0xffffffffu >> (31 - hi)) & (0xffffffffu << lo);
}
// Which P-cell groups of the tile cells [0, len) the cyclic support
// [r, r + w) (mod n, 0 <= r < n) reaches: bit k for cells [k P, k P + P).  The
// support meets the tile in [r, min(r + w, n, len)) when r < len, and in its
// wrapped part [0, min(r + w - n, len)) when r + w > n.
template <int P>
__device__ __forceinline__ unsigned group_mask(int r, int w, int len, int n) {
  unsigned m = 0u;
  if (r < len) m = bit_range(r / P, (min(min(r + w, n), len) - 1) / P);
  const int e = min(r + w - n, len);
  if (e > 0) m |= bit_range(0, (e - 1) / P);
  return m;
}

// ---------------------------------------------------------------------------
// Gather spreading, one CTA per (32 x 16 x 32 tile, transform).
// The CTA lists the bins of its transform that can reach the tile (at most 3
// per dimension), loads their point records, keeps the points whose support
// meets the tile (in candidate order: warp counts, then a prefix over the
// warps) and stages for each its kernel values already shifted onto the
// tile's cells (32 x, 16 y, 32 z with the strength folded in; zero where the
// support does not reach), with a mask of the 8 x 4 patches and of the four
// 8-cell z groups it reaches.  The tile is then accumulated in two passes of
// 16 z cells (16 registers per lane): a warp's visit of a point is two scalar
// loads, a multiply, and per z group of the pass that the point reaches two
// vector loads and four packed FMAs per lane.  The staging serves both passes
// when the tile's points fit the shared-memory capacity (g.chunk points);
// otherwise the points are staged in windows of that many, per pass.  Every
// cell of the tile is written exactly once: no zeroing, no atomics.
// ptw != nullptr (one grid per y index, g.ntr == 1): the weight of a point is
// ptw[y * natoms + record index] instead of strength[species].
// ---------------------------------------------------------------------------
constexpr int ZPASS = 16;  // z cells per accumulation pass

template <typename R>
__device__ __forceinline__ void spread_tile(const R *__restrict__ recs,
                                            const int *__restrict__ starts, const FrameGeom &g,
                                            const R *__restrict__ strength, R *__restrict__ grid,
                                            const R *__restrict__ ptw, const int tile,
                                            const int tr) {
  const int cap = g.chunk;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *s_rows = reinterpret_cast<R *>(smem_raw);                      // [cap][SPREAD_ROW]
  R *s_off = s_rows + (size_t)cap * SPREAD_ROW;                      // [cap][4]
  int4 *s_meta = reinterpret_cast<int4 *>(s_off + (size_t)cap * 4);  // [cap]
  unsigned *s_mask = reinterpret_cast<unsigned *>(s_meta + cap);     // [cap]
  __shared__ int s_bstart[MAX_NB];
  __shared__ int s_bpref[MAX_NB + 1];
  __shared__ int s_borg[MAX_NB][3];
  __shared__ int s_bl[3][MAX_BINS_DIM];
  __shared__ int s_nbl[3];
  __shared__ int s_wcount[SPREAD_WARPS];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cx = (warp & 3) * PATCH_X + (lane & 7);   // this lane's x cell in the tile
  const int cy = (warp >> 2) * PATCH_Y + (lane >> 3);  // and its y cell
  const int t0 = tile % g.ntile[0];
  const int t1 = (tile / g.ntile[0]) % g.ntile[1];
  const int t2 = tile / (g.ntile[0] * g.ntile[1]);
  const int X0 = t0 * g.tile[0], Y0 = t1 * g.tile[1], Z0 = t2 * g.tile[2];
  const int tx = min(g.tile[0], g.nf[0] - X0);
  const int ty = min(g.tile[1], g.nf[1] - Y0);
  const int tz = min(g.tile[2], g.nf[2] - Z0);
  const int w = g.w;
  // bins of transform tr (keys tr * ntiles + tile) when the transforms are
  // binned apart; per-point weights use one set of bins for every grid
  const int key0 = ptw ? 0 : tr * g.ntiles;
  if (ptw) ptw += (int64_t)tr * g.natoms;

  // Bins whose points can reach this tile, per dimension: a support starting
  // at cell c covers c .. c+w-1, so the start cells that matter are
  // X0-(w-1) .. X0+t-1, taken cyclically.
  if (tid < 3) {
    const int d = tid;
    const int T = g.tile[d], nt = g.ntile[d], n = g.nf[d];
    const int t = d == 0 ? t0 : (d == 1 ? t1 : t2);
    const int Xd = t * T, td = min(T, n - Xd);
    int cnt = 0;
    if (w - 1 + td >= n) {
      for (int b = 0; b < nt && cnt < MAX_BINS_DIM; ++b) s_bl[d][cnt++] = b;
    } else {
      const int ws = Xd - (w - 1);
      if (ws >= 0) {
        for (int b = ws / T; b <= t && cnt < MAX_BINS_DIM; ++b) s_bl[d][cnt++] = b;
      } else {
        for (int b = (n + ws) / T; b < nt && cnt < MAX_BINS_DIM; ++b) s_bl[d][cnt++] = b;
        for (int b = 0; b <= t && cnt < MAX_BINS_DIM; ++b) s_bl[d][cnt++] = b;
      }
    }
    s_nbl[d] = cnt;
  }
  __syncthreads();
  const int nb0 = s_nbl[0], nb1 = s_nbl[1];
  const int nb = nb0 * nb1 * s_nbl[2];
  if (warp == 0) {
    // one bin per lane (nb <= MAX_NB <= 32), inclusive prefix by shuffles
    int cnt = 0;
    if (lane < nb) {
      const int bx = s_bl[0][lane % nb0], by = s_bl[1][(lane / nb0) % nb1],
                bz = s_bl[2][lane / (nb0 * nb1)];
      const int key = key0 + (bz * g.ntile[1] + by) * g.ntile[0] + bx;
      const int st = starts[key];
      cnt = starts[key + 1] - st;
      s_bstart[lane] = st;
      s_borg[lane][0] = bx * g.tile[0];
      s_borg[lane][1] = by * g.tile[1];
      s_borg[lane][2] = bz * g.tile[2];
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane < nb) s_bpref[lane + 1] = incl;
    if (lane == 0) s_bpref[0] = 0;
  }
  __syncthreads();
  const int total = s_bpref[nb];

  const unsigned xbit = 1u << (warp & 3), ybit = 1u << (4 + (warp >> 2));
  const R halfw = R(0.5) * (R)w - R(0.5);
  const R c2 = R(4) / ((R)w * (R)w);
  const R beta = (R)g.beta;
  int kept = -1;  // points of the tile (after the first staging)
  int npts = 0;   // points staged in the current window
  R acc[ZPASS];

  for (int h = 0; h * ZPASS < tz; ++h) {
#pragma unroll
    for (int z = 0; z < ZPASS; ++z) acc[z] = R(0);
    for (int win = 0;; win += cap) {
      if (!(h > 0 && kept <= cap)) {
        // ---- stage the kept points win .. win + cap - 1 (candidate order)
        __syncthreads();  // the previous visits have read the rows
        int kbase = 0;
        for (int cb = 0; cb < total; cb += SPREAD_THREADS) {
          const int i = cb + tid;
          bool keep = false;
          int4 meta = make_int4(0, 0, 0, 0);
          unsigned mask = 0u;
          R rec[REC_SLOTS];
          if (i < total) {
            // bin of candidate i: s_bpref[b] <= i < s_bpref[b + 1]
            int lo = 0, hi = nb;
            while (hi - lo > 1) {
              const int mid = (lo + hi) >> 1;
              if (s_bpref[mid] <= i) lo = mid; else hi = mid;
            }
            const int ridx = s_bstart[lo] + (i - s_bpref[lo]);
            load_rec(recs + (int64_t)ridx * REC_SLOTS, rec);
            const uint32_t packed = unpack_rec<R>(rec[0]);
            int rx = s_borg[lo][0] + (int)(packed & 255u) - X0;
            int ry = s_borg[lo][1] + (int)((packed >> 8) & 255u) - Y0;
            int rz = s_borg[lo][2] + (int)((packed >> 16) & 255u) - Z0;
            if (rx < 0) rx += g.nf[0];
            if (ry < 0) ry += g.nf[1];
            if (rz < 0) rz += g.nf[2];
            keep = (rx < tx || rx + w > g.nf[0]) && (ry < ty || ry + w > g.nf[1]) &&
                   (rz < tz || rz + w > g.nf[2]);
            if (keep) {
              mask = group_mask<PATCH_X>(rx, w, tx, g.nf[0]) |
                     (group_mask<PATCH_Y>(ry, w, ty, g.nf[1]) << 4) |
                     (group_mask<8>(rz, w, tz, g.nf[2]) << 8);
              // with per-point weights the slot carries the record index
              meta = make_int4(rx, ry, rz, ptw ? ridx : (int)(packed >> 24));
            }
          }
          const unsigned bal = __ballot_sync(FULL, keep);
          if (lane == 0) s_wcount[warp] = __popc(bal);
          __syncthreads();
          // offsets of the warps' kept points: an inclusive scan of the warp
          // counts across lanes, read back at this warp
          const int wc = lane < SPREAD_WARPS ? s_wcount[lane] : 0;
          int wincl = wc;
#pragma unroll
          for (int o = 1; o < SPREAD_WARPS; o <<= 1) {
            const int t = __shfl_up_sync(FULL, wincl, o);
            if (lane >= o) wincl += t;
          }
          const int woff = __shfl_sync(FULL, wincl - wc, warp);
          const int btot = __shfl_sync(FULL, wincl, SPREAD_WARPS - 1);
          const int k = kbase + woff + __popc(bal & ((1u << lane) - 1u)) - win;
          if (keep && k >= 0 && k < cap) {
            s_meta[k] = meta;
            s_mask[k] = mask;
            store_rec(s_off + (size_t)k * 4, R(0), rec[1], rec[2], rec[3]);
          }
          kbase += btot;
          __syncthreads();  // s_wcount is reused by the next batch
        }
        kept = kbase;
        npts = min(cap, kept - win);

        // kernel values shifted onto the tile's cells: row c of point p holds
        // phi at tile cell c (x: c < 32, y: next 16, z: next 32, times the
        // weight), zero outside the support or the grid.  One thread per
        // (point, axis) clears its row and writes the w support values that
        // fall in the tile (the same thread, so no barrier between the two).
        for (int e = tid; e < 3 * npts; e += SPREAD_THREADS) {
          const int d = e >= 2 * npts ? 2 : (e >= npts ? 1 : 0);
          const int p = e - d * npts;
          const int4 m = s_meta[p];
          const int rel = d == 0 ? m.x : (d == 1 ? m.y : m.z);
          const int len = d == 0 ? TILE_X : (d == 1 ? TILE_Y : TILE_Z);
          const int lim = d == 0 ? tx : (d == 1 ? ty : tz);
          const int n = g.nf[d];
          const R off = s_off[(size_t)p * 4 + 1 + d];
          const R sc = d == 2 ? (ptw ? ptw[m.w] : strength[m.w]) : R(1);
          R *row = s_rows + (size_t)p * SPREAD_ROW +
                   (d == 0 ? 0 : (d == 1 ? TILE_X : TILE_X + TILE_Y));
          for (int j = 0; j < len; j += 4) store_rec(row + j, R(0), R(0), R(0), R(0));
          // support cell k sits at tile cell rel + k, cyclically (rel in [0, n));
          // unrolled to the largest width so the evaluations overlap
#pragma unroll
          for (int k = 0; k < MAX_W; ++k) {
            if (k < w) {
              int cell = rel + k;
              if (cell >= n) cell -= n;
              if (cell < lim) row[cell] = es_at(k, off, halfw, c2, beta) * sc;
            }
          }
        }
        __syncthreads();
      }

      // ---- each warp walks only the points that reach its patch in this pass
      const unsigned zsel = 3u << (8 + 2 * h);
      for (int pb = 0; pb < npts; pb += 32) {
        const int p = pb + lane;
        unsigned m = 0u;
        if (p < npts) m = s_mask[p];
        unsigned am = __ballot_sync(FULL, (m & xbit) && (m & ybit) && (m & zsel));
        while (am) {
          const int src = __ffs(am) - 1;
          am &= am - 1u;
          const unsigned zm = __shfl_sync(FULL, m, src) >> (8 + 2 * h);
          const R *row = s_rows + (size_t)(pb + src) * SPREAD_ROW;
          const R a = row[cx] * row[TILE_X + cy];
          const R *zr = row + TILE_X + TILE_Y + h * ZPASS;
          if (zm & 1u) {
            R z[8];
            load_z8(zr, z);
#pragma unroll
            for (int k = 0; k < 8; k += 2) fma2(a, z[k], z[k + 1], acc[k], acc[k + 1]);
          }
          if (zm & 2u) {
            R z[8];
            load_z8(zr + 8, z);
#pragma unroll
            for (int k = 0; k < 8; k += 2) fma2(a, z[k], z[k + 1], acc[8 + k], acc[9 + k]);
          }
        }
      }
      if (win + cap >= kept) break;
    }

    if (cx < tx && cy < ty) {
      const int64_t zs = (int64_t)g.nf[1] * g.pitch;
      R *out = grid + (int64_t)tr * g.vol_real +
               ((int64_t)(Z0 + h * ZPASS) * g.nf[1] + (Y0 + cy)) * g.pitch + X0 + cx;
#pragma unroll
      for (int z = 0; z < ZPASS; ++z)
        if (h * ZPASS + z < tz) out[z * zs] = acc[z];
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(SPREAD_THREADS, sizeof(R) == 4 ? 2 : 1)
    k_spread(const R *__restrict__ recs, const int *__restrict__ starts, FrameGeom g,
             const R *__restrict__ strength, R *__restrict__ grid,
             const R *__restrict__ ptw = nullptr) {
  spread_tile<R>(recs, starts, g, strength, grid, ptw, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Fused deconvolve + weighted total + pair products + FP64 shell binning.
// NT > 0: exactly NT transforms (unrolled).  NT == 0: any ntr <= MAX_FAST_T.
// Rows (h2, h3) are dealt to warps; lanes walk h1 >= 0 (32 consecutive complex
// values per warp and transform, one coalesced read).
// ---------------------------------------------------------------------------
// Rows r = r0, r0 + rstep, ... of the half space, one warp each, into the
// histograms hist (and xhist for the powder pattern, gnum for the grid).
template <typename R, int NT, bool XR, bool XD>
__device__ __forceinline__ void bin_rows(const int4 *__restrict__ rows, int nrows,
                                         const typename Cplx<R>::T *__restrict__ G,
                                         const BinGeom &b, const R *__restrict__ inv1,
                                         const R *__restrict__ inv2, const R *__restrict__ inv3,
                                         const double *__restrict__ amp,
                                         const double *__restrict__ xcoef, double *hist,
                                         double *xhist, double *__restrict__ gnum, int r0,
                                         int rstep, int lane, int hq = -1, int hs = 1) {
  const int ntr = NT > 0 ? NT : b.ntr;
  constexpr int TM = NT > 0 ? NT : MAX_FAST_T;
  for (int r = r0; r < nrows; r += rstep) {
    const int4 row = rows[r];
    const int h2 = row.x, h3 = row.y, lo = row.z, hi = row.w;
    const int64_t ky = h2 >= 0 ? h2 : b.nf[1] + h2;
    const int64_t kz = h3 >= 0 ? h3 : b.nf[2] + h3;
    const int64_t rowbase = (kz * b.nf[1] + ky) * b.c1;
    const R dyz = inv2[abs(h2)] * inv3[abs(h3)];
    const int64_t gbase =
        ((int64_t)(h3 + b.hm[2]) * b.m2 + (int64_t)(h2 + b.hm[1])) * (int64_t)(b.hm[0] + 1);
    double crow[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
      crow[k] = fma((double)h2, b.recip[3 + k], (double)h3 * b.recip[6 + k]);
    for (int h1b = lo; h1b <= hi; h1b += 32) {
      const int h1 = h1b + lane;
      const bool inrow = h1 <= hi;
      // Issue the loads first: they do not depend on the classification.
      typename Cplx<R>::T v[TM];
#pragma unroll
      for (int t = 0; t < TM; ++t)
        if (t < ntr && inrow) v[t] = G[(int64_t)t * b.vol_cplx + rowbase + h1];
      const R dec = inrow ? inv1[h1] * dyz : R(0);
      bin_mode<R, TM, XR, XD>(b, ntr, inrow, h1, h2, h3, crow, v, dec, amp, xcoef, hist, gnum,
                              gbase + h1, lane, xhist, hq, hs);
    }
  }
}

template <typename R, int NT, bool SMEM, bool XR, bool XD>
__global__ void __launch_bounds__(256, 2)
    k_bin(const int4 *__restrict__ rows, int nrows, const typename Cplx<R>::T *__restrict__ G,
          BinGeom b, const R *__restrict__ inv1, const R *__restrict__ inv2,
          const R *__restrict__ inv3, const double *__restrict__ amp,
          const double *__restrict__ xcoef, double *__restrict__ acc, double *__restrict__ gnum) {
  extern __shared__ double s_hist[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int nhist = hist_len(b);
  double *hist = SMEM ? s_hist : acc;
  double *xhist = XD ? hist + b.nquant * b.nq : nullptr;
  if (SMEM) {
    for (int i = tid; i < nhist; i += blockDim.x) s_hist[i] = 0.0;
    __syncthreads();
  }
  // the shared sums are shell-major (the nquant sums of a shell side by side,
  // fewer bank collisions between the lanes' atomics); the flush restores the
  // accumulators' quantity-major layout
  const int nsh = b.nquant * b.nq;
  bin_rows<R, NT, XR, XD>(rows, nrows, G, b, inv1, inv2, inv3, amp, xcoef, hist, xhist, gnum,
                          blockIdx.x * nwarps + warp, gridDim.x * nwarps, lane,
                          SMEM ? 1 : b.nq, SMEM ? b.nquant : 1);
  if (SMEM) {
    __syncthreads();
    for (int i = tid; i < nhist; i += blockDim.x) {
      const double v = s_hist[i];
      const int g = i < nsh ? (i % b.nquant) * b.nq + i / b.nquant : i;
      if (v != 0.0) atomicAdd(&acc[g], v);
    }
  }
}

// den(shell) and shell_count(shell) over all kept modes (both halves),
// mode_denominator of src/sqc_structure_factor.f90:425-451.
__global__ void __launch_bounds__(256)
    k_norms(const int4 *__restrict__ rows, int nrows, BinGeom b, const double *__restrict__ amp,
            const double *__restrict__ xcoef, const double *__restrict__ counts_t,
            double *__restrict__ den, double *__restrict__ cnt, double *__restrict__ xcnt) {
  extern __shared__ double s_n[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int nx = b.xrd ? b.xbins : 0;
  for (int i = tid; i < 2 * b.nq + nx; i += blockDim.x) s_n[i] = 0.0;
  __syncthreads();
  for (int r = blockIdx.x * nwarps + warp; r < nrows; r += gridDim.x * nwarps) {
    const int4 row = rows[r];
    const int h2 = row.x, h3 = row.y, lo = row.z, hi = row.w;
    for (int h1b = lo; h1b <= hi; h1b += 32) {
      const int h1 = h1b + lane;
      bool keep = h1 <= hi;
      double ql = 0.0;
      int s = 0;
      if (keep) {
        ql = qlen_exact(b, h1, h2, h3);
        keep = !(h1 == 0 && h2 == 0 && h3 == 0) && ql >= b.qmin && ql <= b.qmax;
        s = shell_of(b, ql);
      }
      if (!keep) continue;
      const double mult = h1 > 0 ? 2.0 : 1.0;
      double d;
      if (b.norm == 3) {
        d = (double)b.natoms;
      } else {
        double sw = 0.0, sw2 = 0.0;
        for (int t = 0; t < b.ntr; ++t) {
          const double w = b.xray ? xray_f(xcoef + 9 * t, ql) : amp[t];
          sw = sw + counts_t[t] * w;
          sw2 = sw2 + counts_t[t] * w * w;
        }
        d = b.norm == 1 ? sw * sw / (double)b.natoms : sw2;
      }
      atomicAdd(&s_n[s], mult * d);
      atomicAdd(&s_n[b.nq + s], mult);
      if (nx) {
        int xb;
        double wt;
        xrd_bin_weight(b, ql, xb, wt);
        atomicAdd(&s_n[2 * b.nq + xb], mult);
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < b.nq; i += blockDim.x) {
    if (s_n[i] != 0.0) atomicAdd(&den[i], s_n[i]);
    if (s_n[b.nq + i] != 0.0) atomicAdd(&cnt[i], s_n[b.nq + i]);
  }
  for (int i = tid; i < nx; i += blockDim.x)
    if (s_n[2 * b.nq + i] != 0.0) atomicAdd(&xcnt[i], s_n[2 * b.nq + i]);
}

// Density amplitudes rho_t(h) = sum_{j in t} exp(i q_h . r_j) of requested
// lattice points h (hkl[3m..3m+2], |h_d| <= hm_d) from the half spectra of the
// per-species transforms: the forward FFT gives phihat(h) sum exp(-2 pi i h.s),
// so rho = exp(i q.origin) conj(G(h)) / phihat(h), with G(-h) = conj G(h) for
// h1 < 0.  Output rho[(t nm + m) 2 + {0, 1}] in FP64; modes outside the cube
// give 0.
template <typename R>
__global__ void k_gather_modes(const typename Cplx<R>::T *__restrict__ G, BinGeom b,
                               const int *__restrict__ hkl, int64_t nm,
                               const R *__restrict__ inv1, const R *__restrict__ inv2,
                               const R *__restrict__ inv3, double o0, double o1, double o2,
                               double *__restrict__ rho) {
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nm;
       m += (int64_t)gridDim.x * blockDim.x) {
    const int h1 = hkl[3 * m], h2 = hkl[3 * m + 1], h3 = hkl[3 * m + 2];
    const bool in = abs(h1) <= b.hm[0] && abs(h2) <= b.hm[1] && abs(h3) <= b.hm[2];
    int q1 = h1, q2 = h2, q3 = h3;
    const bool cj = h1 < 0;
    if (cj) {
      q1 = -q1;
      q2 = -q2;
      q3 = -q3;
    }
    const int64_t idx = ((int64_t)(q3 >= 0 ? q3 : b.nf[2] + q3) * b.nf[1] +
                         (q2 >= 0 ? q2 : b.nf[1] + q2)) * b.c1 + q1;
    double ph = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const double q = (double)h1 * b.recip[r] + (double)h2 * b.recip[3 + r] +
                       (double)h3 * b.recip[6 + r];
      ph += q * (r == 0 ? o0 : (r == 1 ? o1 : o2));
    }
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double dec = in ? (double)(inv1[abs(h1)] * inv2[abs(h2)] * inv3[abs(h3)]) : 0.0;
    for (int t = 0; t < b.ntr; ++t) {
      double vx = 0.0, vy = 0.0;
      if (in) {
        const typename Cplx<R>::T gv = G[(int64_t)t * b.vol_cplx + idx];
        vx = (double)gv.x * dec;                   // conj(G(h)) / phihat, G(h) from
        vy = (cj ? (double)gv.y : -(double)gv.y) * dec;  // the stored half
      }
      rho[2 * (t * nm + m)] = vx * cs - vy * sn;
      rho[2 * (t * nm + m) + 1] = vx * sn + vy * cs;
    }
  }
}

// ---------------------------------------------------------------------------
// Multi-system kernels of a batch: each frame stage runs for every system of
// the batch in one launch.  Atoms, spread CTAs and bin CTAs are numbered
// across the systems; a thread or CTA finds its system by binary search in the
// batch's prefix sums and takes that system's geometry and buffers from the
// BatchSys array.
// ---------------------------------------------------------------------------

// The s with pre[s] <= b < pre[s + 1] (pre[0] = 0, pre[nsys] > b).
template <typename T>
__device__ __forceinline__ int find_system(const T *pre, int nsys, T b) {
  int lo = 0, hi = nsys;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= b) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void k_batch_prep(const BatchSys *__restrict__ sys, int nsys,
                             const int64_t *__restrict__ apre, int64_t natoms) {
  __shared__ int64_t s_pre[MAX_BATCH_SYSTEMS + 1];
  for (int i = threadIdx.x; i <= nsys; i += blockDim.x) s_pre[i] = apre[i];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < natoms;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_system(s_pre, nsys, i);
    const BatchSys &S = sys[s];
    prep_atom(S.pos, S.species, S.g, S.counts, S.key, S.slot, i - s_pre[s]);
  }
}

__global__ void __launch_bounds__(1024) k_batch_scan(const BatchSys *__restrict__ sys) {
  const BatchSys &S = sys[blockIdx.x];
  scan_counts(S.counts, S.starts, S.nkeys);
}

template <typename R>
__global__ void k_batch_scatter(const BatchSys *__restrict__ sys, int nsys,
                                const int64_t *__restrict__ apre, int64_t natoms) {
  __shared__ int64_t s_pre[MAX_BATCH_SYSTEMS + 1];
  for (int i = threadIdx.x; i <= nsys; i += blockDim.x) s_pre[i] = apre[i];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < natoms;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_system(s_pre, nsys, i);
    const BatchSys &S = sys[s];
    scatter_atom<R>(S.pos, S.species, S.g, S.key, S.slot, S.starts, (R *)S.recs, nullptr,
                    i - s_pre[s]);
  }
}

// CTA b spreads tile (local % ntiles) of transform (local / ntiles) of its system.
template <typename R>
__global__ void __launch_bounds__(SPREAD_THREADS, sizeof(R) == 4 ? 2 : 1)
    k_batch_spread(const BatchSys *__restrict__ sys, int nsys, const int *__restrict__ bpre) {
  __shared__ FrameGeom s_g;
  __shared__ int s_sys, s_local;
  if (threadIdx.x == 0) {
    const int s = find_system(bpre, nsys, (int)blockIdx.x);
    s_sys = s;
    s_local = (int)blockIdx.x - bpre[s];
    s_g = sys[s].g;
  }
  __syncthreads();
  const BatchSys &S = sys[s_sys];
  spread_tile<R>((const R *)S.recs, S.starts, s_g, (const R *)S.strength, (R *)S.grid, nullptr,
                 s_local % s_g.ntiles, s_local / s_g.ntiles);
}

// The CTAs of a system share its rows; each CTA bins into a shared histogram
// of that system's nquant * nq sums and adds it to the system's accumulators.
template <typename R, int NT, bool XR>
__global__ void __launch_bounds__(256, 2)
    k_batch_bin(const BatchSys *__restrict__ sys, int nsys, const int *__restrict__ bpre) {
  extern __shared__ double s_hist[];
  __shared__ BinGeom s_b;
  __shared__ int s_sys, s_lb, s_nb;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  if (tid == 0) {
    const int s = find_system(bpre, nsys, (int)blockIdx.x);
    s_sys = s;
    s_lb = (int)blockIdx.x - bpre[s];
    s_nb = bpre[s + 1] - bpre[s];
    s_b = sys[s].b;
  }
  __syncthreads();
  const BatchSys &S = sys[s_sys];
  const int nhist = s_b.nquant * s_b.nq;
  for (int i = tid; i < nhist; i += blockDim.x) s_hist[i] = 0.0;
  __syncthreads();
  bin_rows<R, NT, XR, false>(S.rows, S.nrows, (const typename Cplx<R>::T *)S.G, s_b,
                             (const R *)S.inv[0], (const R *)S.inv[1], (const R *)S.inv[2],
                             S.amp, S.xcoef, s_hist, nullptr, S.gnum, s_lb * nwarps + warp,
                             s_nb * nwarps, lane, 1, s_b.nquant);
  __syncthreads();
  // shell-major shared sums back to the quantity-major accumulators
  for (int i = tid; i < nhist; i += blockDim.x) {
    const double v = s_hist[i];
    if (v != 0.0) atomicAdd(&S.acc[(i % s_b.nquant) * s_b.nq + i / s_b.nquant], v);
  }
}

}  // namespace

static int grid_for(int64_t n, int threads);

template <typename R>
cudaError_t launch_gather_modes(const void *G, const BinGeom &b, const int *hkl, int64_t nm,
                                const R *inv1, const R *inv2, const R *inv3,
                                const double *origin, double *rho, cudaStream_t s) {
  k_gather_modes<R><<<grid_for(nm, 256), 256, 0, s>>>(
      (const typename Cplx<R>::T *)G, b, hkl, nm, inv1, inv2, inv3, origin[0], origin[1],
      origin[2], rho);
  return cudaGetLastError();
}
template cudaError_t launch_gather_modes<float>(const void *, const BinGeom &, const int *,
                                                int64_t, const float *, const float *,
                                                const float *, const double *, double *,
                                                cudaStream_t);
template cudaError_t launch_gather_modes<double>(const void *, const BinGeom &, const int *,
                                                 int64_t, const double *, const double *,
                                                 const double *, const double *, double *,
                                                 cudaStream_t);

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------

static int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 32) b = 148 * 32;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename R>
cudaError_t launch_prep(const double *pos, const uint8_t *species, const FrameGeom &g,
                        int *counts, uint32_t *key, uint32_t *slot, cudaStream_t s) {
  k_prep<<<grid_for(g.natoms, 256), 256, 0, s>>>(pos, species, g, counts, key, slot);
  return cudaGetLastError();
}

cudaError_t launch_scan(int *counts, int *starts, int n, cudaStream_t s) {
  k_scan<<<1, 1024, 0, s>>>(counts, starts, n);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_scatter(const double *pos, const uint8_t *species, const FrameGeom &g,
                           const uint32_t *key, const uint32_t *slot, const int *starts,
                           R *recs, int32_t *orig, cudaStream_t s) {
  k_scatter<R><<<grid_for(g.natoms, 256), 256, 0, s>>>(pos, species, g, key, slot, starts, recs,
                                                       orig);
  return cudaGetLastError();
}

size_t spread_point_bytes(bool fp64) {
  const size_t r = fp64 ? 8 : 4;
  return (size_t)(SPREAD_ROW + 4) * r + sizeof(int4) + sizeof(unsigned);
}

size_t spread_smem_bytes(int chunk, bool fp64) {
  return (size_t)chunk * spread_point_bytes(fp64);
}

int spread_chunk(bool fp64) {
  // Two FP32 CTAs per SM share ~216 KB of shared memory; an FP64 CTA has it alone.
  const size_t budget = fp64 ? 216 * 1024 : 106 * 1024;
  int c = (int)(budget / spread_point_bytes(fp64));
  c = c > SPREAD_THREADS ? SPREAD_THREADS : c;
  return c / 32 * 32;
}

// Allow each spread instantiation the device's opt-in shared memory minus its
// static shared memory.
template <typename K> static cudaError_t smem_optin(K kernel, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - (int)fa.sharedSizeBytes);
}

cudaError_t spread_set_attributes() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = smem_optin(k_spread<float>, optin);
  if (e == cudaSuccess) e = smem_optin(k_spread<double>, optin);
  return e;
}

// One CTA per (tile, transform): grid (ntiles, ntr).
template <typename R>
cudaError_t launch_spread(const R *recs, const int *starts, const FrameGeom &g,
                          const R *strength, R *grid, cudaStream_t s) {
  if (g.ntr < 1 || g.ntr > MAX_FAST_T) return cudaErrorInvalidValue;
  const dim3 grd((unsigned)g.ntiles, (unsigned)g.ntr);
  const size_t sm = spread_smem_bytes(g.chunk, sizeof(R) == 8);
  k_spread<R><<<grd, SPREAD_THREADS, sm, s>>>(recs, starts, g, strength, grid);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_spread_pw(const R *recs, const int *starts, const FrameGeom &g,
                             const R *wsorted, R *grid, int ngrids, cudaStream_t s) {
  if (g.ntr != 1 || !wsorted || ngrids < 1 || ngrids > 65535) return cudaErrorInvalidValue;
  const size_t sm = spread_smem_bytes(g.chunk, sizeof(R) == 8);
  const dim3 grd((unsigned)g.ntiles, (unsigned)ngrids);
  k_spread<R><<<grd, SPREAD_THREADS, sm, s>>>(recs, starts, g, nullptr, grid, wsorted);
  return cudaGetLastError();
}

template <typename R, int NT, bool XR>
static cudaError_t bin_dispatch_xr(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                                   const R *i1, const R *i2, const R *i3, const double *amp,
                                   const double *xc, double *acc, double *gnum, int nsm,
                                   cudaStream_t s) {
  using C = typename Cplx<R>::T;
  const size_t hist = (size_t)hist_len(b) * sizeof(double);
  const int blocks = nsm * 4;
  if (hist <= 160 * 1024) {
    if (b.xrd) {
      cudaError_t e = cudaFuncSetAttribute(k_bin<R, NT, true, XR, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist);
      if (e != cudaSuccess) return e;
      k_bin<R, NT, true, XR, true><<<blocks, 256, hist, s>>>(rows, nrows, (const C *)G, b, i1,
                                                             i2, i3, amp, xc, acc, gnum);
    } else {
      cudaError_t e = cudaFuncSetAttribute(k_bin<R, NT, true, XR, false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist);
      if (e != cudaSuccess) return e;
      k_bin<R, NT, true, XR, false><<<blocks, 256, hist, s>>>(rows, nrows, (const C *)G, b, i1,
                                                              i2, i3, amp, xc, acc, gnum);
    }
  } else if (b.xrd) {
    k_bin<R, NT, false, XR, true><<<blocks, 256, 0, s>>>(rows, nrows, (const C *)G, b, i1, i2, i3,
                                                         amp, xc, acc, gnum);
  } else {
    k_bin<R, NT, false, XR, false><<<blocks, 256, 0, s>>>(rows, nrows, (const C *)G, b, i1, i2,
                                                          i3, amp, xc, acc, gnum);
  }
  return cudaGetLastError();
}

template <typename R, int NT>
static cudaError_t bin_dispatch_smem(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                                     const R *i1, const R *i2, const R *i3, const double *amp,
                                     const double *xc, double *acc, double *gnum, int nsm,
                                     cudaStream_t s) {
  if (b.xray) return bin_dispatch_xr<R, NT, true>(rows, nrows, G, b, i1, i2, i3, amp, xc, acc, gnum, nsm, s);
  return bin_dispatch_xr<R, NT, false>(rows, nrows, G, b, i1, i2, i3, amp, xc, acc, gnum, nsm, s);
}

template <typename R>
cudaError_t launch_bin(const int4 *rows, int nrows, const void *G, const BinGeom &b,
                       const R *inv1, const R *inv2, const R *inv3, const double *amp,
                       const double *xcoef, double *acc, double *gnum, int nsm, cudaStream_t s) {
  switch (b.ntr) {
    case 1: return bin_dispatch_smem<R, 1>(rows, nrows, G, b, inv1, inv2, inv3, amp, xcoef, acc, gnum, nsm, s);
    case 2: return bin_dispatch_smem<R, 2>(rows, nrows, G, b, inv1, inv2, inv3, amp, xcoef, acc, gnum, nsm, s);
    case 3: return bin_dispatch_smem<R, 3>(rows, nrows, G, b, inv1, inv2, inv3, amp, xcoef, acc, gnum, nsm, s);
    case 4: return bin_dispatch_smem<R, 4>(rows, nrows, G, b, inv1, inv2, inv3, amp, xcoef, acc, gnum, nsm, s);
    default:
      if (b.ntr > MAX_FAST_T) return cudaErrorInvalidValue;
      return bin_dispatch_smem<R, 0>(rows, nrows, G, b, inv1, inv2, inv3, amp, xcoef, acc, gnum, nsm, s);
  }
}

cudaError_t launch_norms(const int4 *rows, int nrows, const BinGeom &b, const double *amp,
                         const double *xcoef, const double *counts_t, double *den, double *cnt,
                         double *xcnt, int nsm, cudaStream_t s) {
  const size_t sh = (2 * (size_t)b.nq + (b.xrd ? (size_t)b.xbins : 0)) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_norms, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sh);
  if (e != cudaSuccess) return e;
  k_norms<<<nsm * 4, 256, sh, s>>>(rows, nrows, b, amp, xcoef, counts_t, den, cnt, xcnt);
  return cudaGetLastError();
}

template cudaError_t launch_prep<float>(const double *, const uint8_t *, const FrameGeom &, int *,
                                        uint32_t *, uint32_t *, cudaStream_t);
template cudaError_t launch_prep<double>(const double *, const uint8_t *, const FrameGeom &, int *,
                                         uint32_t *, uint32_t *, cudaStream_t);
template cudaError_t launch_scatter<float>(const double *, const uint8_t *, const FrameGeom &,
                                           const uint32_t *, const uint32_t *, const int *,
                                           float *, int32_t *, cudaStream_t);
template cudaError_t launch_scatter<double>(const double *, const uint8_t *, const FrameGeom &,
                                            const uint32_t *, const uint32_t *, const int *,
                                            double *, int32_t *, cudaStream_t);
template cudaError_t launch_spread<float>(const float *, const int *, const FrameGeom &,
                                          const float *, float *, cudaStream_t);
template cudaError_t launch_spread<double>(const double *, const int *, const FrameGeom &,
                                           const double *, double *, cudaStream_t);
template cudaError_t launch_spread_pw<float>(const float *, const int *, const FrameGeom &,
                                             const float *, float *, int, cudaStream_t);
template cudaError_t launch_spread_pw<double>(const double *, const int *, const FrameGeom &,
                                              const double *, double *, int, cudaStream_t);
template cudaError_t launch_bin<float>(const int4 *, int, const void *, const BinGeom &,
                                       const float *, const float *, const float *,
                                       const double *, const double *, double *, double *, int,
                                       cudaStream_t);
template cudaError_t launch_bin<double>(const int4 *, int, const void *, const BinGeom &,
                                        const double *, const double *, const double *,
                                        const double *, const double *, double *, double *, int,
                                        cudaStream_t);

// ---------------------------------------------------------------------------
// Multi-system launches of a batch
// ---------------------------------------------------------------------------
template <typename R>
cudaError_t launch_batch_sort(const BatchSys *sys, int nsys, const BatchPrefix &pre,
                              int64_t natoms, cudaStream_t s) {
  if (nsys < 1 || nsys > MAX_BATCH_SYSTEMS) return cudaErrorInvalidValue;
  k_batch_prep<<<grid_for(natoms, 256), 256, 0, s>>>(sys, nsys, pre.atoms, natoms);
  k_batch_scan<<<nsys, 1024, 0, s>>>(sys);
  k_batch_scatter<R><<<grid_for(natoms, 256), 256, 0, s>>>(sys, nsys, pre.atoms, natoms);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_batch_spread(const BatchSys *sys, int nsys, const BatchPrefix &pre,
                                int nblocks, int chunk, cudaStream_t s) {
  if (nsys < 1 || nblocks < 1) return cudaErrorInvalidValue;
  k_batch_spread<R><<<nblocks, SPREAD_THREADS, spread_smem_bytes(chunk, sizeof(R) == 8), s>>>(
      sys, nsys, pre.spread);
  return cudaGetLastError();
}

template <typename R, int NT>
static cudaError_t batch_bin_nt(const BatchSys *sys, int nsys, const BatchPrefix &pre,
                                int nblocks, bool xray, size_t smem, bool attr_only,
                                cudaStream_t s) {
  if (xray) {
    if (attr_only)
      return cudaFuncSetAttribute(k_batch_bin<R, NT, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_batch_bin<R, NT, true><<<nblocks, 256, smem, s>>>(sys, nsys, pre.bin);
  } else {
    if (attr_only)
      return cudaFuncSetAttribute(k_batch_bin<R, NT, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_batch_bin<R, NT, false><<<nblocks, 256, smem, s>>>(sys, nsys, pre.bin);
  }
  return cudaGetLastError();
}

// attr_only: set the kernel's shared-memory limit (before any capture), launch nothing.
template <typename R>
static cudaError_t batch_bin(const BatchSys *sys, int nsys, const BatchPrefix &pre, int nblocks,
                             int ntr, bool xray, int hist_max, bool attr_only, cudaStream_t s) {
  const size_t smem = (size_t)hist_max * sizeof(double);
  if (smem > 160 * 1024 || ntr < 1 || ntr > MAX_FAST_T) return cudaErrorInvalidValue;
  switch (ntr) {
    case 1: return batch_bin_nt<R, 1>(sys, nsys, pre, nblocks, xray, smem, attr_only, s);
    case 2: return batch_bin_nt<R, 2>(sys, nsys, pre, nblocks, xray, smem, attr_only, s);
    case 3: return batch_bin_nt<R, 3>(sys, nsys, pre, nblocks, xray, smem, attr_only, s);
    case 4: return batch_bin_nt<R, 4>(sys, nsys, pre, nblocks, xray, smem, attr_only, s);
    default: return batch_bin_nt<R, 0>(sys, nsys, pre, nblocks, xray, smem, attr_only, s);
  }
}

template <typename R>
cudaError_t launch_batch_bin(const BatchSys *sys, int nsys, const BatchPrefix &pre, int nblocks,
                             int ntr, bool xray, int hist_max, cudaStream_t s) {
  return batch_bin<R>(sys, nsys, pre, nblocks, ntr, xray, hist_max, false, s);
}

template <typename R>
cudaError_t batch_set_attributes(int ntr, bool xray, int hist_max) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = smem_optin(k_batch_spread<R>, optin);
  BatchPrefix none{};
  if (e == cudaSuccess) e = batch_bin<R>(nullptr, 0, none, 0, ntr, xray, hist_max, true, nullptr);
  return e;
}

template cudaError_t launch_batch_sort<float>(const BatchSys *, int, const BatchPrefix &, int64_t,
                                              cudaStream_t);
template cudaError_t launch_batch_sort<double>(const BatchSys *, int, const BatchPrefix &,
                                               int64_t, cudaStream_t);
template cudaError_t launch_batch_spread<float>(const BatchSys *, int, const BatchPrefix &, int,
                                                int, cudaStream_t);
template cudaError_t launch_batch_spread<double>(const BatchSys *, int, const BatchPrefix &, int,
                                                 int, cudaStream_t);
template cudaError_t launch_batch_bin<float>(const BatchSys *, int, const BatchPrefix &, int, int,
                                             bool, int, cudaStream_t);
template cudaError_t launch_batch_bin<double>(const BatchSys *, int, const BatchPrefix &, int,
                                              int, bool, int, cudaStream_t);
template cudaError_t batch_set_attributes<float>(int, bool, int);
template cudaError_t batch_set_attributes<double>(int, bool, int);

}  // namespace sqn
