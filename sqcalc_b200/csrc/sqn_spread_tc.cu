// Gather spreading on the tensor cores (FP32 plans, sm_100a tcgen05).
//
// A 32 x 16 x 8 tile of one transform is a sum of outer products over the
// points that reach it: grid[x][y][z] = sum_p kx_p[x] (ky_p[y] kz_p[z] c_p).
// With M = (y, z) (128 cells), N = x (32 cells) and K = points, that is one
// GEMM per tile and transform: D[m][n] += A[m][k] B[n][k] with
// A[(y, z)][p] = ky_p[y] kz_p[z] c_p and B[x][p] = kx_p[x].  The CTA stages the
// points exactly as k_spread does (bin lists, candidates, counting sort by
// transform, ES kernel rows shifted onto the tile), then forms A and B for
// eight points at a time in shared memory (K-major, no swizzle) and one
// thread issues tcgen05.mma kind::tf32 (M 128, N 32, K 8) into the
// transform's accumulator in tensor memory (32 columns per transform).  FP32
// accuracy from three TF32 products per step (hi*hi + hi*lo + lo*hi, with
// a = hi + lo, hi the TF32 rounding of a): the dropped lo*lo term and the
// truncation of the lo parts leave ~2^-21 relative per product.  The
// epilogue reads each row (y, z) of the accumulators with tcgen05.ld and
// writes the tile's 32 x cells of it.  Every wait on the MMA barrier is
// bounded: past the limit the kernel records the failure in *err and goes on.
#include <cstdint>
#include <cuda_runtime.h>

#include "sqn_device.cuh"
#include "sqn_internal.h"

namespace sqn {
namespace {

using namespace dev;

constexpr int TC_GROUP = 2;               // K-steps (8 points each) formed per barrier
constexpr int A_BYTES = 128 * 8 * 4;      // one K-step of A (128 rows x 8 tf32)
constexpr int B_BYTES = 32 * 8 * 4;       // one K-step of B (32 rows x 8 tf32)
constexpr int BUF_BYTES = TC_GROUP * 2 * (A_BYTES + B_BYTES);  // one group, hi and lo
constexpr int OPS_BYTES = 2 * BUF_BYTES;  // two groups: one formed while the other multiplies
constexpr uint32_t LBO = 128, SBO = 256;  // K-major core-matrix strides (bytes)
constexpr int FORMER_WARPS = SPREAD_WARPS - 1;  // warp 15 issues the MMAs

// Byte offset of element (row r, k) of a K-major operand step: 8-row groups of
// 16-byte rows (core matrices), the two K halves LBO apart, groups SBO apart.
__device__ __forceinline__ uint32_t kmaj_off(int r, int k) {
  return (uint32_t)((r & 7) * 16 + (r >> 3) * SBO + (k & 3) * 4 + (k >> 2) * LBO);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(LBO >> 4) << 16) |
         ((uint64_t)(SBO >> 4) << 32) | (1ull << 46);
}

// kind::tf32, D F32, A and B TF32 K-major, N = 32, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) |
                           ((128u >> 4) << 24);

__device__ __forceinline__ float to_tf32(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

// Wait for phase `parity` of the barrier, at most ~2^22 polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// One row (32 columns) of the accumulator: lane base + laneid of this warp's
// quarter, columns col .. col + 31.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

template <int NT>
__global__ void __launch_bounds__(SPREAD_THREADS, 2)
    k_spread_tc(const float *__restrict__ recs, const int *__restrict__ starts, FrameGeom g,
                const float *__restrict__ strength, float *__restrict__ grid,
                int *__restrict__ err) {
  constexpr int TCOLS = NT == 1 ? 32 : (NT == 2 ? 64 : 128);  // TMEM columns (power of 2)
  const int chunk = g.chunk;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *s_rows = reinterpret_cast<float *>(smem_raw + OPS_BYTES);  // [chunk][SPREAD_ROW]
  float *s_off = s_rows + (size_t)chunk * SPREAD_ROW;              // [chunk][4]
  int4 *s_meta = reinterpret_cast<int4 *>(s_off + (size_t)chunk * 4);  // [chunk]
  __shared__ int s_bstart[MAX_NB];
  __shared__ int s_bpref[MAX_NB + 1];
  __shared__ int s_borg[MAX_NB][3];
  __shared__ int s_wcount[MAX_FAST_T * SPREAD_WARPS];
  __shared__ int s_bl[3][MAX_BINS_DIM];
  __shared__ int s_nbl[3];
  // per operand buffer: `full` (the formers' arrivals) and `empty` (the MMA commit)
  __shared__ __align__(8) uint64_t s_full[2], s_empty[2];
  __shared__ int s_step[64];   // K-step table: transform << 16 | step within it
  __shared__ int s_tp0[MAX_FAST_T + 1];  // the transforms' point ranges in the chunk
  __shared__ int s_nsteps;
  __shared__ uint32_t s_tmem;
  __shared__ int s_touched[MAX_FAST_T];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int t0 = tile % g.ntile[0];
  const int t1 = (tile / g.ntile[0]) % g.ntile[1];
  const int t2 = tile / (g.ntile[0] * g.ntile[1]);
  const int X0 = t0 * g.tile[0], Y0 = t1 * g.tile[1], Z0 = t2 * g.tile[2];
  const int tx = min(g.tile[0], g.nf[0] - X0);
  const int ty = min(g.tile[1], g.nf[1] - Y0);
  const int tz = min(g.tile[2], g.nf[2] - Z0);
  const int w = g.w;
  const uint32_t full0 = smem_u32(&s_full[0]), full1 = smem_u32(&s_full[1]);
  const uint32_t empty0 = smem_u32(&s_empty[0]), empty1 = smem_u32(&s_empty[1]);

  // tensor memory for the accumulators, the MMA barrier
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(full0), "r"(32 * FORMER_WARPS) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(full1), "r"(32 * FORMER_WARPS) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < MAX_FAST_T) s_touched[tid] = 0;

  // bins whose points can reach this tile (as k_spread)
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
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int nb0 = s_nbl[0], nb1 = s_nbl[1];
  const int nb = nb0 * nb1 * s_nbl[2];
  if (warp == 0) {
    int cnt2[2];
    int sum = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int b = 2 * lane + h;
      cnt2[h] = 0;
      if (b < nb) {
        const int bx = s_bl[0][b % nb0], by = s_bl[1][(b / nb0) % nb1],
                  bz = s_bl[2][b / (nb0 * nb1)];
        const int key = (bz * g.ntile[1] + by) * g.ntile[0] + bx;
        const int st = starts[key];
        cnt2[h] = starts[key + 1] - st;
        s_bstart[b] = st;
        s_borg[b][0] = bx * g.tile[0];
        s_borg[b][1] = by * g.tile[1];
        s_borg[b][2] = bz * g.tile[2];
      }
      sum += cnt2[h];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const int excl = incl - sum;
    if (2 * lane < nb + 1) s_bpref[2 * lane] = excl;
    if (2 * lane + 1 < nb + 1) s_bpref[2 * lane + 1] = excl + cnt2[0];
    if (lane == 31 && nb == MAX_NB) s_bpref[MAX_NB] = incl;
  }
  __syncthreads();
  const int total = s_bpref[nb];
  const float halfw = 0.5f * (float)w - 0.5f;
  const float c2 = 4.0f / ((float)w * (float)w);
  const float beta = (float)g.beta;

  int gbase = 0;  // groups so far: group g uses buffer g & 1 for the (g >> 1)-th time
  bool started[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) started[t] = false;  // used by the issuing thread

  for (int base = 0; base < total; base += chunk) {
    // 1. candidates that overlap the tile, counting-sorted by transform
    const int i = base + tid;
    bool keep = false;
    int4 meta = make_int4(0, 0, 0, 0);
    float rec[REC_SLOTS];
    if (tid < chunk && i < total) {
      int b = 0;
      while (i >= s_bpref[b + 1]) ++b;
      const int ridx = s_bstart[b] + (i - s_bpref[b]);
      load_rec(recs + (int64_t)ridx * REC_SLOTS, rec);
      const uint32_t packed = unpack_rec<float>(rec[0]);
      int rx = s_borg[b][0] + (int)(packed & 255u) - X0;
      int ry = s_borg[b][1] + (int)((packed >> 8) & 255u) - Y0;
      int rz = s_borg[b][2] + (int)((packed >> 16) & 255u) - Z0;
      if (rx < 0) rx += g.nf[0];
      if (ry < 0) ry += g.nf[1];
      if (rz < 0) rz += g.nf[2];
      keep = (rx < tx || rx + w > g.nf[0]) && (ry < ty || ry + w > g.nf[1]) &&
             (rz < tz || rz + w > g.nf[2]);
      meta = make_int4(rx, ry, rz, (int)(packed >> 24));
    }
    const int my_t = NT > 1 ? meta.w : 0;
    unsigned my_bal = 0u;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const unsigned bt = __ballot_sync(FULL, keep && my_t == t);
      if (lane == 0) s_wcount[t * SPREAD_WARPS + warp] = __popc(bt);
      if (t == my_t) my_bal = bt;
    }
    __syncthreads();
    int tstart[NT + 1];
    tstart[0] = 0;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      int tot = 0;
#pragma unroll
      for (int k = 0; k < SPREAD_WARPS; ++k) tot += s_wcount[t * SPREAD_WARPS + k];
      tstart[t + 1] = tstart[t] + tot;
    }
    const int npts = tstart[NT];
    if (keep) {
      int p = __popc(my_bal & ((1u << lane) - 1u));
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (t == my_t) p += tstart[t];
      for (int k = 0; k < warp; ++k) p += s_wcount[my_t * SPREAD_WARPS + k];
      s_meta[p] = meta;
      store_rec(s_off + (size_t)p * 4, 0.0f, rec[1], rec[2], rec[3]);
    }
    __syncthreads();

    // K-step table of this chunk (read after the barrier that ends the rows)
    if (tid == 0) {
      int ks[NT], kmax = 0, n = 0;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        ks[t] = (tstart[t + 1] - tstart[t] + 7) / 8;
        kmax = max(kmax, ks[t]);
        s_tp0[t] = tstart[t];
      }
      s_tp0[NT] = tstart[NT];
      for (int r = 0; r < kmax; ++r)
#pragma unroll
        for (int t = 0; t < NT; ++t)
          if (r < ks[t] && n < 64) s_step[n++] = (t << 16) | r;
      s_nsteps = n;
    }
    // 2. kernel rows shifted onto the tile's cells (x 32, y 16, z 8 times the
    //    strength), zero outside the support or the grid
    for (int e = tid; e < 3 * npts; e += SPREAD_THREADS) {
      const int d = e >= 2 * npts ? 2 : (e >= npts ? 1 : 0);
      const int p = e - d * npts;
      const int4 m = s_meta[p];
      const int rel = d == 0 ? m.x : (d == 1 ? m.y : m.z);
      const int len = d == 0 ? TILE_X : (d == 1 ? TILE_Y : TILE_Z);
      const int lim = d == 0 ? tx : (d == 1 ? ty : tz);
      const int n = g.nf[d];
      const float off = s_off[(size_t)p * 4 + 1 + d];
      const float sc = d == 2 ? strength[m.w] : 1.0f;
      float *row = s_rows + (size_t)p * SPREAD_ROW + (d == 0 ? 0 : (d == 1 ? TILE_X : TILE_X + TILE_Y));
      for (int j = 0; j < len; j += 4) store_rec(row + j, 0.0f, 0.0f, 0.0f, 0.0f);
      for (int k = 0; k < w; ++k) {
        int cell = rel + k;
        if (cell >= n) cell -= n;
        const float v = es_at(k, off, halfw, c2, beta) * sc;
        if (cell < lim) row[cell] = v;
      }
    }
    __syncthreads();

    // 3. K-steps of eight points of one transform, interleaved across the
    //    transforms (consecutive MMAs go to different accumulators), in groups of
    //    TC_GROUP.  Warps 0..14 form the operands of a group into one of two
    //    buffers and arrive on its `full` barrier; warp 15 waits for it, issues
    //    the group's MMAs and commits them to the buffer's `empty` barrier, which
    //    the formers wait for before they refill that buffer.
    const int nsteps = s_nsteps;
    const int ngroups = (nsteps + TC_GROUP - 1) / TC_GROUP;
    if (warp < FORMER_WARPS) {
      for (int gi = 0; gi < ngroups; ++gi) {
        const int gg = gbase + gi, bsel = gg & 1, use = gg >> 1;
        unsigned char *ops = smem_raw + bsel * BUF_BYTES;
        if (use > 0) {
          bool ok = true;
          if (lane == 0) ok = mbar_wait(bsel ? empty1 : empty0, (uint32_t)(use - 1) & 1u);
          __syncwarp();
          if (!ok) atomicExch(err, 1);
        }
        if (tid < 128 * TC_GROUP) {
          // A: thread -> (row m = (y, z), step j)
          const int m = tid & 127, j = tid >> 7, sidx = gi * TC_GROUP + j;
          if (sidx < nsteps) {
            const int st = s_step[sidx], t = st >> 16;
            const int p0 = s_tp0[t] + 8 * (st & 0xFFFF), pend = s_tp0[t + 1];
            const int y = m >> 3, z = m & 7;
            unsigned char *ah = ops + j * A_BYTES;
            unsigned char *al = ops + TC_GROUP * A_BYTES + j * A_BYTES;
            float hi[8], lo[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const int pp = p0 + k;
              float a = 0.0f;
              if (pp < pend) {
                const float *row = s_rows + (size_t)pp * SPREAD_ROW;
                a = row[TILE_X + y] * row[TILE_X + TILE_Y + z];
              }
              hi[k] = to_tf32(a);
              lo[k] = to_tf32(a - hi[k]);
            }
            *reinterpret_cast<float4 *>(ah + kmaj_off(m, 0)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4 *>(ah + kmaj_off(m, 4)) = make_float4(hi[4], hi[5], hi[6], hi[7]);
            *reinterpret_cast<float4 *>(al + kmaj_off(m, 0)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            *reinterpret_cast<float4 *>(al + kmaj_off(m, 4)) = make_float4(lo[4], lo[5], lo[6], lo[7]);
          }
        } else if (tid < 128 * TC_GROUP + 32 * TC_GROUP) {
          // B: thread -> (row n = x, step j)
          const int q = tid - 128 * TC_GROUP;
          const int n = q & 31, j = q >> 5, sidx = gi * TC_GROUP + j;
          if (sidx < nsteps) {
            const int st = s_step[sidx], t = st >> 16;
            const int p0 = s_tp0[t] + 8 * (st & 0xFFFF), pend = s_tp0[t + 1];
            unsigned char *bh = ops + 2 * TC_GROUP * A_BYTES + j * B_BYTES;
            unsigned char *bl = ops + 2 * TC_GROUP * A_BYTES + TC_GROUP * B_BYTES + j * B_BYTES;
            float hi[8], lo[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const int pp = p0 + k;
              const float b = pp < pend ? s_rows[(size_t)pp * SPREAD_ROW + n] : 0.0f;
              hi[k] = to_tf32(b);
              lo[k] = to_tf32(b - hi[k]);
            }
            *reinterpret_cast<float4 *>(bh + kmaj_off(n, 0)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4 *>(bh + kmaj_off(n, 4)) = make_float4(hi[4], hi[5], hi[6], hi[7]);
            *reinterpret_cast<float4 *>(bl + kmaj_off(n, 0)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            *reinterpret_cast<float4 *>(bl + kmaj_off(n, 4)) = make_float4(lo[4], lo[5], lo[6], lo[7]);
          }
        }
        // this thread's generic-proxy writes -> the tensor core's reads; then
        // every former thread arrives on the buffer's `full` barrier
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(bsel ? full1 : full0);
      }
    } else {
      for (int gi = 0; gi < ngroups; ++gi) {
        const int gg = gbase + gi, bsel = gg & 1, use = gg >> 1;
        bool ok = true;
        if (lane == 0) ok = mbar_wait(bsel ? full1 : full0, (uint32_t)use & 1u);
        __syncwarp();
        if (lane == 0) {
          if (!ok) atomicExch(err, 1);
          tc_fence_after();
          const uint32_t obase = smem_u32(smem_raw + bsel * BUF_BYTES);
          for (int j = 0; j < TC_GROUP; ++j) {
            const int sidx = gi * TC_GROUP + j;
            if (sidx >= nsteps) break;
            const int t = s_step[sidx] >> 16;
            const uint32_t ah = obase + j * A_BYTES, al = obase + (TC_GROUP + j) * A_BYTES;
            const uint32_t bh = obase + 2 * TC_GROUP * A_BYTES + j * B_BYTES;
            const uint32_t bl = bh + TC_GROUP * B_BYTES;
            const uint32_t d = tmem + 32u * (uint32_t)t;
            bool stt = false;
#pragma unroll
            for (int u = 0; u < NT; ++u)
              if (u == t) stt = started[u];
            mma_tf32(d, smem_desc(ah), smem_desc(bh), stt ? 1u : 0u);
            mma_tf32(d, smem_desc(ah), smem_desc(bl), 1u);
            mma_tf32(d, smem_desc(al), smem_desc(bh), 1u);
#pragma unroll
            for (int u = 0; u < NT; ++u)
              if (u == t) started[u] = true;
            s_touched[t] = 1;
          }
          mma_commit(bsel ? empty1 : empty0);
        }
        __syncwarp();
      }
    }
    gbase += ngroups;
    // the next chunk rewrites s_meta, s_off, s_rows and the step table, which
    // the MMAs do not read
    __syncthreads();
  }

  // 4. the last groups' MMAs done (the last use of each buffer), each row
  //    (y, z) of each transform out
  {
    const int uses0 = (gbase + 1) / 2, uses1 = gbase / 2;
    bool ok = true;
    if (uses0 > 0) ok = mbar_wait(empty0, (uint32_t)(uses0 - 1) & 1u) && ok;
    if (uses1 > 0) ok = mbar_wait(empty1, (uint32_t)(uses1 - 1) & 1u) && ok;
    if (!ok && tid == 0) atomicExch(err, 1);
  }
  tc_fence_after();
  __syncthreads();
  if (warp < 4 * NT) {
    const int t = warp >> 2, qtr = warp & 3;
    float v[32];
    tmem_ld32(tmem + ((uint32_t)(32 * qtr) << 16) + 32u * (uint32_t)t, v);
    const bool touched = s_touched[t] != 0;
    const int m = 32 * qtr + lane, y = m >> 3, z = m & 7;
    if (y < ty && z < tz) {
      float *out = grid + (int64_t)t * g.vol_real + ((int64_t)(Z0 + z) * g.nf[1] + (Y0 + y)) * g.pitch + X0;
      if (tx == 32 && (g.pitch & 3) == 0) {
#pragma unroll
        for (int c = 0; c < 32; c += 4)
          *reinterpret_cast<float4 *>(out + c) = touched ? make_float4(v[c], v[c + 1], v[c + 2], v[c + 3])
                                                        : make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (c < tx) out[c] = touched ? v[c] : 0.0f;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS)
                 : "memory");
  }
}

}  // namespace

// Points per chunk for the tensor-core spread: two CTAs per SM with the
// operand buffers next to the staged points.
int spread_tc_chunk() {
  const size_t per_point = SPREAD_ROW * 4 + 16 + 16;  // row, offsets, meta
  const size_t budget = 106 * 1024 - OPS_BYTES;
  int c = (int)(budget / per_point);
  c = c > SPREAD_THREADS ? SPREAD_THREADS : c;
  return c / 32 * 32;
}

size_t spread_tc_smem(int chunk) {
  return OPS_BYTES + (size_t)chunk * (SPREAD_ROW * 4 + 16 + 16);
}

cudaError_t spread_tc_set_attributes() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  const int dyn = (int)spread_tc_smem(spread_tc_chunk());
  e = cudaFuncSetAttribute(k_spread_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_spread_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_spread_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_spread_tc<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  return e;
}

cudaError_t launch_spread_tc(const float *recs, const int *starts, const FrameGeom &g,
                             const float *strength, float *grid, int *err, cudaStream_t s) {
  const dim3 grd((unsigned)g.ntiles);
  const size_t sm = spread_tc_smem(g.chunk);
  switch (g.ntr) {
    case 1: k_spread_tc<1><<<grd, SPREAD_THREADS, sm, s>>>(recs, starts, g, strength, grid, err); break;
    case 2: k_spread_tc<2><<<grd, SPREAD_THREADS, sm, s>>>(recs, starts, g, strength, grid, err); break;
    case 3: k_spread_tc<3><<<grd, SPREAD_THREADS, sm, s>>>(recs, starts, g, strength, grid, err); break;
    case 4: k_spread_tc<4><<<grd, SPREAD_THREADS, sm, s>>>(recs, starts, g, strength, grid, err); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace sqn
