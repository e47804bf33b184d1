// sqn_spread_frame_noalloc: the wrap + bin-sort + spread stage of one frame,
// for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- a host
// framework that owns all device memory through its own pool and forbids
// side allocations (custom operators of ML frameworks, plugins inside a host
// application that has already reserved the device memory), or a
// long-running service that must keep a fixed footprint and cannot risk an
// allocation failing in the middle of a request.  Such a caller brings its
// own positions and output grids; the scratch this stage needs (bin counts,
// bin starts, per-atom keys and slots, sorted point records, species and
// strengths) lives in one file-scope __device__ array of fixed size instead of
// being allocated.
//
// Contract (see include/sqnufft.h):
//   * The array is SQN_NOALLOC_SCRATCH_BYTES (32 MiB) per GPU.  Every GPU that
//     loads this library reserves it for the life of the process.
//   * The first call on a device looks up the array's device address with that
//     device current (cudaGetSymbolAddress) and sets the spread kernel's shared
//     memory limit; make that first call before any stream capture.
//   * All calls share the one array and it keeps the last call's contents; the
//     bin counts are cleared at the start of every call.  Two calls whose work
//     overlaps on the GPU (different streams, or different host threads on the
//     same device) race on the array and must be serialised by the caller.
//   * Requests whose scratch would not fit are rejected with
//     SQN_ERR_SCRATCH_LIMIT, and more than MAX_FAST_T (8) grids with
//     SQN_ERR_INVALID_ARGUMENT, before anything is queued.
//   * species and strength are host arrays: the call checks every species
//     index on the host and copies both with cudaMemcpyAsync on `stream`.
//   * No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/sqnufft.h"
#include "sqn_internal.h"

using namespace sqn;

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SQN_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Device address of the scratch array on the current device (set up once).
int scratch_for_current_device(unsigned char **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return SQN_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return SQN_ERR_CUDA;
    }
    if (spread_set_attributes() != cudaSuccess) {
      cudaGetLastError();
      return SQN_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return SQN_OK;
}

}  // namespace

extern "C" int sqn_spread_frame_noalloc(const double *pos, int64_t natoms,
                                        const uint8_t *species, int32_t ntr,
                                        const float *strength, const double *cell,
                                        const double *origin, const int64_t *nf,
                                        int32_t kernel_width, double beta, float *grid,
                                        void *stream) {
  if (!pos || !species || !strength || !cell || !origin || !nf || !grid)
    return SQN_ERR_INVALID_ARGUMENT;
  if (natoms < 1 || natoms > (int64_t)INT32_MAX / 2) return SQN_ERR_NUM_NU_PTS_INVALID;
  if (ntr < 1 || ntr > MAX_FAST_T) return SQN_ERR_INVALID_ARGUMENT;
  const int w = kernel_width;
  if (w < 2 || w > MAX_W || !(beta > 0.0)) return SQN_ERR_INVALID_ARGUMENT;
  for (int d = 0; d < 3; ++d)
    if (nf[d] < 2 * w || nf[d] > 65536) return SQN_ERR_INVALID_ARGUMENT;
  // Species index every atom on the host: it selects a bin and a grid, so an
  // out-of-range value must never reach the kernels.
  for (int64_t i = 0; i < natoms; ++i)
    if (species[i] >= ntr) return SQN_ERR_INVALID_ARGUMENT;

  // Geometry, as the plan sets it up for the same fine grid and kernel.
  FrameGeom g{};
  const double a[9] = {cell[0], cell[1], cell[2], cell[3], cell[4], cell[5], cell[6], cell[7], cell[8]};
  auto M = [&a](int r, int c) { return a[3 * (c - 1) + (r - 1)]; };
  const double det = M(1, 1) * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)) -
                     M(1, 2) * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1)) +
                     M(1, 3) * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
  if (det == 0.0 || !std::isfinite(det)) return SQN_ERR_DEGENERATE_CELL;
  double inv[9];
  auto I = [&inv](int r, int c) -> double & { return inv[3 * (c - 1) + (r - 1)]; };
  I(1, 1) = (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2));
  I(2, 1) = -(M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1));
  I(3, 1) = (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
  I(1, 2) = -(M(1, 2) * M(3, 3) - M(1, 3) * M(3, 2));
  I(2, 2) = (M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1));
  I(3, 2) = -(M(1, 1) * M(3, 2) - M(1, 2) * M(3, 1));
  I(1, 3) = (M(1, 2) * M(2, 3) - M(1, 3) * M(2, 2));
  I(2, 3) = -(M(1, 1) * M(2, 3) - M(1, 3) * M(2, 1));
  I(3, 3) = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1));
  for (int k = 0; k < 9; ++k) g.inv[k] = inv[k] / det;
  std::memcpy(g.origin, origin, sizeof(g.origin));
  // the same spread tiles a plan of this grid uses (they depend on the SM count)
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_NO_DEVICE;
  }
  const int tmax[3] = {TILE_X, TILE_Y, spread_tile_z(nf, ntr, nsm)};
  for (int d = 0; d < 3; ++d) {
    g.nf[d] = (int)nf[d];
    g.tile[d] = (int)(nf[d] < tmax[d] ? nf[d] : tmax[d]);
    g.ntile[d] = (int)((nf[d] + g.tile[d] - 1) / g.tile[d]);
  }
  g.w = w;
  g.beta = beta;
  g.ntr = ntr;
  g.ntiles = g.ntile[0] * g.ntile[1] * g.ntile[2];
  g.pitch = nf[0];
  g.vol_real = nf[0] * nf[1] * nf[2];
  g.natoms = natoms;
  g.rec_stride = rec_stride(w, false);
  g.chunk = spread_chunk(false);
  const int64_t nkeys = spread_nkeys(g);  // one bin per (grid, tile)
  if (nkeys >= INT32_MAX) return SQN_ERR_SCRATCH_LIMIT;

  // Scratch layout inside the static array, each section 256-byte aligned.
  const size_t o_counts = 0;
  const size_t o_starts = o_counts + align256(sizeof(int) * (size_t)nkeys);
  const size_t o_key = o_starts + align256(sizeof(int) * (size_t)(nkeys + 1));
  const size_t o_slot = o_key + align256(sizeof(uint32_t) * (size_t)natoms);
  const size_t o_recs = o_slot + align256(sizeof(uint32_t) * (size_t)natoms);
  const size_t o_species = o_recs + align256(sizeof(float) * (size_t)g.rec_stride * (size_t)natoms);
  const size_t o_strength = o_species + align256((size_t)natoms);
  const size_t total = o_strength + align256(sizeof(float) * (size_t)ntr);
  if (total > (size_t)SQN_NOALLOC_SCRATCH_BYTES) return SQN_ERR_SCRATCH_LIMIT;

  unsigned char *base = nullptr;
  int st = scratch_for_current_device(&base);
  if (st != SQN_OK) return st;
  int *counts = reinterpret_cast<int *>(base + o_counts);
  int *starts = reinterpret_cast<int *>(base + o_starts);
  uint32_t *key = reinterpret_cast<uint32_t *>(base + o_key);
  uint32_t *slot = reinterpret_cast<uint32_t *>(base + o_slot);
  float *recs = reinterpret_cast<float *>(base + o_recs);
  uint8_t *d_species = base + o_species;
  float *d_strength = reinterpret_cast<float *>(base + o_strength);

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The bin counts must start at zero; the array keeps whatever the previous
  // call (or an aborted one) left there.
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nkeys, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_species, species, (size_t)natoms, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_strength, strength, sizeof(float) * (size_t)ntr, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_prep<float>(pos, d_species, g, counts, key, slot, s);
  if (e == cudaSuccess) e = launch_scan(counts, starts, (int)nkeys, s);
  if (e == cudaSuccess) e = launch_scatter<float>(pos, d_species, g, key, slot, starts, recs, nullptr, s);
  if (e == cudaSuccess) e = launch_spread<float>(recs, starts, g, d_strength, grid, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_CUDA;
  }
  return SQN_OK;
}
