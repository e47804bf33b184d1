// cuFINUFFT-shaped type-1 3D NUFFT on this library's kernels.
//
//   fk[t][k] = sum_j c[t][j] exp(iflag i (k1 x_j + k2 y_j + k3 z_j)),
//   k_d in [-N_d/2, (N_d - 1)/2]
//
// with the plan / setpts / execute / destroy life cycle and argument meaning of
// cufinufft[f]_makeplan / setpts / execute / destroy for type 1, dim 3
// (external/finufft/include/cufinufft.h; sqcalc binds them in
// src/sqc_cufinufft.f90:183-259 and calls them from src/sqc_gpu.f90:108-362),
// so that the library can stand in for those calls literally.  The points are
// periodic coordinates (any real value, period 2 pi); the strengths are complex.
//
// B200 form: setpts wraps and bin-sorts the points once (k_prep, k_scan,
// k_scatter with the sorted-to-original index); execute spreads the real and
// the imaginary parts of every transform as separate real grids with
// per-point weights (k_spread), runs one batched cuFFT R2C over them, and
// k_type1_out assembles each requested mode from the two half spectra
// (G(-k) = conj G(k) for a real grid), applies the (-1)^(k1+k2+k3) phase of the
// [-pi, pi) coordinates and the deconvolution 1 / (phihat1 phihat2 phihat3),
// and writes the modes in the requested order (modeord 0: -N/2 first,
// modeord 1: 0 first, as cuFINUFFT).
#include <cufft.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/sqnufft.h"
#include "sqn_device.cuh"
#include "sqn_internal.h"

using namespace sqn;

struct sqn_type1_s {
  int device = 0;
  bool fp64 = true;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int iflag = 1, ntr = 1, modeord = 0;
  int64_t N[3] = {0, 0, 0};
  int w = 0;
  double beta = 0.0, sigma = 0.0;
  int64_t nf[3] = {0, 0, 0};
  FrameGeom g{};
  int64_t M = 0, Mcap = 0;
  double *d_pos = nullptr;
  uint8_t *d_species = nullptr;
  int *d_counts = nullptr, *d_starts = nullptr;
  uint32_t *d_key = nullptr, *d_slot = nullptr;
  int32_t *d_orig = nullptr;
  void *d_recs = nullptr, *d_w = nullptr;
  void *d_grid = nullptr, *d_G = nullptr;
  void *d_inv[3] = {nullptr, nullptr, nullptr};
  cufftHandle fft = 0;
  bool fft_ok = false;
  std::vector<void *> fixed, perpts;  // allocations of makeplan / of setpts
};

namespace {

using namespace dev;

template <typename R>
__global__ void k_pack_points(const R *__restrict__ x, const R *__restrict__ y,
                              const R *__restrict__ z, int64_t M, double *__restrict__ pos) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < M;
       j += (int64_t)gridDim.x * blockDim.x) {
    pos[3 * j + 0] = (double)x[j];
    pos[3 * j + 1] = (double)y[j];
    pos[3 * j + 2] = (double)z[j];
  }
}

// Sorted weights: w[2t][p] = Re c[t][orig[p]], w[2t+1][p] = Im c[t][orig[p]].
template <typename R>
__global__ void k_sorted_weights(const R *__restrict__ c, const int32_t *__restrict__ orig,
                                 int64_t M, int ntr, R *__restrict__ w) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < M;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = orig[p];
    for (int t = 0; t < ntr; ++t) {
      w[(2 * t) * M + p] = c[2 * (t * M + j)];
      w[(2 * t + 1) * M + p] = c[2 * (t * M + j) + 1];
    }
  }
}

__device__ __forceinline__ int64_t wrap_index(int64_t k, int64_t n) { return k >= 0 ? k : n + k; }

template <typename R>
__global__ void k_type1_out(const typename Cplx<R>::T *__restrict__ G, int ntr, int64_t N1,
                            int64_t N2, int64_t N3, int64_t nf0, int64_t nf1, int64_t nf2,
                            int iflag, int modeord, const R *__restrict__ inv1,
                            const R *__restrict__ inv2, const R *__restrict__ inv3,
                            R *__restrict__ fk) {
  using C = typename Cplx<R>::T;
  const int64_t c1 = nf0 / 2 + 1;
  const int64_t volc = c1 * nf1 * nf2;
  const int64_t nm = N1 * N2 * N3;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nm * ntr;
       m += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(m / nm);
    int64_t r = m - (int64_t)t * nm;
    const int64_t i1 = r % N1;
    r /= N1;
    const int64_t i2 = r % N2, i3 = r / N2;
    int64_t k1, k2, k3;
    if (modeord == 0) {
      k1 = i1 - N1 / 2;
      k2 = i2 - N2 / 2;
      k3 = i3 - N3 / 2;
    } else {
      k1 = i1 < (N1 + 1) / 2 ? i1 : i1 - N1;
      k2 = i2 < (N2 + 1) / 2 ? i2 : i2 - N2;
      k3 = i3 < (N3 + 1) / 2 ? i3 : i3 - N3;
    }
    // the forward FFT gives sum exp(-2 pi i k.s); iflag > 0 reads the mirror mode
    int64_t q1 = iflag > 0 ? -k1 : k1, q2 = iflag > 0 ? -k2 : k2, q3 = iflag > 0 ? -k3 : k3;
    bool conj = false;
    if (q1 < 0) {
      q1 = -q1;
      q2 = -q2;
      q3 = -q3;
      conj = true;
    }
    const int64_t idx = (wrap_index(q3, nf2) * nf1 + wrap_index(q2, nf1)) * c1 + q1;
    C gr = G[(int64_t)(2 * t) * volc + idx], gi = G[(int64_t)(2 * t + 1) * volc + idx];
    if (conj) {
      gr.y = -gr.y;
      gi.y = -gi.y;
    }
    // Re + i Im of the complex strengths: (gr.x - gi.y) + i (gr.y + gi.x)
    R fre = gr.x - gi.y, fim = gr.y + gi.x;
    const R dec = inv1[k1 >= 0 ? k1 : -k1] * inv2[k2 >= 0 ? k2 : -k2] * inv3[k3 >= 0 ? k3 : -k3];
    const R sgn = ((k1 + k2 + k3) & 1) ? R(-1) : R(1);
    fk[2 * m] = sgn * dec * fre;
    fk[2 * m + 1] = sgn * dec * fim;
  }
}

unsigned grid1d(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)b;
}

template <typename T> int talloc(std::vector<void *> &list, T **ptr, size_t count) {
  *ptr = nullptr;
  void *v = nullptr;
  if (cudaMalloc(&v, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_ALLOC;
  }
  list.push_back(v);
  *ptr = static_cast<T *>(v);
  return SQN_OK;
}

void free_list(std::vector<void *> &list) {
  for (void *v : list) cudaFree(v);
  list.clear();
}

void free_type1(sqn_type1_plan *p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->fft_ok) cufftDestroy(p->fft);
  free_list(p->perpts);
  free_list(p->fixed);
  if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

int make_type1(int type, int dim, const int64_t *n_modes, int iflag, int ntransf, double tol,
               sqn_type1_plan **out, const sqn_type1_opts *opts, bool fp64) {
  if (!out) return SQN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (type != 1 || dim != 3) return SQN_ERR_NOT_SUPPORTED;
  if (!n_modes || ntransf < 1 || ntransf > 64 || !(tol > 0.0)) return SQN_ERR_INVALID_ARGUMENT;
  for (int d = 0; d < 3; ++d)
    if (n_modes[d] < 1 || n_modes[d] > (1 << 20)) return SQN_ERR_INVALID_ARGUMENT;
  sqn_type1_opts o;
  sqn_type1_default_opts(&o);
  if (opts) o = *opts;
  if (o.modeord != 0 && o.modeord != 1) return SQN_ERR_INVALID_ARGUMENT;
  if (o.upsampfac != 0.0 && o.upsampfac <= 1.0) return SQN_ERR_UPSAMPFAC_TOO_SMALL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || o.gpu_device_id < 0 || o.gpu_device_id >= ndev) {
    cudaGetLastError();
    return SQN_ERR_NO_DEVICE;
  }
  sqn_type1_plan *p = new (std::nothrow) sqn_type1_s();
  if (!p) return SQN_ERR_ALLOC;
  p->device = o.gpu_device_id;
  p->fp64 = fp64;
  p->iflag = iflag >= 0 ? 1 : -1;
  p->ntr = ntransf;
  p->modeord = o.modeord;
  for (int d = 0; d < 3; ++d) p->N[d] = n_modes[d];
  int st = SQN_OK, warn = SQN_OK;
  auto fail = [&](int code) {
    free_type1(p);
    return code;
  };
  if (cudaSetDevice(p->device) != cudaSuccess) return fail(SQN_ERR_NO_DEVICE);
  if (o.gpu_stream) {
    p->stream = (cudaStream_t)o.gpu_stream;
  } else {
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(SQN_ERR_CUDA);
    p->own_stream = true;
  }
  if (spread_set_attributes() != cudaSuccess) return fail(SQN_ERR_CUDA);
  // fine grid and kernel: the modes play the part of the reciprocal grid
  const double floor_eps = fp64 ? 2.3e-16 : 1.2e-7;
  double eps = tol;
  if (eps < floor_eps) {
    eps = floor_eps;
    warn = SQN_WARN_EPS_TOO_SMALL;
  }
  int modes[3];
  for (int d = 0; d < 3; ++d) modes[d] = (int)std::max<int64_t>(p->N[d], 2);
  if (!hostmath::choose_fine_grid(modes, eps, o.upsampfac, 0, fp64 ? MAX_W : 12, p->nf, &p->w,
                                  &p->sigma))
    warn = SQN_WARN_EPS_TOO_SMALL;
  for (int d = 0; d < 3; ++d)
    if (p->nf[d] < p->N[d] || p->nf[d] > 65536) return fail(SQN_ERR_NOT_SUPPORTED);
  p->beta = hostmath::es_beta(p->w, p->sigma);
  FrameGeom &g = p->g;
  const double two_pi = 2.0 * std::acos(-1.0);
  for (int k = 0; k < 9; ++k) g.inv[k] = 0.0;
  g.inv[0] = g.inv[4] = g.inv[8] = 1.0 / two_pi;
  for (int d = 0; d < 3; ++d) g.origin[d] = -0.5 * two_pi;
  int nsm = 148;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess)
    return fail(SQN_ERR_CUDA);
  const int tmax[3] = {TILE_X, TILE_Y, spread_tile_z(p->nf, 2 * p->ntr, nsm)};
  for (int d = 0; d < 3; ++d) {
    g.nf[d] = (int)p->nf[d];
    g.tile[d] = (int)std::min<int64_t>(p->nf[d], tmax[d]);
    g.ntile[d] = (int)((p->nf[d] + g.tile[d] - 1) / g.tile[d]);
  }
  g.w = p->w;
  g.beta = p->beta;
  g.ntr = 1;
  g.ntiles = g.ntile[0] * g.ntile[1] * g.ntile[2];
  g.pitch = p->nf[0];
  g.vol_real = p->nf[0] * p->nf[1] * p->nf[2];
  g.rec_stride = REC_SLOTS;
  g.chunk = spread_chunk(fp64);
  g.natoms = 0;
  const size_t rsz = fp64 ? 8 : 4;
  const int ngrid = 2 * p->ntr;
  const int64_t c1 = p->nf[0] / 2 + 1;
  const int64_t volc = c1 * p->nf[1] * p->nf[2];
  char *v = nullptr;
  if ((st = talloc(p->fixed, &v, (size_t)ngrid * g.vol_real * rsz))) return fail(st);
  p->d_grid = v;
  if ((st = talloc(p->fixed, &v, (size_t)ngrid * volc * 2 * rsz))) return fail(st);
  p->d_G = v;
  if ((st = talloc(p->fixed, &p->d_counts, (size_t)g.ntiles + 1))) return fail(st);
  if ((st = talloc(p->fixed, &p->d_starts, (size_t)g.ntiles + 1))) return fail(st);
  if (cudaMemset(p->d_counts, 0, sizeof(int) * ((size_t)g.ntiles + 1)) != cudaSuccess)
    return fail(SQN_ERR_CUDA);
  for (int d = 0; d < 3; ++d) {
    const int kmax = (int)(p->N[d] / 2);
    std::vector<double> ft = hostmath::kernel_ft(p->nf[d], p->w, p->beta, kmax);
    for (double &x : ft) x = 1.0 / x;
    if ((st = talloc(p->fixed, &v, ft.size() * rsz))) return fail(st);
    p->d_inv[d] = v;
    cudaError_t e;
    if (fp64) {
      e = cudaMemcpy(v, ft.data(), ft.size() * 8, cudaMemcpyHostToDevice);
    } else {
      std::vector<float> f(ft.begin(), ft.end());
      e = cudaMemcpy(v, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return fail(SQN_ERR_CUDA);
  }
  if (cufftCreate(&p->fft) != CUFFT_SUCCESS) return fail(SQN_ERR_CUFFT);
  p->fft_ok = true;
  long long n[3] = {p->nf[2], p->nf[1], p->nf[0]};
  long long inembed[3] = {p->nf[2], p->nf[1], p->nf[0]};
  long long onembed[3] = {p->nf[2], p->nf[1], c1};
  size_t ws = 0;
  if (cufftMakePlanMany64(p->fft, 3, n, inembed, 1, g.vol_real, onembed, 1, volc,
                          fp64 ? CUFFT_D2Z : CUFFT_R2C, ngrid, &ws) != CUFFT_SUCCESS ||
      cufftSetStream(p->fft, p->stream) != CUFFT_SUCCESS)
    return fail(SQN_ERR_CUFFT);
  *out = p;
  return warn;
}

template <typename R>
int setpts_type1(sqn_type1_plan *p, int64_t M, const R *x, const R *y, const R *z) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (M < 1 || M > (int64_t)INT32_MAX / 2) return SQN_ERR_NUM_NU_PTS_INVALID;
  if (!x || !y || !z) return SQN_ERR_INVALID_ARGUMENT;
  if ((sizeof(R) == 8) != p->fp64) return SQN_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(p->device) != cudaSuccess) return SQN_ERR_NO_DEVICE;
  cudaStream_t s = p->stream;
  if (M > p->Mcap) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return SQN_ERR_CUDA;
    free_list(p->perpts);
    p->Mcap = 0;
    int st;
    const size_t rsz = sizeof(R);
    char *v = nullptr;
    if ((st = talloc(p->perpts, &p->d_pos, 3 * (size_t)M))) return st;
    if ((st = talloc(p->perpts, &p->d_species, (size_t)M))) return st;
    if ((st = talloc(p->perpts, &p->d_key, (size_t)M))) return st;
    if ((st = talloc(p->perpts, &p->d_slot, (size_t)M))) return st;
    if ((st = talloc(p->perpts, &p->d_orig, (size_t)M))) return st;
    if ((st = talloc(p->perpts, &v, (size_t)M * REC_SLOTS * rsz))) return st;
    p->d_recs = v;
    if ((st = talloc(p->perpts, &v, (size_t)M * 2 * p->ntr * rsz))) return st;
    p->d_w = v;
    if (cudaMemset(p->d_species, 0, (size_t)M) != cudaSuccess) return SQN_ERR_CUDA;
    p->Mcap = M;
  }
  p->M = M;
  p->g.natoms = M;
  k_pack_points<R><<<grid1d(M), 256, 0, s>>>(x, y, z, M, p->d_pos);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = launch_prep<R>(p->d_pos, p->d_species, p->g, p->d_counts, p->d_key, p->d_slot, s);
  if (e == cudaSuccess) e = launch_scan(p->d_counts, p->d_starts, p->g.ntiles, s);
  if (e == cudaSuccess)
    e = launch_scatter<R>(p->d_pos, p->d_species, p->g, p->d_key, p->d_slot, p->d_starts,
                          (R *)p->d_recs, p->d_orig, s);
  return e == cudaSuccess ? SQN_OK : SQN_ERR_CUDA;
}

template <typename R> int execute_type1(sqn_type1_plan *p, const R *c, R *fk) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!c || !fk) return SQN_ERR_INVALID_ARGUMENT;
  if ((sizeof(R) == 8) != p->fp64) return SQN_ERR_INVALID_ARGUMENT;
  if (p->M < 1) return SQN_ERR_NUM_NU_PTS_INVALID;
  if (cudaSetDevice(p->device) != cudaSuccess) return SQN_ERR_NO_DEVICE;
  cudaStream_t s = p->stream;
  const int64_t M = p->M;
  R *w = (R *)p->d_w;
  R *grid = (R *)p->d_grid;
  k_sorted_weights<R><<<grid1d(M), 256, 0, s>>>(c, p->d_orig, M, p->ntr, w);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = launch_spread_pw<R>((const R *)p->d_recs, p->d_starts, p->g, w, grid, 2 * p->ntr, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  cufftResult fr = p->fp64 ? cufftExecD2Z(p->fft, (cufftDoubleReal *)p->d_grid,
                                          (cufftDoubleComplex *)p->d_G)
                           : cufftExecR2C(p->fft, (cufftReal *)p->d_grid, (cufftComplex *)p->d_G);
  if (fr != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
  const int64_t nm = p->N[0] * p->N[1] * p->N[2] * p->ntr;
  k_type1_out<R><<<grid1d(nm), 256, 0, s>>>(
      (const typename Cplx<R>::T *)p->d_G, p->ntr, p->N[0], p->N[1], p->N[2], p->nf[0],
      p->nf[1], p->nf[2], p->iflag, p->modeord, (const R *)p->d_inv[0], (const R *)p->d_inv[1],
      (const R *)p->d_inv[2], fk);
  if (cudaGetLastError() != cudaSuccess) return SQN_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? SQN_OK : SQN_ERR_CUDA;
}

}  // namespace

extern "C" {

void sqn_type1_default_opts(sqn_type1_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->gpu_device_id = 0;
  o->modeord = 0;
  o->upsampfac = 0.0;
  o->gpu_stream = nullptr;
}

int sqn_type1_makeplan(int32_t type, int32_t dim, const int64_t *n_modes, int32_t iflag,
                       int32_t ntransf, double tol, sqn_type1_plan **plan,
                       const sqn_type1_opts *opts) {
  return make_type1(type, dim, n_modes, iflag, ntransf, tol, plan, opts, true);
}

int sqn_type1f_makeplan(int32_t type, int32_t dim, const int64_t *n_modes, int32_t iflag,
                        int32_t ntransf, float tol, sqn_type1_plan **plan,
                        const sqn_type1_opts *opts) {
  return make_type1(type, dim, n_modes, iflag, ntransf, (double)tol, plan, opts, false);
}

int sqn_type1_setpts(sqn_type1_plan *plan, int64_t M, const double *d_x, const double *d_y,
                     const double *d_z) {
  return setpts_type1<double>(plan, M, d_x, d_y, d_z);
}

int sqn_type1f_setpts(sqn_type1_plan *plan, int64_t M, const float *d_x, const float *d_y,
                      const float *d_z) {
  return setpts_type1<float>(plan, M, d_x, d_y, d_z);
}

int sqn_type1_execute(sqn_type1_plan *plan, const double *d_c, double *d_fk) {
  return execute_type1<double>(plan, d_c, d_fk);
}

int sqn_type1f_execute(sqn_type1_plan *plan, const float *d_c, float *d_fk) {
  return execute_type1<float>(plan, d_c, d_fk);
}

int sqn_type1_destroy(sqn_type1_plan *plan) {
  if (!plan) return SQN_ERR_PLAN_NOTVALID;
  free_type1(plan);
  return SQN_OK;
}

}  // extern "C"
