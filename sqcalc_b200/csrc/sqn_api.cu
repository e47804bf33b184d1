// C ABI of libsqnufft.so: plan set up, per-frame pipeline, accumulators.
//
// The plan is the B200 counterpart of three reference objects at once:
//   * structure_factor_t's grid bookkeeping (src/sqc_structure_factor.f90:313-451),
//   * cufinufft_structure_factor_t (src/sqc_gpu.f90:108-404),
//   * the cuFINUFFT type-1 plan it drives (external/finufft/include/cufinufft/impl.h:51-330).
// Everything per frame stays on the device; only nq-sized accumulators return.
#include <cufft.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "../../include/sqnufft.h"
#include "sqn_internal.h"

using namespace sqn;

namespace {
constexpr int64_t kRefMaxGridModes = 400000000LL;  // src/sqc_structure_factor.f90:63-64
}  // namespace

// Host math shared with the type-1 entry points (sqn_type1.cu).
namespace sqn {
namespace hostmath {

// ---------------------------------------------------------------------------
// Host math
// ---------------------------------------------------------------------------

// determinant3 / inverse3 of src/sqc_cell.f90:131-152; m[3*c + r] = m(r+1, c+1).
double det3(const double *a) {
  auto M = [a](int r, int c) { return a[3 * (c - 1) + (r - 1)]; };
  return M(1, 1) * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)) -
         M(1, 2) * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1)) +
         M(1, 3) * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
}

void inverse3(const double *a, double *inv) {
  auto M = [a](int r, int c) { return a[3 * (c - 1) + (r - 1)]; };
  auto I = [inv](int r, int c) -> double & { return inv[3 * (c - 1) + (r - 1)]; };
  const double det = det3(a);
  I(1, 1) = (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2));
  I(2, 1) = -(M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1));
  I(3, 1) = (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
  I(1, 2) = -(M(1, 2) * M(3, 3) - M(1, 3) * M(3, 2));
  I(2, 2) = (M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1));
  I(3, 2) = -(M(1, 1) * M(3, 2) - M(1, 2) * M(3, 1));
  I(1, 3) = (M(1, 2) * M(2, 3) - M(1, 3) * M(2, 2));
  I(2, 3) = -(M(1, 1) * M(2, 3) - M(1, 3) * M(2, 1));
  I(3, 3) = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1));
  for (int k = 0; k < 9; ++k) inv[k] = inv[k] / det;
}

// Smallest even integer >= n whose prime factors are 2, 3 and 5.
int64_t next235even(int64_t n) {
  if (n <= 2) return 2;
  if (n % 2) ++n;
  for (int64_t c = n;; c += 2) {
    int64_t d = c;
    while (d % 2 == 0) d /= 2;
    while (d % 3 == 0) d /= 3;
    while (d % 5 == 0) d /= 5;
    if (d == 1) return c;
  }
}

// Kernel width for tolerance eps at upsampling sigma and the ES shape beta, the
// published exponential-of-semicircle choices (Barnett, Magland, af Klinteberg,
// SIAM J. Sci. Comput. 41 (2019)) in the form external/finufft/src/cuda/
// spreadinterp.cpp:59-85 applies them.
int es_width(double eps, double sigma) {
  int w;
  if (sigma == 2.0)
    w = (int)std::ceil(-std::log10(eps / 10.0));
  else
    w = (int)std::ceil(-std::log(eps) / (M_PI * std::sqrt(1.0 - 1.0 / sigma)));
  return std::max(2, w);
}

double es_beta(int w, double sigma) {
  double bw = 2.30;
  if (w == 2) bw = 2.20;
  if (w == 3) bw = 2.26;
  if (w == 4) bw = 2.38;
  if (sigma != 2.0) bw = 0.97 * M_PI * (1.0 - 1.0 / (2.0 * sigma));
  return bw * w;
}

// Relative cost of one cell of a 3D real-to-complex FFT of size n on B200:
// measured cuFFT throughput is ~6 ps per cell for powers of two >= 256 and
// ~9-13 ps for other 2,3,5-smooth sizes.
double fft_cell_cost(int64_t n) {
  const bool pow2 = (n & (n - 1)) == 0;
  return (pow2 && n >= 256) ? 0.65 : 1.0;
}

// Fine grid and ES width.  With sigma given, nf = next235even(max(sigma m, 2w))
// per dimension (the reference's rule, external/finufft/src/cuda/common.cu:166-177).
// Otherwise each dimension takes the cheapest FFT size n >= 1.2 m whose
// upsampling n/m reaches eps with a width <= wcap; the width is then the one the
// smallest upsampling needs.  Returns false when eps needs a width above MAX_W.
bool choose_fine_grid(const int *modes, double eps, double sigma_req, int w_req, int wcap,
                      int64_t *nf, int *w_out, double *sigma_out) {
  bool ok = true;
  if (sigma_req > 0.0) {
    int w = w_req > 0 ? w_req : es_width(eps, sigma_req);
    if (w > MAX_W) {
      w = MAX_W;
      ok = false;
    }
    for (int i = 0; i < 3; ++i)
      nf[i] = next235even(std::max<int64_t>((int64_t)std::ceil(sigma_req * modes[i]), 2 * w));
    *w_out = w;
    *sigma_out = sigma_req;
    return ok;
  }
  double smin = 1e30;
  for (int i = 0; i < 3; ++i) {
    const int m = modes[i];
    int64_t best = 0;
    double best_cost = 1e300;
    int64_t n = next235even((int64_t)std::ceil(1.2 * m));
    for (int k = 0; k < 64 && n <= (int64_t)std::ceil(2.5 * m) + 64; ++k) {
      const double s = (double)n / m;
      const int w = std::max(w_req > 0 ? w_req : es_width(eps, s), 2);
      if (w <= wcap && n >= 2 * w) {
        const double cost = (double)n * fft_cell_cost(n);
        if (cost < best_cost) {
          best_cost = cost;
          best = n;
        }
      }
      n = next235even(n + 2);
    }
    if (best == 0) best = next235even(std::max<int64_t>(2 * m, 2 * MAX_W));
    nf[i] = best;
    smin = std::min(smin, (double)best / m);
  }
  int w = w_req > 0 ? w_req : es_width(eps, smin);
  if (w > MAX_W) {
    w = MAX_W;
    ok = false;
  }
  for (int i = 0; i < 3; ++i) nf[i] = std::max<int64_t>(nf[i], next235even(2 * w));
  *w_out = w;
  *sigma_out = smin;
  return ok;
}

double es_phi_host(double t, int w, double beta) {
  const double z = 2.0 * t / w;
  const double zz = z * z;
  return zz < 1.0 ? std::exp(beta * (std::sqrt(1.0 - zz) - 1.0)) : 0.0;
}

// n-point Gauss-Legendre rule on [-1, 1] (Newton iteration on P_n).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &wt) {
  x.assign(n, 0.0);
  wt.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    wt[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Fourier transform of the kernel at the integer frequencies 0..kmax of an
// nf-periodic grid: phihat(k) = 2 int_0^{w/2} phi(t) cos(2 pi k t / nf) dt,
// by Gauss-Legendre quadrature (cf. external/finufft/src/cuda/common.cu:196-210).
std::vector<double> kernel_ft(int64_t nf, int w, double beta, int kmax) {
  const int n = 4 * w + 24;
  std::vector<double> x, wt;
  gauss_legendre(n, x, wt);
  std::vector<double> out(kmax + 1);
  const double half = 0.5 * w;
  for (int k = 0; k <= kmax; ++k) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
      const double t = 0.5 * half * (x[i] + 1.0);
      s += 0.5 * half * wt[i] * es_phi_host(t, w, beta) * std::cos(2.0 * M_PI * k * t / (double)nf);
    }
    out[k] = 2.0 * s;
  }
  return out;
}

// |q| in the reference's operation order (src/sqc_structure_factor.f90:366-368).
inline double qlen_ref(const double *b, int h1, int h2, int h3) {
  double q[3];
  for (int r = 0; r < 3; ++r) q[r] = b[r] * (double)h1 + b[3 + r] * (double)h2 + b[6 + r] * (double)h3;
  return std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
}

double xray_f_host(const double *c, double q) {
  double st = q / (4.0 * std::acos(-1.0));
  st = st * st;
  double f = c[8];
  for (int i = 0; i < 4; ++i) f = f + c[i] * std::exp(-c[4 + i] * st);
  return f;
}

}  // namespace hostmath
}  // namespace sqn
using namespace sqn::hostmath;

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------

struct sqn_plan_s {
  sqn_plan_desc desc{};
  bool fp64 = false;
  int device = 0;
  cudaStream_t stream = nullptr, copy_stream = nullptr;
  bool own_stream = false;
  int nsm = 148;

  double cell[9], origin[3], inv[9], recip[9];
  int modes[3], hm[3];
  int64_t gridpoints = 0, nmodes = 0;
  int w = 0;
  double beta = 0, sigma = 0, eps_used = 0;
  int64_t nf[3];
  FrameGeom fg{};
  BinGeom bg{};
  int ntr = 0, nspecies = 0, nquant = 1, nrows = 0;
  int nkeys = 0;
  std::vector<int> species_type;   // type id of each species
  std::vector<int64_t> type_counts;  // atoms per type id (index t-1)
  std::vector<double> amp_sp, xcoef_sp;
  std::vector<double> den, cnt;    // per shell, from the set-up pass

  double *d_pos[2] = {nullptr, nullptr};
  uint8_t *d_species = nullptr;
  int *d_counts = nullptr, *d_starts = nullptr;
  uint32_t *d_key = nullptr, *d_slot = nullptr;
  void *d_recs = nullptr, *d_grid = nullptr, *d_G = nullptr;
  void *d_inv[3] = {nullptr, nullptr, nullptr};
  void *d_strength = nullptr;
  double *d_amp = nullptr, *d_xcoef = nullptr, *d_amp_sp = nullptr, *d_xcoef_sp = nullptr,
         *d_counts_sp = nullptr;
  int4 *d_rows = nullptr;
  double *d_acc = nullptr, *d_gnum = nullptr, *d_den = nullptr, *d_cnt = nullptr;
  cufftHandle fft = 0;
  bool fft_ok = false;
  bool inplace = false;  // cuFFT R2C in place over padded real rows (dS/dr plans)
  int64_t c1pitch = 0;  // complex row pitch of the half spectrum
  // pruned 512-point passes (every axis 512): compact half spectrum in d_G
  bool fft512 = false;
  void *d_tw512 = nullptr;
  int *d_h1end = nullptr;  // per h2 (FFT order): one past the largest kept h1 of any h3
  short2 *d_h2band = nullptr;  // per 16-column block of h1: the h2 band it needs
  BinGeom bg512{};
  // density amplitudes (sqn_density_modes): request buffers, grown on demand
  int *d_hkl = nullptr;
  double *d_rho = nullptr;
  int64_t modes_cap = 0;
  // adjoint (SQN_FLAG_GRAD)
  bool grad_ok = false;
  int32_t *d_orig = nullptr;
  void *d_F = nullptr, *d_U = nullptr, *d_wstrength = nullptr;
  double *d_grad = nullptr, *d_gsh = nullptr, *d_num1 = nullptr;
  cufftHandle fft_fwd1 = 0, fft_inv3 = 0;
  bool fft_fwd1_ok = false, fft_inv3_ok = false;
  int64_t gnum_half = 0;
  int64_t nsums = 0;           // shell + powder-pattern sums at the head of d_acc
  double *d_xcnt = nullptr;    // kept modes per two-theta bin

  // SQN_FLAG_AUTOTUNE: fine grid and width chosen by timing
  int autotuned = 0, tune_candidates = 0;
  double tune_ms = 0.0;

  int64_t nframes = 0;
  int slot_next = 0;
  cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  bool timing = false;
  std::vector<cudaEvent_t> tev_pool;  // 5 per timed frame
  size_t tev_used = 0;
  double stage_ms[4] = {0, 0, 0, 0};
  int64_t stage_frames = 0;
  int64_t launches = 0;
  int64_t device_bytes = 0;
  std::vector<void *> allocs;
};

namespace {

int cuda_status(cudaError_t e) { return e == cudaSuccess ? SQN_OK : SQN_ERR_CUDA; }

template <typename T> int dalloc(sqn_plan *p, T **ptr, size_t count) {
  *ptr = nullptr;
  if (count == 0) count = 1;
  void *v = nullptr;
  if (cudaMalloc(&v, count * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_ALLOC;
  }
  p->allocs.push_back(v);
  p->device_bytes += (int64_t)(count * sizeof(T));
  *ptr = static_cast<T *>(v);
  return SQN_OK;
}

void free_plan(sqn_plan *p) {
  if (!p) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->copy_stream) cudaStreamSynchronize(p->copy_stream);
  if (p->fft_ok) cufftDestroy(p->fft);
  if (p->fft_fwd1_ok) cufftDestroy(p->fft_fwd1);
  if (p->fft_inv3_ok) cufftDestroy(p->fft_inv3);
  for (void *v : p->allocs) cudaFree(v);
  if (p->d_hkl) cudaFree(p->d_hkl);
  if (p->d_rho) cudaFree(p->d_rho);
  for (int i = 0; i < 2; ++i) {
    if (p->ev_copied[i]) cudaEventDestroy(p->ev_copied[i]);
    if (p->ev_free[i]) cudaEventDestroy(p->ev_free[i]);
  }
  for (cudaEvent_t e : p->tev_pool) cudaEventDestroy(e);
  if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
  if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
  cudaSetDevice(cur);
  delete p;
}

// Rows (h2, h3) of the half space h1 >= 0 that reach |q| <= qmax, with a
// conservative h1 range; the kernels test every mode exactly.
std::vector<int4> build_rows(const double *b, const int *hm, double qmax) {
  std::vector<int4> rows;
  const double *b1 = b, *b2 = b + 3, *b3 = b + 6;
  const double A = b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2];
  const double qm = qmax * (1.0 + 1e-9) + 1e-12;
  for (int h3 = -hm[2]; h3 <= hm[2]; ++h3) {
    for (int h2 = -hm[1]; h2 <= hm[1]; ++h2) {
      double c[3];
      for (int r = 0; r < 3; ++r) c[r] = h2 * b2[r] + h3 * b3[r];
      const double B = 2.0 * (b1[0] * c[0] + b1[1] * c[1] + b1[2] * c[2]);
      const double C = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] - qm * qm;
      const double disc = B * B - 4.0 * A * C;
      if (disc < 0.0) continue;
      const double sq = std::sqrt(disc);
      const double r1 = (-B - sq) / (2.0 * A), r2 = (-B + sq) / (2.0 * A);
      int lo = (int)std::max(0.0, std::floor(r1) - 1.0);
      const double hi_d = std::min((double)hm[0], std::ceil(r2) + 1.0);
      if (hi_d < 0.0) continue;
      const int hi = (int)hi_d;
      if (lo > hi) continue;
      rows.push_back(make_int4(h2, h3, lo, hi));
    }
  }
  return rows;
}

template <typename R> std::vector<R> to_r(const std::vector<double> &v) {
  return std::vector<R>(v.begin(), v.end());
}

// ---------------------------------------------------------------------------
// Autotuner (SQN_FLAG_AUTOTUNE): candidate (sigma, w) pairs that reach eps --
// for each kernel width up to the precision's cap the smallest 2,3,5-smooth
// upsampling of the largest mode count that reaches it, plus the cost model's
// own choice -- each timed on the plan's shape (same cell, atoms, types, q
// range, precision and flags) over a few frames of uniform positions; the
// fastest is kept and cached per shape for the life of the process.
// ---------------------------------------------------------------------------
struct TuneResult {
  double sigma;  // 0: the cost model's grid
  int w;
  int ncand;
  double ms;
};
std::mutex g_tune_mutex;
std::map<std::string, TuneResult> g_tune_cache;

std::string tune_key(const sqn_plan *p, const sqn_plan_desc *d, double eps) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%d/%d/%d|%.17g|%d|%lld|%d|%d|%d|%d|%d|%.17g|%.17g|%d|%x",
                p->modes[0], p->modes[1], p->modes[2], eps, (int)p->fp64,
                (long long)d->natoms, p->ntr, d->partials, d->weight, d->want_grid, d->device,
                d->qmin, d->qmax, d->nq, (unsigned)(d->flags & ~SQN_FLAG_AUTOTUNE));
  return std::string(buf);
}

int autotune_grid(sqn_plan *p, const sqn_plan_desc *d, double eps, TuneResult *out) {
  const std::string key = tune_key(p, d, eps);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      *out = it->second;
      out->ncand = 0;
      return SQN_OK;
    }
  }
  const int m = std::max(p->modes[0], std::max(p->modes[1], p->modes[2]));
  const int wcap = p->fp64 ? MAX_W : 12;
  std::vector<std::pair<double, int>> cand;
  cand.push_back({0.0, 0});  // the cost model's choice
  int last_w = 1 << 30;
  for (int64_t n = next235even((int64_t)std::ceil(1.2 * m)); n <= (int64_t)(2.05 * m) + 2;
       n = next235even(n + 2)) {
    const double s = (double)n / m;
    const int w = es_width(eps, s);
    if (w > wcap || n < 2 * w || w >= last_w) continue;
    cand.push_back({s, w});
    last_w = w;
  }
  // uniform positions in the cell, one frame, device resident
  const int64_t N = d->natoms;
  std::vector<double> pos((size_t)N * 3);
  std::mt19937_64 rng(12345);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  for (int64_t i = 0; i < N; ++i) {
    const double f0 = U(rng), f1 = U(rng), f2 = U(rng);
    for (int r = 0; r < 3; ++r)
      pos[3 * i + r] = d->origin[r] + f0 * d->cell[r] + f1 * d->cell[3 + r] + f2 * d->cell[6 + r];
  }
  double *dpos = nullptr;
  if (cudaMalloc(&dpos, pos.size() * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_ALLOC;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int st = cudaMemcpy(dpos, pos.data(), pos.size() * sizeof(double), cudaMemcpyHostToDevice) ==
                   cudaSuccess
               ? SQN_OK
               : SQN_ERR_CUDA;
  // dS/dr plans are timed on their gradient evaluation (forward recomputed,
  // three type-2 interpolations), the others on frame accumulation
  const bool grad = (d->flags & SQN_FLAG_GRAD) != 0;
  std::vector<double> ones((size_t)d->nq, 1.0), S((size_t)d->nq);
  double *dgrad = nullptr;
  if (st == SQN_OK && grad && cudaMalloc(&dgrad, sizeof(double) * 3 * (size_t)N) != cudaSuccess) {
    cudaGetLastError();
    st = SQN_ERR_ALLOC;
  }
  auto run = [&](sqn_plan *sp) {
    return grad ? sqn_sq_grad(sp, dpos, SQN_DEVICE, ones.data(), S.data(), dgrad)
                : sqn_accumulate_frames(sp, dpos, 1, SQN_DEVICE);
  };
  TuneResult best{0.0, 0, 0, 1e300};
  constexpr int kFrames = 3;
  for (size_t c = 0; c < cand.size() && st == SQN_OK; ++c) {
    sqn_plan_desc sd = *d;
    sd.flags &= ~(SQN_FLAG_AUTOTUNE | SQN_FLAG_TIMING);
    sd.upsampfac = cand[c].first;
    sd.kernel_width = cand[c].second;
    sqn_plan *sp = nullptr;
    if (sqn_plan_create(&sd, &sp) > SQN_WARN_EPS_TOO_SMALL || !sp) continue;  // e.g. no memory
    int rc = run(sp);
    if (rc == SQN_OK) rc = sqn_sync(sp);
    float ms = 0.f;
    if (rc == SQN_OK && cudaEventRecord(e0, sp->stream) == cudaSuccess) {
      for (int f = 0; f < kFrames && rc == SQN_OK; ++f) rc = run(sp);
      if (rc == SQN_OK && (cudaEventRecord(e1, sp->stream) != cudaSuccess ||
                           cudaEventSynchronize(e1) != cudaSuccess ||
                           cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        rc = SQN_ERR_CUDA;
    }
    sqn_plan_destroy(sp);
    if (rc != SQN_OK) {
      st = rc;
      break;
    }
    ms /= kFrames;
    if (ms < best.ms) best = {cand[c].first, cand[c].second, 0, ms};
    best.ncand = (int)c + 1;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dpos);
  if (dgrad) cudaFree(dgrad);
  if (st != SQN_OK) return st;
  if (best.ms >= 1e300) return SQN_ERR_ALLOC;
  best.ncand = (int)cand.size();
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best;
  }
  *out = best;
  return SQN_OK;
}

int setup_plan(sqn_plan *p, const sqn_plan_desc *d) {
  p->desc = *d;
  p->desc.type_id = nullptr;
  p->desc.amp_const = nullptr;
  p->desc.xray_coef = nullptr;
  p->fp64 = d->precision == SQN_PREC_DOUBLE;
  p->timing = (d->flags & SQN_FLAG_TIMING) != 0;
  int warn = SQN_OK;

  // --- device ----------------------------------------------------------
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return SQN_ERR_NO_DEVICE;
  }
  if (d->device < 0 || d->device >= ndev) return SQN_ERR_NO_DEVICE;
  p->device = d->device;
  if (cudaSetDevice(p->device) != cudaSuccess) return SQN_ERR_CUDA;
  cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device);
  if (d->stream) {
    p->stream = (cudaStream_t)d->stream;
  } else {
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
      return SQN_ERR_CUDA;
    p->own_stream = true;
  }
  if (cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return SQN_ERR_CUDA;
  for (int i = 0; i < 2; ++i) {
    if (cudaEventCreateWithFlags(&p->ev_copied[i], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_free[i], cudaEventDisableTiming) != cudaSuccess)
      return SQN_ERR_CUDA;
  }
  if (spread_set_attributes() != cudaSuccess) return SQN_ERR_CUDA;

  // --- cell and reciprocal grid (sf_configure, :313-399) --------------------
  std::memcpy(p->cell, d->cell, sizeof(p->cell));
  std::memcpy(p->origin, d->origin, sizeof(p->origin));
  if (det3(p->cell) == 0.0) return SQN_ERR_DEGENERATE_CELL;
  inverse3(p->cell, p->inv);
  const double two_pi = 2.0 * std::acos(-1.0);
  for (int j = 0; j < 3; ++j)
    for (int r = 0; r < 3; ++r) p->recip[3 * j + r] = two_pi * p->inv[3 * r + j];
  for (int i = 0; i < 3; ++i) {
    const double *v = p->cell + 3 * i;
    const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (len <= 0.0) return SQN_ERR_DEGENERATE_CELL;
    p->modes[i] = std::max(2 * (int)std::ceil(d->qmax * len / two_pi) + 1, 3);
    p->hm[i] = (p->modes[i] - 1) / 2;
  }
  p->gridpoints = (int64_t)p->modes[0] * p->modes[1] * p->modes[2];
  const int64_t cap = d->max_grid_modes == 0 ? kRefMaxGridModes : d->max_grid_modes;
  if (cap > 0 && p->gridpoints > cap) return SQN_ERR_GRID_TOO_LARGE;
  if (!(d->qmax > d->qmin) || d->nq < 1) return SQN_ERR_INVALID_ARGUMENT;

  // --- species (sf_shared_setup + sf_prepare_species, :256-292, :1109-1163) --
  if (d->natoms < 1 || d->natoms > (int64_t)INT32_MAX / 2) return SQN_ERR_NUM_NU_PTS_INVALID;
  if (d->ntypes < 1 || !d->type_id) return SQN_ERR_INVALID_ARGUMENT;
  p->type_counts.assign(d->ntypes, 0);
  for (int64_t i = 0; i < d->natoms; ++i) {
    const int t = d->type_id[i];
    if (t < 1 || t > d->ntypes) return SQN_ERR_TYPE_ID;
    p->type_counts[t - 1]++;
  }
  std::vector<int> species_of_type(d->ntypes + 1, -1);
  for (int t = 1; t <= d->ntypes; ++t)
    if (p->type_counts[t - 1] > 0) {
      species_of_type[t] = (int)p->species_type.size();
      p->species_type.push_back(t);
    }
  p->nspecies = (int)p->species_type.size();
  if (p->nspecies > 255) return SQN_ERR_NOT_SUPPORTED;
  const bool xray = d->weight == SQN_WEIGHT_XRAY;
  if (d->weight == SQN_WEIGHT_NEUTRON && !d->amp_const) return SQN_ERR_INVALID_ARGUMENT;
  if (xray && !d->xray_coef) return SQN_ERR_INVALID_ARGUMENT;
  p->amp_sp.assign(p->nspecies, 1.0);
  p->xcoef_sp.assign(9 * (size_t)p->nspecies, 0.0);
  for (int s = 0; s < p->nspecies; ++s) {
    const int t = p->species_type[s];
    if (d->weight == SQN_WEIGHT_NEUTRON) p->amp_sp[s] = d->amp_const[t - 1];
    if (xray) std::memcpy(&p->xcoef_sp[9 * s], d->xray_coef + 9 * (size_t)(t - 1), 9 * sizeof(double));
  }
  // One transform per species for pair columns or q-dependent weights, else a
  // single weighted transform (src/sqc_gpu.f90:190-197).
  p->ntr = (d->partials || xray) ? p->nspecies : 1;
  if (p->ntr > MAX_FAST_T) return SQN_ERR_NOT_SUPPORTED;
  p->nquant = 1 + (d->partials ? p->ntr * (p->ntr + 1) / 2 : 0);

  // --- kernel and fine grid ----------------------------------------------
  double eps = d->eps;
  const double floor_eps = p->fp64 ? DBL_EPSILON : (double)FLT_EPSILON;
  if (!(eps > 0.0)) return SQN_ERR_INVALID_ARGUMENT;
  if (eps < floor_eps) {
    eps = floor_eps;
    warn = SQN_WARN_EPS_TOO_SMALL;
  }
  p->eps_used = eps;
  if (d->upsampfac != 0.0 && d->upsampfac <= 1.0) return SQN_ERR_UPSAMPFAC_TOO_SMALL;
  int w = 0;
  double sigma = 0.0;
  double sigma_req = d->upsampfac;
  int w_req = d->kernel_width;
  if ((d->flags & SQN_FLAG_AUTOTUNE) && sigma_req == 0.0 && w_req == 0) {
    TuneResult tr{};
    const int ts = autotune_grid(p, d, eps, &tr);
    if (ts != SQN_OK) return ts;
    sigma_req = tr.sigma;
    w_req = tr.w;
    p->autotuned = 1;
    p->tune_candidates = tr.ncand;
    p->tune_ms = tr.ms;
    if (cudaSetDevice(p->device) != cudaSuccess) return SQN_ERR_CUDA;
  }
  if (!choose_fine_grid(p->modes, eps, sigma_req, w_req, p->fp64 ? MAX_W : 12, p->nf, &w,
                        &sigma)) {
    w = MAX_W;
    warn = SQN_WARN_EPS_TOO_SMALL;
  }
  p->w = w;
  p->sigma = sigma;
  p->beta = es_beta(w, sigma);

  // --- tiles ---------------------------------------------------------------
  FrameGeom &g = p->fg;
  const int tmax[3] = {TILE_X, TILE_Y, spread_tile_z(p->nf, p->ntr, p->nsm)};
  for (int i = 0; i < 3; ++i) {
    g.nf[i] = (int)p->nf[i];
    g.tile[i] = (int)std::min<int64_t>(tmax[i], p->nf[i]);
    g.ntile[i] = (int)((p->nf[i] + g.tile[i] - 1) / g.tile[i]);
  }
  std::memcpy(g.inv, p->inv, sizeof(g.inv));
  std::memcpy(g.origin, p->origin, sizeof(g.origin));
  g.w = w;
  g.beta = p->beta;
  g.ntr = p->ntr;
  g.ntiles = g.ntile[0] * g.ntile[1] * g.ntile[2];
  // Grid layout.  Plans for dS/dr run their R2C in place (real rows padded to
  // 2 (nf0/2 + 1), the half spectrum overwriting them): measured on B200 that
  // makes the gradient evaluation ~25 % faster, while the S(q) frame path is
  // fastest out of place (dense real rows: aligned spread stores; any row
  // padding slows cuFFT).
  p->inplace = (d->flags & SQN_FLAG_GRAD) != 0;
  p->c1pitch = p->nf[0] / 2 + 1;
  g.pitch = p->inplace ? 2 * p->c1pitch : p->nf[0];
  g.vol_real = g.pitch * p->nf[1] * p->nf[2];
  g.natoms = d->natoms;
  g.rec_stride = rec_stride(w, p->fp64);
  g.chunk = spread_chunk(p->fp64);
  if ((int64_t)g.ntiles * p->ntr >= INT32_MAX) return SQN_ERR_NOT_SUPPORTED;
  p->nkeys = (int)spread_nkeys(g);  // one bin per (transform, tile)

  BinGeom &b = p->bg;
  std::memcpy(b.recip, p->recip, sizeof(b.recip));
  b.qmin = d->qmin;
  b.qmax = d->qmax;
  b.dq = (d->qmax - d->qmin) / (double)d->nq;
  b.qminf = (float)d->qmin;
  b.qmaxf = (float)d->qmax;
  b.invdqf = (float)(1.0 / b.dq);
  b.nq = d->nq;
  for (int i = 0; i < 3; ++i) {
    b.hm[i] = p->hm[i];
    b.nf[i] = (int)p->nf[i];
  }
  b.c1 = p->c1pitch;  // row pitch of the half spectrum (>= nf0/2 + 1)
  b.vol_cplx = b.c1 * p->nf[1] * p->nf[2];
  b.ntr = p->ntr;
  b.nquant = p->nquant;
  b.partials = d->partials ? 1 : 0;
  b.xray = xray ? 1 : 0;
  b.want_grid = d->want_grid ? 1 : 0;
  b.m2 = p->modes[1];
  b.norm = d->norm;
  b.natoms = d->natoms;
  if (d->norm < 1 || d->norm > 3) return SQN_ERR_INVALID_ARGUMENT;

  // --- powder XRD bins (sf_configure_xrd, src/sqc_structure_factor.f90:846-905)
  b.xrd = 0;
  b.xbins = 0;
  b.xquant = 0;
  if (d->xrd_lambda > 0.0) {
    const double tmin = d->xrd_2theta_min, tmax = d->xrd_2theta_max;
    if (!(tmin > 0.0 && tmax < 180.0 && tmax > tmin)) return SQN_ERR_INVALID_ARGUMENT;
    const double deg2rad = M_PI / 180.0;
    double step = d->xrd_step;
    if (!(step > 0.0)) {
      // the narrowest cell width, every direction taken as periodic
      const double *a = d->cell;
      double bound = 1e300;
      for (int i = 0; i < 3; ++i) {
        const double *u = a + 3 * ((i + 1) % 3), *v = a + 3 * ((i + 2) % 3);
        const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2],
                     cz = u[0] * v[1] - u[1] * v[0];
        const double area = std::sqrt(cx * cx + cy * cy + cz * cz);
        if (area > 0.0) bound = std::min(bound, std::fabs(det3(a)) / area);
      }
      if (!(bound > 0.0 && bound < 1e300)) return SQN_ERR_DEGENERATE_CELL;
      const double theta_max = std::min(0.5 * deg2rad * tmax, 60.0 * deg2rad);
      step = (d->xrd_lambda / (bound * std::cos(theta_max))) / deg2rad;
    }
    const double nb = std::ceil((tmax - tmin) / step);
    if (!(nb < 1e7)) return SQN_ERR_INVALID_ARGUMENT;
    b.xbins = std::max(1, (int)nb);
    b.xstep = (tmax - tmin) / (double)b.xbins;
    b.xmin = tmin;
    b.xlambda = d->xrd_lambda;
    b.xlp = d->xrd_lp ? 1 : 0;
    b.xquant = p->nquant;
    b.xrd = 1;
  }

  // --- device buffers --------------------------------------------------------
  const int64_t N = d->natoms;
  const size_t rsz = p->fp64 ? 8 : 4;
  int st;
  for (int i = 0; i < 2; ++i)
    if ((st = dalloc(p, &p->d_pos[i], 3 * (size_t)N))) return st;
  if ((st = dalloc(p, &p->d_species, (size_t)N))) return st;
  if ((st = dalloc(p, &p->d_key, (size_t)N))) return st;
  if ((st = dalloc(p, &p->d_slot, (size_t)N))) return st;
  if ((st = dalloc(p, &p->d_counts, (size_t)p->nkeys))) return st;
  if ((st = dalloc(p, &p->d_starts, (size_t)p->nkeys + 1))) return st;
  {
    char *v;
    if ((st = dalloc(p, &v, (size_t)N * g.rec_stride * rsz)))
      return st;
    p->d_recs = v;
    if ((st = dalloc(p, &v, (size_t)p->ntr * g.vol_real * rsz))) return st;
    p->d_grid = v;
    if (p->inplace) {
      p->d_G = v;
    } else {
      if ((st = dalloc(p, &v, (size_t)p->ntr * b.vol_cplx * 2 * rsz))) return st;
      p->d_G = v;
    }
    for (int i = 0; i < 3; ++i) {
      if ((st = dalloc(p, &v, (size_t)(p->hm[i] + 1) * rsz))) return st;
      p->d_inv[i] = v;
    }
    if ((st = dalloc(p, &v, (size_t)p->nspecies * rsz))) return st;
    p->d_strength = v;
  }
  if ((st = dalloc(p, &p->d_amp, (size_t)p->ntr))) return st;
  if ((st = dalloc(p, &p->d_xcoef, 9 * (size_t)p->ntr))) return st;
  if ((st = dalloc(p, &p->d_amp_sp, (size_t)p->nspecies))) return st;
  if ((st = dalloc(p, &p->d_xcoef_sp, 9 * (size_t)p->nspecies))) return st;
  if ((st = dalloc(p, &p->d_counts_sp, (size_t)p->nspecies))) return st;
  // The FP64 sums (shell sums, pair sums, then the per-mode sums with
  // want_grid) share one allocation, so that ranks holding disjoint frames can
  // add them with a single all-reduce (sqn_accumulator_view).
  if (d->want_grid) p->gnum_half = (int64_t)(p->hm[0] + 1) * p->modes[1] * p->modes[2];
  p->nsums = (int64_t)hist_len(b);  // shell sums, then the powder-pattern sums
  if ((st = dalloc(p, &p->d_acc, (size_t)p->nsums + (size_t)p->gnum_half))) return st;
  if (d->want_grid) p->d_gnum = p->d_acc + p->nsums;
  if (b.xrd && (st = dalloc(p, &p->d_xcnt, (size_t)b.xbins))) return st;
  if ((st = dalloc(p, &p->d_den, (size_t)d->nq))) return st;
  if ((st = dalloc(p, &p->d_cnt, (size_t)d->nq))) return st;

  // --- constant tables ----------------------------------------------------
  cudaStream_t s = p->stream;
  std::vector<uint8_t> sp_of(N);
  for (int64_t i = 0; i < N; ++i) sp_of[i] = (uint8_t)species_of_type[d->type_id[i]];
  cudaError_t e = cudaMemcpyAsync(p->d_species, sp_of.data(), (size_t)N, cudaMemcpyHostToDevice, s);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
    std::vector<double> ft = kernel_ft(p->nf[i], w, p->beta, p->hm[i]);
    for (double &v : ft) v = 1.0 / v;
    if (p->fp64) {
      e = cudaMemcpyAsync(p->d_inv[i], ft.data(), ft.size() * 8, cudaMemcpyHostToDevice, s);
    } else {
      std::vector<float> f = to_r<float>(ft);
      e = cudaMemcpyAsync(p->d_inv[i], f.data(), f.size() * 4, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  {
    // strength of each species in the spread: 1 per species transform, or its
    // amplitude in the single weighted transform.
    std::vector<double> strength(p->nspecies, 1.0);
    if (p->ntr == 1 && !d->partials && !xray) strength = p->amp_sp;
    std::vector<double> amp_tr(p->ntr, 1.0), xc_tr(9 * (size_t)p->ntr, 0.0);
    if (p->ntr > 1 || d->partials || xray) {
      amp_tr = p->amp_sp;
      xc_tr = p->xcoef_sp;
    }
    std::vector<double> cnt_sp(p->nspecies);
    for (int k = 0; k < p->nspecies; ++k) cnt_sp[k] = (double)p->type_counts[p->species_type[k] - 1];
    if (p->fp64) {
      e = cudaMemcpy(p->d_strength, strength.data(), strength.size() * 8, cudaMemcpyHostToDevice);
    } else {
      std::vector<float> f = to_r<float>(strength);
      e = cudaMemcpy(p->d_strength, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(p->d_amp, amp_tr.data(), amp_tr.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_xcoef, xc_tr.data(), xc_tr.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_amp_sp, p->amp_sp.data(), p->amp_sp.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_xcoef_sp, p->xcoef_sp.data(), p->xcoef_sp.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_counts_sp, cnt_sp.data(), cnt_sp.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return SQN_ERR_CUDA;
  }
  if (cudaMemsetAsync(p->d_counts, 0, sizeof(int) * (size_t)p->nkeys, s) != cudaSuccess ||
      cudaMemsetAsync(p->d_acc, 0, sizeof(double) * (size_t)p->nsums, s) != cudaSuccess ||
      cudaMemsetAsync(p->d_den, 0, sizeof(double) * (size_t)d->nq, s) != cudaSuccess ||
      cudaMemsetAsync(p->d_cnt, 0, sizeof(double) * (size_t)d->nq, s) != cudaSuccess)
    return SQN_ERR_CUDA;
  if (p->d_gnum &&
      cudaMemsetAsync(p->d_gnum, 0, sizeof(double) * (size_t)p->gnum_half, s) != cudaSuccess)
    return SQN_ERR_CUDA;
  if (p->d_xcnt &&
      cudaMemsetAsync(p->d_xcnt, 0, sizeof(double) * (size_t)b.xbins, s) != cudaSuccess)
    return SQN_ERR_CUDA;

  // --- rows, shell normalisation, kept-mode count --------------------------
  std::vector<int4> rows = build_rows(p->recip, p->hm, d->qmax);
  p->nrows = (int)rows.size();
  if (p->nrows == 0) return SQN_ERR_NO_MODES;
  if ((st = dalloc(p, &p->d_rows, rows.size()))) return st;
  if (cudaMemcpy(p->d_rows, rows.data(), rows.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess)
    return SQN_ERR_CUDA;
  {
    BinGeom nb = b;
    nb.ntr = p->nspecies;
    nb.xray = xray ? 1 : 0;
    if (launch_norms(p->d_rows, p->nrows, nb, p->d_amp_sp, p->d_xcoef_sp, p->d_counts_sp, p->d_den,
                     p->d_cnt, p->d_xcnt, p->nsm, s) != cudaSuccess)
      return SQN_ERR_CUDA;
    p->launches++;
    p->den.assign(d->nq, 0.0);
    p->cnt.assign(d->nq, 0.0);
    if (cudaMemcpyAsync(p->den.data(), p->d_den, sizeof(double) * d->nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(p->cnt.data(), p->d_cnt, sizeof(double) * d->nq, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return SQN_ERR_CUDA;
    double tot = 0.0;
    for (double c : p->cnt) tot += c;
    p->nmodes = (int64_t)std::llround(tot);
    if (p->nmodes == 0) return SQN_ERR_NO_MODES;
  }

  // --- cuFFT: batched 3D real-to-complex, out of place --------------------
  {
    if (cufftCreate(&p->fft) != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
    p->fft_ok = true;
    long long n[3] = {p->nf[2], p->nf[1], p->nf[0]};
    long long inembed[3] = {p->nf[2], p->nf[1], g.pitch};
    long long onembed[3] = {p->nf[2], p->nf[1], b.c1};
    size_t ws = 0;
    if (cufftMakePlanMany64(p->fft, 3, n, inembed, 1, g.vol_real, onembed, 1, b.vol_cplx,
                            p->fp64 ? CUFFT_D2Z : CUFFT_R2C, p->ntr, &ws) != CUFFT_SUCCESS)
      return SQN_ERR_CUFFT;
    p->device_bytes += (int64_t)ws;
    if (cufftSetStream(p->fft, s) != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
  }

  // --- pruned 512-point passes -------------------------------------------------
  // cuFFT stays for plans that ask for it, dS/dr plans (in-place spectra)
  // and other grid sizes.
  if (!p->inplace && !(d->flags & SQN_FLAG_CUFFT) && p->nf[0] == 512 &&
      p->nf[1] == 512 && p->nf[2] == 512) {
    std::vector<double> tw;
    fft512_twiddles(tw);
    char *v;
    if ((st = dalloc(p, &v, tw.size() * rsz))) return st;
    p->d_tw512 = v;
    cudaError_t ce;
    if (p->fp64) {
      ce = cudaMemcpy(v, tw.data(), tw.size() * 8, cudaMemcpyHostToDevice);
      if (ce == cudaSuccess) ce = fft512_set_attributes<double>();
    } else {
      std::vector<float> f = to_r<float>(tw);
      ce = cudaMemcpy(v, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
      if (ce == cudaSuccess) ce = fft512_set_attributes<float>();
    }
    if (ce != cudaSuccess) return SQN_ERR_CUDA;
    p->bg512 = b;
    p->bg512.nf[1] = 2 * p->hm[1] + 1;
    p->bg512.nf[2] = 2 * p->hm[2] + 1;
    // rows of the compact spectrum padded to 16 complex values (128-byte
    // aligned segments for the column passes); h1 = 0 .. hm0 used
    p->bg512.c1 = ((p->hm[0] + 1) + 15) / 16 * 16;
    p->bg512.vol_cplx = p->bg512.c1 * p->bg512.nf[1] * p->bg512.nf[2];
    // columns (h1, h2) the binning reads: h1 <= the largest kept h1 over the rows
    // with that h2 (the rows' h1 ranges are conservative supersets)
    {
      const int M2 = 2 * p->hm[1] + 1;
      std::vector<int> h1end((size_t)M2, 0);
      for (const int4 &r : build_rows(p->recip, p->hm, d->qmax)) {
        const int h2w = r.x >= 0 ? r.x : M2 + r.x;
        h1end[(size_t)h2w] = std::max(h1end[(size_t)h2w], r.w + 1);
      }
      if ((st = dalloc(p, &p->d_h1end, h1end.size()))) return st;
      if (cudaMemcpy(p->d_h1end, h1end.data(), h1end.size() * sizeof(int),
                     cudaMemcpyHostToDevice) != cudaSuccess)
        return SQN_ERR_CUDA;
      // per 16-column block of h1 (from h1 = 16 j): the h2 some column of it needs
      // (h1end[h2] > 16 j), as one band [lo, hi] (empty: lo > hi)
      const int nblk = (p->hm[0] + 1 + 15) / 16;
      std::vector<short2> band((size_t)nblk, make_short2(1, 0));
      for (int j = 0; j < nblk; ++j)
        for (int hw = 0; hw < M2; ++hw)
          if (h1end[(size_t)hw] > 16 * j) {
            const short h2 = (short)(hw <= p->hm[1] ? hw : hw - M2);
            short2 &e = band[(size_t)j];
            if (e.x > e.y) e = make_short2(h2, h2);
            else e = make_short2(std::min(e.x, h2), std::max(e.y, h2));
          }
      if ((st = dalloc(p, &p->d_h2band, band.size()))) return st;
      if (cudaMemcpy(p->d_h2band, band.data(), band.size() * sizeof(short2),
                     cudaMemcpyHostToDevice) != cudaSuccess)
        return SQN_ERR_CUDA;
    }
    p->fft512 = true;
  }

  // --- adjoint buffers (dS/dr) -----------------------------------------------
  if (d->flags & SQN_FLAG_GRAD) {
    if (xray) return SQN_ERR_NOT_SUPPORTED;
    char *v;
    if ((st = dalloc(p, &p->d_orig, (size_t)N))) return st;
    if ((st = dalloc(p, &v, (size_t)3 * b.vol_cplx * 2 * rsz))) return st;
    p->d_F = v;
    if ((st = dalloc(p, &v, (size_t)3 * g.vol_real * rsz))) return st;
    p->d_U = v;
    if ((st = dalloc(p, &v, (size_t)p->nspecies * rsz))) return st;
    p->d_wstrength = v;
    if ((st = dalloc(p, &p->d_grad, (size_t)3 * N))) return st;
    if ((st = dalloc(p, &p->d_gsh, (size_t)d->nq))) return st;
    if ((st = dalloc(p, &p->d_num1, (size_t)d->nq))) return st;
    cudaError_t ce;
    if (p->fp64) {
      ce = cudaMemcpy(p->d_wstrength, p->amp_sp.data(), p->amp_sp.size() * 8, cudaMemcpyHostToDevice);
    } else {
      std::vector<float> f = to_r<float>(p->amp_sp);
      ce = cudaMemcpy(p->d_wstrength, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
    }
    if (ce != cudaSuccess) return SQN_ERR_CUDA;
    long long n[3] = {p->nf[2], p->nf[1], p->nf[0]};
    long long rembed[3] = {p->nf[2], p->nf[1], g.pitch};
    long long cembed[3] = {p->nf[2], p->nf[1], b.c1};
    size_t ws = 0;
    if (cufftCreate(&p->fft_fwd1) != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
    p->fft_fwd1_ok = true;
    if (cufftMakePlanMany64(p->fft_fwd1, 3, n, rembed, 1, g.vol_real, cembed, 1, b.vol_cplx,
                            p->fp64 ? CUFFT_D2Z : CUFFT_R2C, 1, &ws) != CUFFT_SUCCESS)
      return SQN_ERR_CUFFT;
    p->device_bytes += (int64_t)ws;
    if (cufftCreate(&p->fft_inv3) != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
    p->fft_inv3_ok = true;
    if (cufftMakePlanMany64(p->fft_inv3, 3, n, cembed, 1, b.vol_cplx, rembed, 1, g.vol_real,
                            p->fp64 ? CUFFT_Z2D : CUFFT_C2R, 3, &ws) != CUFFT_SUCCESS)
      return SQN_ERR_CUFFT;
    p->device_bytes += (int64_t)ws;
    if (cufftSetStream(p->fft_fwd1, s) != CUFFT_SUCCESS ||
        cufftSetStream(p->fft_inv3, s) != CUFFT_SUCCESS)
      return SQN_ERR_CUFFT;
    p->grad_ok = true;
  }

  if (cudaStreamSynchronize(s) != cudaSuccess) return SQN_ERR_CUDA;
  return warn;
}

// Kernels of ours that one frame launches.
int frame_launches(const sqn_plan *p) { return p->fft512 ? 8 : 5; }

// All queued work of the plan finished.
int sync_plan(sqn_plan *p) {
  if (cudaStreamSynchronize(p->stream) != cudaSuccess) return SQN_ERR_CUDA;
  return SQN_OK;
}

// The frame plan's forward transform of `in` into `out` on stream s.
cufftResult exec_forward(sqn_plan *p, cudaStream_t s, void *in, void *out) {
  cufftResult fr = cufftSetStream(p->fft, s);
  if (fr != CUFFT_SUCCESS) return fr;
  return p->fp64 ? cufftExecD2Z(p->fft, (cufftDoubleReal *)in, (cufftDoubleComplex *)out)
                 : cufftExecR2C(p->fft, (cufftReal *)in, (cufftComplex *)out);
}

template <typename R> int grad_frame(sqn_plan *p, const double *dpos, bool want_grad) {
  cudaStream_t s = p->stream;
  FrameGeom g = p->fg;
  g.ntr = 1;  // the total T(h) = sum_j c_j exp(i q.r_j): one weighted transform
  g.chunk = spread_chunk(p->fp64);
  BinGeom b = p->bg;
  b.ntr = 1;
  b.partials = 0;
  b.want_grid = 0;
  b.nquant = 1;
  cudaError_t e = launch_prep<R>(dpos, p->d_species, g, p->d_counts, p->d_key, p->d_slot, s);
  if (e == cudaSuccess) e = launch_scan(p->d_counts, p->d_starts, p->nkeys, s);
  if (e == cudaSuccess)
    e = launch_scatter<R>(dpos, p->d_species, g, p->d_key, p->d_slot, p->d_starts,
                          (R *)p->d_recs, p->d_orig, s);
  if (e == cudaSuccess)
    e = launch_spread<R>((const R *)p->d_recs, p->d_starts, g, (const R *)p->d_wstrength,
                         (R *)p->d_grid, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  cufftResult fr = p->fp64 ? cufftExecD2Z(p->fft_fwd1, (cufftDoubleReal *)p->d_grid,
                                          (cufftDoubleComplex *)p->d_G)
                           : cufftExecR2C(p->fft_fwd1, (cufftReal *)p->d_grid, (cufftComplex *)p->d_G);
  if (fr != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
  if (cudaMemsetAsync(p->d_num1, 0, sizeof(double) * (size_t)b.nq, s) != cudaSuccess)
    return SQN_ERR_CUDA;
  if (want_grad &&
      cudaMemsetAsync(p->d_F, 0, (size_t)3 * b.vol_cplx * 2 * sizeof(R), s) != cudaSuccess)
    return SQN_ERR_CUDA;
  e = launch_adj_coef<R>(p->d_rows, p->nrows, p->d_G, b, (const R *)p->d_inv[0],
                         (const R *)p->d_inv[1], (const R *)p->d_inv[2], p->d_gsh, p->d_num1,
                         want_grad ? p->d_F : nullptr, p->nsm, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  p->launches += 5;
  if (!want_grad) return SQN_OK;
  fr = p->fp64 ? cufftExecZ2D(p->fft_inv3, (cufftDoubleComplex *)p->d_F, (cufftDoubleReal *)p->d_U)
               : cufftExecC2R(p->fft_inv3, (cufftComplex *)p->d_F, (cufftReal *)p->d_U);
  if (fr != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
  Recip rb;
  std::memcpy(rb.b, p->recip, sizeof(rb.b));
  e = launch_interp<R>((const R *)p->d_recs, p->d_orig, dpos, p->fg, (const R *)p->d_U, rb,
                       p->d_amp_sp, p->d_grad, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  p->launches += 1;
  return SQN_OK;
}

// One frame's per-species spectra (sort, spread, R2C) without binning, then
// the density amplitudes of the requested lattice points.
template <typename R> int density_frame(sqn_plan *p, const double *dpos, int64_t nm) {
  const FrameGeom &g = p->fg;
  cudaStream_t s = p->stream;
  cudaError_t e = launch_prep<R>(dpos, p->d_species, g, p->d_counts, p->d_key, p->d_slot, s);
  if (e == cudaSuccess) e = launch_scan(p->d_counts, p->d_starts, p->nkeys, s);
  if (e == cudaSuccess)
    e = launch_scatter<R>(dpos, p->d_species, g, p->d_key, p->d_slot, p->d_starts,
                          (R *)p->d_recs, nullptr, s);
  if (e == cudaSuccess)
    e = launch_spread<R>((const R *)p->d_recs, p->d_starts, g, (const R *)p->d_strength,
                         (R *)p->d_grid, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  if (exec_forward(p, s, p->d_grid, p->d_G) != CUFFT_SUCCESS) return SQN_ERR_CUFFT;
  e = launch_gather_modes<R>(p->d_G, p->bg, p->d_hkl, nm, (const R *)p->d_inv[0],
                             (const R *)p->d_inv[1], (const R *)p->d_inv[2], p->origin,
                             p->d_rho, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  p->launches += 5;
  return SQN_OK;
}

template <typename R> int run_frame(sqn_plan *p, const double *dpos, int slot) {
  const FrameGeom &g = p->fg;
  cudaStream_t s = p->stream;
  cudaEvent_t ev[5] = {};
  if (p->timing) {
    while (p->tev_pool.size() < p->tev_used + 5) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return SQN_ERR_CUDA;
      p->tev_pool.push_back(e);
    }
    for (int i = 0; i < 5; ++i) ev[i] = p->tev_pool[p->tev_used + i];
    p->tev_used += 5;
    cudaEventRecord(ev[0], s);
  }
  cudaError_t e = launch_prep<R>(dpos, p->d_species, g, p->d_counts, p->d_key, p->d_slot, s);
  if (e == cudaSuccess) e = launch_scan(p->d_counts, p->d_starts, p->nkeys, s);
  if (e == cudaSuccess)
    e = launch_scatter<R>(dpos, p->d_species, g, p->d_key, p->d_slot, p->d_starts,
                          (R *)p->d_recs, nullptr, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  if (slot >= 0) cudaEventRecord(p->ev_free[slot], s);
  if (p->timing) cudaEventRecord(ev[1], s);
  void *grid = p->d_grid;
  e = launch_spread<R>((const R *)p->d_recs, p->d_starts, g, (const R *)p->d_strength, (R *)grid,
                       s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  if (p->timing) cudaEventRecord(ev[2], s);
  if (p->fft512) {
    // x pass into d_G, y pass back into the (consumed) grid, z pass into d_G
    e = launch_fft512<R>((const R *)grid, p->d_G, grid, p->d_G, p->ntr, g.pitch, p->hm[0] + 1,
                         (int)p->bg512.c1, p->hm[1], p->hm[2], p->d_tw512, p->d_h1end,
                         p->d_h2band, p->nsm, s);
    if (e != cudaSuccess) return SQN_ERR_CUDA;
    p->launches += 3;
  } else if (exec_forward(p, s, grid, p->d_G) != CUFFT_SUCCESS) {
    return SQN_ERR_CUFFT;
  }
  if (p->timing) cudaEventRecord(ev[3], s);
  e = launch_bin<R>(p->d_rows, p->nrows, p->d_G, p->fft512 ? p->bg512 : p->bg,
                    (const R *)p->d_inv[0], (const R *)p->d_inv[1], (const R *)p->d_inv[2],
                    p->d_amp, p->d_xcoef, p->d_acc, p->d_gnum, p->nsm, s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  if (p->timing) cudaEventRecord(ev[4], s);
  p->launches += 5;
  p->nframes++;
  return SQN_OK;
}

void harvest_timing(sqn_plan *p) {
  for (size_t k = 0; k + 5 <= p->tev_used; k += 5) {
    for (int st = 0; st < 4; ++st) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p->tev_pool[k + st], p->tev_pool[k + st + 1]) == cudaSuccess)
        p->stage_ms[st] += ms;
      else
        cudaGetLastError();
    }
    p->stage_frames++;
  }
  p->tev_used = 0;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// Entry points
// ---------------------------------------------------------------------------

extern "C" {

int sqn_abi_version(void) { return SQN_ABI_VERSION; }

const char *sqn_error_string(int code) {
  switch (code) {
    case SQN_OK: return "ok";
    case SQN_WARN_EPS_TOO_SMALL: return "warning: requested tolerance below what the precision or kernel width can reach";
    case SQN_ERR_UPSAMPFAC_TOO_SMALL: return "upsampling factor must exceed 1";
    case SQN_ERR_ALLOC: return "device memory allocation failed";
    case SQN_ERR_CUDA: return "CUDA runtime error";
    case SQN_ERR_PLAN_NOTVALID: return "invalid plan";
    case SQN_ERR_NUM_NU_PTS_INVALID: return "invalid number of atoms";
    case SQN_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SQN_ERR_ABI_MISMATCH: return "descriptor ABI version does not match the library";
    case SQN_ERR_NO_DEVICE: return "no usable CUDA device";
    case SQN_ERR_GRID_TOO_LARGE: return "reciprocal grid exceeds the mode limit; reduce --qmax";
    case SQN_ERR_NO_MODES: return "no reciprocal lattice points fall inside the requested q range";
    case SQN_ERR_DEGENERATE_CELL: return "degenerate simulation cell";
    case SQN_ERR_TYPE_ID: return "atom type id outside 1..ntypes";
    case SQN_ERR_CUFFT: return "cuFFT failure";
    case SQN_ERR_DUMP: return "dump file unreadable or malformed";
    case SQN_ERR_TIMEOUT: return "device wait timed out";
    case SQN_ERR_NOT_SUPPORTED: return "configuration not supported by this build";
    default: return "unknown status";
  }
}

void sqn_default_desc(sqn_plan_desc *d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->abi_version = SQN_ABI_VERSION;
  d->qmin = 0.0;
  d->qmax = 20.0;
  d->nq = 500;
  d->eps = 1e-9;
  d->norm = SQN_NORM_MEAN;
  d->partials = 1;
  d->weight = SQN_WEIGHT_UNIT;
  d->precision = SQN_PREC_DOUBLE;
  d->xrd_lambda = 0.0;
  d->xrd_2theta_min = 1.0;
  d->xrd_2theta_max = 179.0;
  d->xrd_step = 0.0;
  d->xrd_lp = 1;
}

int sqn_plan_create(const sqn_plan_desc *desc, sqn_plan **out) {
  if (!out) return SQN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!desc) return SQN_ERR_INVALID_ARGUMENT;
  if (desc->abi_version != SQN_ABI_VERSION) return SQN_ERR_ABI_MISMATCH;
  sqn_plan *p = new (std::nothrow) sqn_plan_s();
  if (!p) return SQN_ERR_ALLOC;
  int prev = -1;
  cudaGetDevice(&prev);
  int st = setup_plan(p, desc);
  if (st > SQN_WARN_EPS_TOO_SMALL) {
    free_plan(p);
    if (prev >= 0) cudaSetDevice(prev);
    return st;
  }
  if (prev >= 0) cudaSetDevice(prev);
  *out = p;
  return st;
}

int sqn_plan_info_get(const sqn_plan *p, sqn_plan_info *info) {
  if (!p || !info) return SQN_ERR_INVALID_ARGUMENT;
  std::memset(info, 0, sizeof(*info));
  for (int i = 0; i < 3; ++i) {
    info->modes[i] = p->modes[i];
    info->nf[i] = p->nf[i];
    info->tile[i] = p->fg.tile[i];
  }
  info->kernel_width = p->w;
  info->gridpoints = p->gridpoints;
  info->nmodes = p->nmodes;
  info->upsampfac = p->sigma;
  info->beta = p->beta;
  info->eps_used = p->eps_used;
  info->ntransforms = p->ntr;
  info->nspecies = p->nspecies;
  info->device_bytes = p->device_bytes;
  info->pruned_fft512 = p->fft512 ? 1 : 0;
  info->natoms = p->desc.natoms;
  info->xrd_bins = p->bg.xrd ? p->bg.xbins : 0;
  info->xrd_step = p->bg.xrd ? p->bg.xstep : 0.0;
  info->autotuned = p->autotuned;
  info->tune_candidates = p->tune_candidates;
  info->tune_ms = p->tune_ms;
  return SQN_OK;
}

int sqn_accumulate_frames(sqn_plan *p, const double *pos, int64_t nframes, int32_t where) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!pos || nframes < 0 || (where != SQN_HOST && where != SQN_DEVICE))
    return SQN_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(p->device);
  const int64_t N = p->desc.natoms;
  const size_t bytes = sizeof(double) * 3 * (size_t)N;
  int last_slot = -1;
  for (int64_t f = 0; f < nframes; ++f) {
    const double *dpos;
    int slot = -1;
    if (where == SQN_HOST) {
      slot = p->slot_next;
      p->slot_next ^= 1;
      // Double buffer: the copy into this slot waits until the frame that used
      // it last has been sorted, and runs beside the previous frame's spread/FFT.
      if (cudaStreamWaitEvent(p->copy_stream, p->ev_free[slot], 0) != cudaSuccess ||
          cudaMemcpyAsync(p->d_pos[slot], pos + 3 * (size_t)N * f, bytes, cudaMemcpyHostToDevice,
                          p->copy_stream) != cudaSuccess ||
          cudaEventRecord(p->ev_copied[slot], p->copy_stream) != cudaSuccess ||
          cudaStreamWaitEvent(p->stream, p->ev_copied[slot], 0) != cudaSuccess)
        return SQN_ERR_CUDA;
      dpos = p->d_pos[slot];
      last_slot = slot;
    } else {
      dpos = pos + 3 * (size_t)N * f;
    }
    const int st = p->fp64 ? run_frame<double>(p, dpos, slot) : run_frame<float>(p, dpos, slot);
    if (st != SQN_OK) return st;
  }
  // Host positions must have been read before the call returns.
  if (last_slot >= 0 && cudaEventSynchronize(p->ev_copied[last_slot]) != cudaSuccess)
    return SQN_ERR_CUDA;
  return SQN_OK;
}

int sqn_join(sqn_plan *p) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  DeviceGuard guard(p->device);
  return SQN_OK;  // every kernel of the plan runs on its one stream
}

int sqn_sync(sqn_plan *p) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  DeviceGuard guard(p->device);
  return sync_plan(p);
}

int sqn_peek_num_async(sqn_plan *p, double *num_host) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!num_host) return SQN_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(p->device);
  // after the binning of the queued frames, on the stream that runs it
  cudaStream_t s = p->stream;
  return cuda_status(cudaMemcpyAsync(num_host, p->d_acc, sizeof(double) * p->desc.nq,
                                     cudaMemcpyDeviceToHost, s));
}

int sqn_get_accumulators(sqn_plan *p, double *num, double *den, int64_t *shell_count,
                         double *partial_num, double *gnum, double *gden, int64_t *nframes) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  DeviceGuard guard(p->device);
  if (sync_plan(p) != SQN_OK) return SQN_ERR_CUDA;
  const int nq = p->desc.nq, T = p->desc.ntypes;
  std::vector<double> acc((size_t)p->nquant * nq);
  if (cudaMemcpy(acc.data(), p->d_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return SQN_ERR_CUDA;
  if (num) std::memcpy(num, acc.data(), sizeof(double) * nq);
  if (den) std::memcpy(den, p->den.data(), sizeof(double) * nq);
  if (shell_count)
    for (int s = 0; s < nq; ++s) shell_count[s] = (int64_t)std::llround(p->cnt[s]);
  if (partial_num) {
    std::memset(partial_num, 0, sizeof(double) * (size_t)T * T * nq);
    if (p->desc.partials) {
      int q = 1;
      for (int a = 0; a < p->ntr; ++a)
        for (int c = a; c < p->ntr; ++c, ++q) {
          const int ta = p->species_type[a], tb = p->species_type[c];
          for (int s = 0; s < nq; ++s)
            partial_num[(size_t)(ta - 1) + (size_t)T * ((size_t)(tb - 1) + (size_t)T * s)] =
                acc[(size_t)q * nq + s];
        }
    }
  }
  if (gnum || gden) {
    if (!p->desc.want_grid) return SQN_ERR_INVALID_ARGUMENT;
    std::vector<double> half((size_t)p->gnum_half);
    if (gnum &&
        cudaMemcpy(half.data(), p->d_gnum, half.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      return SQN_ERR_CUDA;
    const int *m = p->modes, *hm = p->hm;
    const bool xray = p->desc.weight == SQN_WEIGHT_XRAY;
    int64_t g = 0;
    for (int p3 = 1; p3 <= m[2]; ++p3)
      for (int p2 = 1; p2 <= m[1]; ++p2)
        for (int p1 = 1; p1 <= m[0]; ++p1, ++g) {
          int h1 = p1 - (m[0] + 1) / 2, h2 = p2 - (m[1] + 1) / 2, h3 = p3 - (m[2] + 1) / 2;
          if (gnum) {
            int a1 = h1, a2 = h2, a3 = h3;
            if (h1 < 0) { a1 = -h1; a2 = -h2; a3 = -h3; }
            gnum[g] = half[((size_t)(a3 + hm[2]) * m[1] + (size_t)(a2 + hm[1])) * (hm[0] + 1) + a1];
          }
          if (gden) {
            gden[g] = 0.0;
            if (h1 == 0 && h2 == 0 && h3 == 0) continue;
            const double ql = qlen_ref(p->recip, h1, h2, h3);
            if (ql > p->desc.qmax || ql < p->desc.qmin) continue;
            double dd;
            if (p->desc.norm == SQN_NORM_NATOM) {
              dd = (double)p->desc.natoms;
            } else {
              double sw = 0.0, sw2 = 0.0;
              for (int k = 0; k < p->nspecies; ++k) {
                const double w = xray ? xray_f_host(&p->xcoef_sp[9 * k], ql) : p->amp_sp[k];
                const double c = (double)p->type_counts[p->species_type[k] - 1];
                sw = sw + c * w;
                sw2 = sw2 + c * w * w;
              }
              dd = p->desc.norm == SQN_NORM_MEAN ? sw * sw / (double)p->desc.natoms : sw2;
            }
            gden[g] = dd;
          }
        }
  }
  if (nframes) *nframes = p->nframes;
  return SQN_OK;
}

int sqn_finalize(sqn_plan *p, int32_t faber_ziman, double *S_total, double *S_partial,
                 double *S_grid, int64_t *nframes) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  const int nq = p->desc.nq, T = p->desc.ntypes;
  std::vector<double> num(nq), den(nq), pn;
  std::vector<int64_t> cnt(nq);
  if (S_partial) pn.resize((size_t)T * T * nq);
  int st = sqn_get_accumulators(p, num.data(), den.data(), cnt.data(),
                                S_partial ? pn.data() : nullptr, nullptr, nullptr, nullptr);
  if (st) return st;
  const double frames = (double)std::max<int64_t>(p->nframes, 1);
  if (S_total)
    for (int s = 0; s < nq; ++s) S_total[s] = den[s] > 0.0 ? num[s] / (frames * den[s]) : 0.0;
  if (S_partial) {
    const double N = (double)p->desc.natoms;
    for (int s = 0; s < nq; ++s)
      for (int ib = 1; ib <= T; ++ib)
        for (int ia = 1; ia <= T; ++ia) {
          const size_t k = (size_t)(ia - 1) + (size_t)T * ((size_t)(ib - 1) + (size_t)T * s);
          double v = pn[k] / (frames * N * (double)std::max<int64_t>(cnt[s], 1));
          if (faber_ziman) {
            const double xa = (double)p->type_counts[ia - 1] / N, xb = (double)p->type_counts[ib - 1] / N;
            v = xa * xb <= 0.0 ? 0.0 : (v - (ia == ib ? xa : 0.0)) / (xa * xb) + 1.0;
          }
          S_partial[k] = v;
        }
  }
  if (S_grid) {
    if (!p->desc.want_grid) return SQN_ERR_INVALID_ARGUMENT;
    std::vector<double> gnum((size_t)p->gridpoints), gden((size_t)p->gridpoints);
    st = sqn_get_accumulators(p, nullptr, nullptr, nullptr, nullptr, gnum.data(), gden.data(), nullptr);
    if (st) return st;
    const int *m = p->modes;
    int64_t g = 0, im = 0;
    for (int p3 = 1; p3 <= m[2]; ++p3)
      for (int p2 = 1; p2 <= m[1]; ++p2)
        for (int p1 = 1; p1 <= m[0]; ++p1, ++g) {
          const int h1 = p1 - (m[0] + 1) / 2, h2 = p2 - (m[1] + 1) / 2, h3 = p3 - (m[2] + 1) / 2;
          if (h1 == 0 && h2 == 0 && h3 == 0) continue;
          const double ql = qlen_ref(p->recip, h1, h2, h3);
          if (ql > p->desc.qmax || ql < p->desc.qmin) continue;
          S_grid[im++] = gden[g] > 0.0 ? gnum[g] / (frames * gden[g]) : 0.0;
        }
  }
  if (nframes) *nframes = p->nframes;
  return SQN_OK;
}

int sqn_density_modes(sqn_plan *p, const double *pos, int32_t where, const int32_t *hkl,
                      int64_t nmodes, double *rho) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!pos || !hkl || !rho || nmodes < 1 || (where != SQN_HOST && where != SQN_DEVICE))
    return SQN_ERR_INVALID_ARGUMENT;
  // unit-strength transform per species, on the cuFFT spectrum
  if (p->ntr != p->nspecies || !(p->desc.partials || p->bg.xray))
    return SQN_ERR_NOT_SUPPORTED;
  DeviceGuard guard(p->device);
  cudaStream_t s = p->stream;
  if (sync_plan(p) != SQN_OK || cudaStreamSynchronize(p->copy_stream) != cudaSuccess)
    return SQN_ERR_CUDA;
  if (nmodes > p->modes_cap) {
    if (p->d_hkl) cudaFree(p->d_hkl);
    if (p->d_rho) cudaFree(p->d_rho);
    p->d_hkl = nullptr;
    p->d_rho = nullptr;
    p->modes_cap = 0;
    if (cudaMalloc(&p->d_hkl, sizeof(int) * 3 * (size_t)nmodes) != cudaSuccess ||
        cudaMalloc(&p->d_rho, sizeof(double) * 2 * (size_t)p->ntr * nmodes) != cudaSuccess) {
      cudaGetLastError();
      return SQN_ERR_ALLOC;
    }
    p->modes_cap = nmodes;
  }
  const int64_t N = p->desc.natoms;
  const double *dpos = pos;
  if (where == SQN_HOST) {
    if (cudaMemcpyAsync(p->d_pos[0], pos, sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice,
                        s) != cudaSuccess)
      return SQN_ERR_CUDA;
    dpos = p->d_pos[0];
  }
  if (cudaMemcpyAsync(p->d_hkl, hkl, sizeof(int) * 3 * (size_t)nmodes, cudaMemcpyHostToDevice,
                      s) != cudaSuccess)
    return SQN_ERR_CUDA;
  const int st = p->fp64 ? density_frame<double>(p, dpos, nmodes)
                         : density_frame<float>(p, dpos, nmodes);
  if (st != SQN_OK) return st;
  if (cudaMemcpyAsync(rho, p->d_rho, sizeof(double) * 2 * (size_t)p->ntr * nmodes,
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return SQN_ERR_CUDA;
  return SQN_OK;
}

int sqn_get_xrd(sqn_plan *p, double *two_theta, double *I, double *I_partial, int64_t *count,
                int64_t *nframes) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  const BinGeom &b = p->bg;
  if (!b.xrd) return SQN_ERR_NOT_SUPPORTED;
  DeviceGuard guard(p->device);
  if (sync_plan(p) != SQN_OK) return SQN_ERR_CUDA;
  const int nb = b.xbins, T = p->desc.ntypes;
  std::vector<double> xs((size_t)b.xquant * nb), xc((size_t)nb);
  if (cudaMemcpy(xs.data(), p->d_acc + (size_t)b.nquant * b.nq, xs.size() * sizeof(double),
                 cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(xc.data(), p->d_xcnt, xc.size() * sizeof(double), cudaMemcpyDeviceToHost) !=
          cudaSuccess)
    return SQN_ERR_CUDA;
  // per atom and per frame (sf_write_xrd, src/sqc_structure_factor.f90:1008-1027)
  const double norm = (double)std::max<int64_t>(p->nframes, 1) * (double)p->desc.natoms;
  for (int k = 0; k < nb; ++k) {
    if (two_theta) two_theta[k] = b.xmin + ((double)k + 0.5) * b.xstep;
    if (I) I[k] = xs[(size_t)k] / norm;
    if (count) count[k] = (int64_t)std::llround(xc[(size_t)k]);
  }
  if (I_partial) {
    std::memset(I_partial, 0, sizeof(double) * (size_t)T * T * nb);
    if (p->desc.partials) {
      int q = 1;
      for (int a = 0; a < p->ntr; ++a)
        for (int c = a; c < p->ntr; ++c, ++q) {
          const int ta = p->species_type[a], tb = p->species_type[c];
          for (int k = 0; k < nb; ++k)
            I_partial[(size_t)(ta - 1) + (size_t)T * ((size_t)(tb - 1) + (size_t)T * k)] =
                xs[(size_t)q * nb + k] / norm;
        }
    }
  }
  if (nframes) *nframes = p->nframes;
  return SQN_OK;
}

int sqn_accumulator_view(sqn_plan *p, double **acc, int64_t *count, int64_t *nframes) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!acc || !count) return SQN_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(p->device);
  if (sync_plan(p) != SQN_OK) return SQN_ERR_CUDA;
  *acc = p->d_acc;
  *count = p->nsums + p->gnum_half;
  if (nframes) *nframes = p->nframes;
  return SQN_OK;
}

int sqn_set_frame_count(sqn_plan *p, int64_t nframes) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (nframes < 0) return SQN_ERR_INVALID_ARGUMENT;
  p->nframes = nframes;
  return SQN_OK;
}

int sqn_reset(sqn_plan *p) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  DeviceGuard guard(p->device);
  if (sync_plan(p) != SQN_OK) return SQN_ERR_CUDA;
  cudaError_t e = cudaMemset(p->d_acc, 0, sizeof(double) * ((size_t)p->nsums + (size_t)p->gnum_half));
  p->nframes = 0;
  p->tev_used = 0;
  for (double &v : p->stage_ms) v = 0.0;
  p->stage_frames = 0;
  return cuda_status(e);
}

int sqn_stage_times(sqn_plan *p, double *out, int32_t n) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!out || n < 1) return SQN_ERR_INVALID_ARGUMENT;
  if (!p->timing) return SQN_ERR_NOT_SUPPORTED;
  DeviceGuard guard(p->device);
  if (sync_plan(p) != SQN_OK) return SQN_ERR_CUDA;
  harvest_timing(p);
  double v[5] = {p->stage_ms[0], p->stage_ms[1], p->stage_ms[2], p->stage_ms[3], (double)p->stage_frames};
  for (int i = 0; i < n && i < 5; ++i) out[i] = v[i];
  return SQN_OK;
}

int sqn_sq_grad(sqn_plan *p, const double *pos, int32_t where, const double *dLdS, double *S,
                double *grad) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  if (!p->grad_ok) return SQN_ERR_NOT_SUPPORTED;
  if (!pos || (where != SQN_HOST && where != SQN_DEVICE) || (dLdS && !grad))
    return SQN_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(p->device);
  cudaStream_t s = p->stream;
  const int64_t N = p->desc.natoms;
  const int nq = p->desc.nq;
  const double *dpos = pos;
  if (where == SQN_HOST) {
    // the copy stream may still be filling this slot for an earlier call
    if (cudaStreamSynchronize(p->copy_stream) != cudaSuccess ||
        cudaMemcpyAsync(p->d_pos[0], pos, sizeof(double) * 3 * (size_t)N, cudaMemcpyHostToDevice,
                        s) != cudaSuccess)
      return SQN_ERR_CUDA;
    dpos = p->d_pos[0];
  }
  std::vector<double> gsh(nq, 0.0);
  if (dLdS)
    for (int k = 0; k < nq; ++k) gsh[k] = p->den[k] > 0.0 ? dLdS[k] / p->den[k] : 0.0;
  if (cudaMemcpyAsync(p->d_gsh, gsh.data(), sizeof(double) * nq, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return SQN_ERR_CUDA;
  const int st = p->fp64 ? grad_frame<double>(p, dpos, dLdS != nullptr)
                         : grad_frame<float>(p, dpos, dLdS != nullptr);
  if (st != SQN_OK) return st;
  std::vector<double> num(nq);
  cudaError_t e = cudaMemcpyAsync(num.data(), p->d_num1, sizeof(double) * nq,
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && dLdS)
    e = cudaMemcpyAsync(grad, p->d_grad, sizeof(double) * 3 * (size_t)N,
                        where == SQN_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  if (S)
    for (int k = 0; k < nq; ++k) S[k] = p->den[k] > 0.0 ? num[k] / p->den[k] : 0.0;
  return SQN_OK;
}

int64_t sqn_launch_count(const sqn_plan *p) { return p ? p->launches : -1; }

int sqn_plan_destroy(sqn_plan *p) {
  if (!p) return SQN_ERR_PLAN_NOTVALID;
  free_plan(p);
  return SQN_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches of independent systems behind one CUDA graph
// ---------------------------------------------------------------------------

struct sqn_batch_s {
  int device = 0;
  std::vector<sqn_plan *> plans;
  cudaStream_t root = nullptr;
  bool own_root = false;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t replays = 0;
  // Multi-system path: the sort, the spread and the binning of every system
  // in one launch each (BatchSys table and prefix sums in device memory);
  // the FFTs stay per system, as parallel branches.
  bool multi = false;
  bool fp64 = false;
  int ntr = 0, hist_max = 0;
  bool xray = false;
  int64_t natoms = 0;
  int spread_blocks = 0, bin_blocks = 0;
  BatchSys *d_sys = nullptr;
  int64_t *d_apre = nullptr;
  int *d_spre = nullptr, *d_bpre = nullptr;
  int64_t launches_per_step = 0;  // kernels of ours per frame of every system
  int64_t launches = 0;
};

namespace {

void free_batch(sqn_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->root) cudaStreamSynchronize(b->root);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaEvent_t e : b->joins)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  for (sqn_plan *p : b->plans) free_plan(p);
  if (b->d_sys) cudaFree(b->d_sys);
  if (b->d_apre) cudaFree(b->d_apre);
  if (b->d_spre) cudaFree(b->d_spre);
  if (b->d_bpre) cudaFree(b->d_bpre);
  if (b->own_root && b->root) cudaStreamDestroy(b->root);
  delete b;
}

// The multi-system path needs one precision, one transform count and weight
// kind, no powder pattern and at most MAX_BATCH_SYSTEMS systems.
bool batch_multi_ok(const sqn_batch *b) {
  if (b->plans.empty() || b->plans.size() > (size_t)MAX_BATCH_SYSTEMS) return false;
  const sqn_plan *p0 = b->plans[0];
  for (const sqn_plan *p : b->plans) {
    if (p->fp64 != p0->fp64 || p->ntr != p0->ntr || p->bg.xray != p0->bg.xray || p->bg.xrd ||
        p->inplace || p->ntr > MAX_FAST_T || (size_t)hist_len(p->bg) * 8 > 160 * 1024)
      return false;
  }
  return true;
}

// Build the BatchSys table and the prefix sums of the multi-system launches.
int setup_batch_multi(sqn_batch *b) {
  const size_t n = b->plans.size();
  std::vector<BatchSys> sys(n);
  std::vector<int64_t> apre(n + 1, 0);
  std::vector<int> spre(n + 1, 0), bpre(n + 1, 0);
  constexpr int kRowsPerBinBlock = 256;  // 8 warps x 32 rows
  int64_t sblk = 0, bblk = 0;
  b->hist_max = 0;
  for (size_t k = 0; k < n; ++k) {
    sqn_plan *p = b->plans[k];
    BatchSys &S = sys[k];
    std::memset(&S, 0, sizeof(S));
    S.g = p->fg;
    S.b = p->fft512 ? p->bg512 : p->bg;
    S.pos = p->d_pos[0];
    S.species = p->d_species;
    S.counts = p->d_counts;
    S.starts = p->d_starts;
    S.key = p->d_key;
    S.slot = p->d_slot;
    S.recs = p->d_recs;
    S.strength = p->d_strength;
    S.grid = p->d_grid;
    S.G = p->d_G;
    S.rows = p->d_rows;
    for (int d = 0; d < 3; ++d) S.inv[d] = p->d_inv[d];
    S.amp = p->d_amp;
    S.xcoef = p->d_xcoef;
    S.acc = p->d_acc;
    S.gnum = p->d_gnum;
    S.nkeys = p->nkeys;
    S.nrows = p->nrows;
    apre[k + 1] = apre[k] + p->desc.natoms;
    sblk += (int64_t)p->fg.ntiles * p->ntr;
    bblk += std::max<int64_t>(1, (p->nrows + kRowsPerBinBlock - 1) / kRowsPerBinBlock);
    if (sblk >= INT32_MAX || bblk >= INT32_MAX) return SQN_ERR_NOT_SUPPORTED;
    spre[k + 1] = (int)sblk;
    bpre[k + 1] = (int)bblk;
    b->hist_max = std::max(b->hist_max, hist_len(p->bg));
  }
  b->natoms = apre[n];
  b->spread_blocks = (int)sblk;
  b->bin_blocks = (int)bblk;
  b->fp64 = b->plans[0]->fp64;
  b->ntr = b->plans[0]->ntr;
  b->xray = b->plans[0]->bg.xray != 0;
  if (cudaMalloc(&b->d_sys, n * sizeof(BatchSys)) != cudaSuccess ||
      cudaMalloc(&b->d_apre, (n + 1) * sizeof(int64_t)) != cudaSuccess ||
      cudaMalloc(&b->d_spre, (n + 1) * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&b->d_bpre, (n + 1) * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_ALLOC;
  }
  if (cudaMemcpy(b->d_sys, sys.data(), n * sizeof(BatchSys), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_apre, apre.data(), (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_spre, spre.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_bpre, bpre.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return SQN_ERR_CUDA;
  const cudaError_t e = b->fp64 ? batch_set_attributes<double>(b->ntr, b->xray, b->hist_max)
                                : batch_set_attributes<float>(b->ntr, b->xray, b->hist_max);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  b->multi = true;
  return SQN_OK;
}

// One frame of every system on the multi-system path, queued on the root
// stream: sort and spread of all systems (four launches), the systems' FFTs
// as parallel branches, the binning of all systems (one launch).
template <typename R> int batch_frame_multi(sqn_batch *b) {
  cudaStream_t root = b->root;
  BatchPrefix pre{b->d_apre, b->d_spre, b->d_bpre};
  const int n = (int)b->plans.size();
  cudaError_t e = launch_batch_sort<R>(b->d_sys, n, pre, b->natoms, root);
  if (e == cudaSuccess)
    e = launch_batch_spread<R>(b->d_sys, n, pre, b->spread_blocks, b->plans[0]->fg.chunk, root);
  if (e != cudaSuccess || cudaEventRecord(b->fork, root) != cudaSuccess) return SQN_ERR_CUDA;
  int64_t own = 5;
  for (int k = 0; k < n; ++k) {
    sqn_plan *p = b->plans[k];
    if (cudaStreamWaitEvent(p->stream, b->fork, 0) != cudaSuccess) return SQN_ERR_CUDA;
    if (p->fft512) {
      if (launch_fft512<R>((const R *)p->d_grid, p->d_G, p->d_grid, p->d_G, p->ntr, p->fg.pitch,
                           p->hm[0] + 1, (int)p->bg512.c1, p->hm[1], p->hm[2], p->d_tw512,
                           p->d_h1end, p->d_h2band, p->nsm, p->stream) != cudaSuccess)
        return SQN_ERR_CUDA;
      own += 3;
    } else if (exec_forward(p, p->stream, p->d_grid, p->d_G) != CUFFT_SUCCESS) {
      return SQN_ERR_CUFFT;
    }
    if (cudaEventRecord(b->joins[k], p->stream) != cudaSuccess ||
        cudaStreamWaitEvent(root, b->joins[k], 0) != cudaSuccess)
      return SQN_ERR_CUDA;
  }
  e = launch_batch_bin<R>(b->d_sys, n, pre, b->bin_blocks, b->ntr, b->xray, b->hist_max, root);
  if (e != cudaSuccess) return SQN_ERR_CUDA;
  b->launches_per_step = own;
  return SQN_OK;
}

// One frame of every system, captured once: the root stream forks to each
// system's own stream (its prep, scan, scatter, spread, FFT and bin launches
// form one branch) and joins them again.  Each replay reads the positions
// from the systems' staging buffers d_pos[0].
int capture_batch(sqn_batch *b) {
  cudaStream_t root = b->root;
  if (cudaStreamBeginCapture(root, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return SQN_ERR_CUDA;
  int st = SQN_OK;
  if (b->multi) {
    st = b->fp64 ? batch_frame_multi<double>(b) : batch_frame_multi<float>(b);
  } else if (cudaEventRecord(b->fork, root) != cudaSuccess) {
    st = SQN_ERR_CUDA;
  }
  for (size_t k = 0; k < b->plans.size() && st == SQN_OK && !b->multi; ++k) {
    sqn_plan *p = b->plans[k];
    if (cudaStreamWaitEvent(p->stream, b->fork, 0) != cudaSuccess) {
      st = SQN_ERR_CUDA;
      break;
    }
    st = p->fp64 ? run_frame<double>(p, p->d_pos[0], -1) : run_frame<float>(p, p->d_pos[0], -1);
    // the capture itself accumulates nothing
    p->nframes -= 1;
    p->launches -= frame_launches(p);
    b->launches_per_step += frame_launches(p);
    if (st == SQN_OK && (cudaEventRecord(b->joins[k], p->stream) != cudaSuccess ||
                         cudaStreamWaitEvent(root, b->joins[k], 0) != cudaSuccess))
      st = SQN_ERR_CUDA;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(root, &g);
  if (st != SQN_OK || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return st != SQN_OK ? st : SQN_ERR_CUDA;
  }
  b->graph = g;
  if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    return SQN_ERR_CUDA;
  }
  return SQN_OK;
}

}  // namespace

extern "C" {

int sqn_batch_create(const sqn_plan_desc *descs, int32_t nsystems, void *stream,
                     sqn_batch **out) {
  if (!out) return SQN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!descs || nsystems < 1) return SQN_ERR_INVALID_ARGUMENT;
  for (int32_t k = 1; k < nsystems; ++k)
    if (descs[k].device != descs[0].device) return SQN_ERR_INVALID_ARGUMENT;
  sqn_batch *b = new (std::nothrow) sqn_batch_s();
  if (!b) return SQN_ERR_ALLOC;
  b->device = descs[0].device;
  int prev = -1;
  cudaGetDevice(&prev);
  int warn = SQN_OK;
  int st = cudaSetDevice(b->device) == cudaSuccess ? SQN_OK : SQN_ERR_NO_DEVICE;
  if (st == SQN_OK) {
    if (stream) {
      b->root = (cudaStream_t)stream;
    } else if (cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) == cudaSuccess) {
      b->own_root = true;
    } else {
      st = SQN_ERR_CUDA;
    }
  }
  if (st == SQN_OK && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    st = SQN_ERR_CUDA;
  for (int32_t k = 0; k < nsystems && st == SQN_OK; ++k) {
    // every system runs on a stream of its own (a branch of the graph)
    sqn_plan_desc d = descs[k];
    d.stream = nullptr;
    d.flags &= ~(uint32_t)SQN_FLAG_TIMING;
    sqn_plan *p = nullptr;
    const int ps = sqn_plan_create(&d, &p);
    if (ps > SQN_WARN_EPS_TOO_SMALL) {
      st = ps;
      break;
    }
    if (ps != SQN_OK) warn = ps;
    b->plans.push_back(p);
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) st = SQN_ERR_CUDA;
    b->joins.push_back(e);
  }
  if (st == SQN_OK) {
    cudaSetDevice(b->device);
    // every plan's set-up work is done before the capture starts
    for (sqn_plan *p : b->plans)
      if (st == SQN_OK && sync_plan(p) != SQN_OK) st = SQN_ERR_CUDA;
    if (st == SQN_OK && batch_multi_ok(b)) st = setup_batch_multi(b);
    if (st == SQN_OK) st = capture_batch(b);
  }
  if (st != SQN_OK) {
    free_batch(b);
    if (prev >= 0) cudaSetDevice(prev);
    return st;
  }
  if (prev >= 0) cudaSetDevice(prev);
  *out = b;
  return warn;
}

int sqn_batch_accumulate(sqn_batch *b, const double *const *pos, int64_t nframes,
                         int32_t where) {
  if (!b) return SQN_ERR_PLAN_NOTVALID;
  if (!pos || nframes < 0 || (where != SQN_HOST && where != SQN_DEVICE))
    return SQN_ERR_INVALID_ARGUMENT;
  for (size_t k = 0; k < b->plans.size(); ++k)
    if (!pos[k]) return SQN_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(b->device);
  const cudaMemcpyKind kind = where == SQN_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  for (int64_t f = 0; f < nframes; ++f) {
    // stage this frame of every system (in stream order after the previous
    // replay has read the staging buffers), then replay the graph
    for (size_t k = 0; k < b->plans.size(); ++k) {
      sqn_plan *p = b->plans[k];
      const size_t n3 = 3 * (size_t)p->desc.natoms;
      if (cudaMemcpyAsync(p->d_pos[0], pos[k] + n3 * (size_t)f, sizeof(double) * n3, kind,
                          b->root) != cudaSuccess)
        return SQN_ERR_CUDA;
    }
    if (cudaGraphLaunch(b->exec, b->root) != cudaSuccess) return SQN_ERR_CUDA;
    b->replays++;
    b->launches += b->launches_per_step;
    for (sqn_plan *p : b->plans) {
      p->nframes++;
      if (!b->multi) p->launches += frame_launches(p);
    }
  }
  return SQN_OK;
}

int sqn_batch_sync(sqn_batch *b) {
  if (!b) return SQN_ERR_PLAN_NOTVALID;
  DeviceGuard guard(b->device);
  return cuda_status(cudaStreamSynchronize(b->root));
}

int sqn_batch_plan(sqn_batch *b, int32_t system, sqn_plan **plan) {
  if (!b) return SQN_ERR_PLAN_NOTVALID;
  if (!plan || system < 0 || (size_t)system >= b->plans.size()) return SQN_ERR_INVALID_ARGUMENT;
  *plan = b->plans[(size_t)system];
  return SQN_OK;
}

int64_t sqn_batch_graph_launches(const sqn_batch *b) { return b ? b->replays : -1; }

int64_t sqn_batch_launch_count(const sqn_batch *b) { return b ? b->launches : -1; }

int32_t sqn_batch_multi(const sqn_batch *b) { return b ? (b->multi ? 1 : 0) : -1; }

int sqn_batch_destroy(sqn_batch *b) {
  if (!b) return SQN_ERR_PLAN_NOTVALID;
  free_batch(b);
  return SQN_OK;
}

}  // extern "C"
