/*
 * CPU restatement of the NUFFT form of the static S(q) path.  Test and CPU-baseline
 * infrastructure only: it is the timed CPU baseline of the benchmark and a second
 * checker for the tests; the product path never links or calls it.
 *
 * The reference's CPU path is FINUFFT (sort, spread, FFTW, deconvolve; called
 * from src/sqc_structure_factor.f90:1165-1319) followed by the host partial and
 * shell sums (src/sqc_structure_factor.f90:457-643).  FINUFFT needs FFTW3 and
 * xsimd, neither of which exists in this image, so this file restates its math:
 *
 *   kernel width and ES beta     external/finufft/src/cuda/spreadinterp.cpp:59-85
 *   ES kernel                    external/finufft/include/cufinufft/spreadinterp.h:84-98
 *   fine grid size (2,3,5 even)  external/finufft/src/cuda/common.cu:166-177,
 *                                external/finufft/src/common/utils.cpp:124-143
 *   kernel Fourier series        external/finufft/src/cuda/common.cu:196-210 (Gauss-Legendre)
 *   deconvolution                external/finufft/src/cuda/deconvolve_wrapper.cu:76-118
 *
 * The FFT itself is done by the caller (numpy / scipy pocketfft, real-to-complex)
 * between sqo_spread_real() and sqo_bin_halfspace().  Strengths are real, so the
 * transform of the spread grid is Hermitian and only the half space h1 >= 0 is
 * visited; every mode with h1 > 0 also stands for its mirror -h.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* next235beven: smallest even n' >= n with prime factors 2, 3, 5 only. */
int64_t sqo_next235even(int64_t n) {
  if (n <= 2) return 2;
  if (n % 2 == 1) n += 1;
  for (int64_t c = n;; c += 2) {
    int64_t d = c;
    while (d % 2 == 0) d /= 2;
    while (d % 3 == 0) d /= 3;
    while (d % 5 == 0) d /= 5;
    if (d == 1) return c;
  }
}

/* Kernel width and shape for tolerance eps at upsampling factor sigma.  The
 * formulas are the published ES choices (Barnett, Magland, af Klinteberg 2019)
 * in the form cuFINUFFT uses them. */
void sqo_es_params(double eps, double sigma, int32_t *w_out, double *beta_out) {
  int w;
  if (sigma == 2.0)
    w = (int)ceil(-log10(eps / 10.0));
  else
    w = (int)ceil(-log(eps) / (acos(-1.0) * sqrt(1.0 - 1.0 / sigma)));
  if (w < 2) w = 2;
  if (w > 16) w = 16;
  double bw = 2.30;
  if (w == 2) bw = 2.20;
  if (w == 3) bw = 2.26;
  if (w == 4) bw = 2.38;
  if (sigma != 2.0) bw = 0.97 * acos(-1.0) * (1.0 - 1.0 / (2.0 * sigma));
  *w_out = w;
  *beta_out = bw * (double)w;
}

static inline double es_kernel(double t, int w, double beta) {
  double z = 2.0 * t / (double)w;
  double zz = z * z;
  if (zz >= 1.0) return 0.0;
  return exp(beta * (sqrt(1.0 - zz) - 1.0));
}

/* n-point Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n. */
static void gauss_legendre(int n, double *x, double *wt) {
  const double pi = acos(-1.0);
  for (int i = 0; i < n; ++i) {
    double z = cos(pi * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      /* p1 = P_n(z), p0 = P_{n-1}(z) */
      pp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    wt[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

/* phihat[k] = int phi(t) cos(2 pi k t / nf) dt for k = 0..kmax. */
void sqo_kernel_fseries(int64_t nf, int32_t w, double beta, int32_t kmax, double *phihat) {
  int n = 4 * w + 24;
  double *x = (double *)malloc(sizeof(double) * n), *wt = (double *)malloc(sizeof(double) * n);
  gauss_legendre(n, x, wt);
  const double half = 0.5 * w, pi = acos(-1.0);
  for (int k = 0; k <= kmax; ++k) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
      double t = 0.5 * half * (x[i] + 1.0); /* [0, w/2] */
      s += 0.5 * half * wt[i] * es_kernel(t, w, beta) * cos(2.0 * pi * (double)k * t / (double)nf);
    }
    phihat[k] = 2.0 * s;
  }
  free(x);
  free(wt);
}

/* Spread real strengths onto ntr real periodic grids grid[tr][nf3][nf2][nf1].
 * frac[3*N] are wrapped fractional coordinates in [0,1); tr_of[j] selects the
 * grid of atom j (or -1 to skip it); strength[j] is its real weight.  Planes
 * are split between threads so that no two threads write the same cell. */
void sqo_spread_real(int64_t natoms, const double *frac, const int32_t *tr_of,
                     const double *strength, int32_t ntr, const int64_t *nf, int32_t w,
                     double beta, double *grid) {
  const int64_t n1 = nf[0], n2 = nf[1], n3 = nf[2];
  const int64_t plane = n1 * n2, vol = plane * n3;
  memset(grid, 0, sizeof(double) * (size_t)(vol * ntr));
  /* bucket atoms by the first plane of their z support */
  int64_t *start = (int64_t *)calloc((size_t)n3 + 1, sizeof(int64_t));
  int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)natoms);
  int32_t *iz0 = (int32_t *)malloc(sizeof(int32_t) * (size_t)natoms);
  for (int64_t j = 0; j < natoms; ++j) {
    double X = (double)n3 * frac[3 * j + 2];
    int64_t i0 = (int64_t)ceil(X - 0.5 * w);
    int64_t iw = ((i0 % n3) + n3) % n3;
    iz0[j] = (int32_t)iw;
    start[iw + 1]++;
  }
  for (int64_t k = 0; k < n3; ++k) start[k + 1] += start[k];
  {
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n3 + 1));
    memcpy(cur, start, sizeof(int64_t) * (size_t)(n3 + 1));
    for (int64_t j = 0; j < natoms; ++j) order[cur[iz0[j]]++] = j;
    free(cur);
  }
#pragma omp parallel
  {
    int nth = 1, tid = 0;
#ifdef _OPENMP
    nth = omp_get_num_threads();
    tid = omp_get_thread_num();
#endif
    int64_t z0 = n3 * tid / nth, z1 = n3 * (tid + 1) / nth;
    double kx[16], ky[16], kz[16];
    int64_t blo = z0 - w + 1;
    if (z1 - blo > n3) blo = z1 - n3; /* one thread: visit every bucket once */
    for (int64_t b = blo; b < z1; ++b) {
      int64_t bw = ((b % n3) + n3) % n3;
      for (int64_t k = start[bw]; k < start[bw + 1]; ++k) {
        int64_t j = order[k];
        if (tr_of[j] < 0) continue;
        double c = strength[j];
        double X = (double)n1 * frac[3 * j], Y = (double)n2 * frac[3 * j + 1],
               Z = (double)n3 * frac[3 * j + 2];
        int64_t ix0 = (int64_t)ceil(X - 0.5 * w), iy0 = (int64_t)ceil(Y - 0.5 * w),
                izs = (int64_t)ceil(Z - 0.5 * w);
        for (int d = 0; d < w; ++d) {
          kx[d] = es_kernel((double)(ix0 + d) - X, w, beta);
          ky[d] = es_kernel((double)(iy0 + d) - Y, w, beta);
          kz[d] = es_kernel((double)(izs + d) - Z, w, beta);
        }
        double *g = grid + vol * tr_of[j];
        for (int dz = 0; dz < w; ++dz) {
          int64_t iz = ((izs + dz) % n3 + n3) % n3;
          if (iz < z0 || iz >= z1) continue;
          for (int dy = 0; dy < w; ++dy) {
            int64_t iy = ((iy0 + dy) % n2 + n2) % n2;
            double cyz = c * kz[dz] * ky[dy];
            double *row = g + iz * plane + iy * n1;
            for (int dx = 0; dx < w; ++dx) {
              int64_t ix = ((ix0 + dx) % n1 + n1) % n1;
              row[ix] += cyz * kx[dx];
            }
          }
        }
      }
    }
  }
  free(start);
  free(order);
  free(iz0);
}

/* Deconvolve the half-space transform G[tr][nf3][nf2][nf1/2+1] (complex,
 * interleaved re/im) and accumulate, for the kept modes, num(shell) +=
 * mult*|sum_tr amp_tr rho_tr|^2 and partial(tr_a, tr_b, shell) +=
 * mult*Re(rho_a conj(rho_b)) into pair slot a<=b (packed upper triangle,
 * slot = a*ntr - a*(a-1)/2 + (b-a)).  amp[tr] are q-independent amplitudes
 * (amp == NULL: unit).  mult is 2 for h1 > 0 (the mirror mode) and 1 on h1 = 0. */
void sqo_bin_halfspace(const double *G, int32_t ntr, const int64_t *nf, const int32_t *modes,
                       const double *recip, double qmin, double qmax, int32_t nq,
                       const double *phihat1, const double *phihat2, const double *phihat3,
                       const double *amp, double *num, double *partial) {
  const int64_t c1 = nf[0] / 2 + 1, n2 = nf[1], n3 = nf[2];
  const int64_t vol = c1 * n2 * n3;
  const int hm1 = (modes[0] - 1) / 2, hm2 = (modes[1] - 1) / 2, hm3 = (modes[2] - 1) / 2;
  const double dq = (qmax - qmin) / (double)nq;
  const int npair = ntr * (ntr + 1) / 2;
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  double *lnum = (double *)calloc((size_t)nq * nthreads, sizeof(double));
  double *lpar = (double *)calloc((size_t)nq * npair * nthreads, sizeof(double));
  const int rows = (2 * hm2 + 1) * (2 * hm3 + 1);
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double re[64], im[64];
    double *mynum = lnum + (size_t)nq * tid, *mypar = lpar + (size_t)nq * npair * tid;
#pragma omp for schedule(dynamic, 16)
    for (int r = 0; r < rows; ++r) {
      int h2 = r % (2 * hm2 + 1) - hm2, h3 = r / (2 * hm2 + 1) - hm3;
      int64_t ky = h2 >= 0 ? h2 : n2 + h2, kz = h3 >= 0 ? h3 : n3 + h3;
      double dyz = phihat2[abs(h2)] * phihat3[abs(h3)];
      for (int h1 = 0; h1 <= hm1; ++h1) {
        if (h1 == 0 && h2 == 0 && h3 == 0) continue;
        double q[3];
        for (int k = 0; k < 3; ++k)
          q[k] = recip[k] * (double)h1 + recip[3 + k] * (double)h2 + recip[6 + k] * (double)h3;
        double ql = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        if (ql > qmax || ql < qmin) continue;
        int s = (int)((ql - qmin) / dq);
        if (s < 0) s = 0;
        if (s > nq - 1) s = nq - 1;
        double mult = h1 > 0 ? 2.0 : 1.0;
        double inv = 1.0 / (phihat1[h1] * dyz);
        int64_t idx = (kz * n2 + ky) * c1 + h1;
        double tre = 0.0, tim = 0.0;
        for (int t = 0; t < ntr; ++t) {
          re[t] = G[2 * (vol * t + idx)] * inv;
          im[t] = G[2 * (vol * t + idx) + 1] * inv;
          double a = amp ? amp[t] : 1.0;
          tre += a * re[t];
          tim += a * im[t];
        }
        mynum[s] += mult * (tre * tre + tim * tim);
        int p = 0;
        for (int a = 0; a < ntr; ++a)
          for (int b = a; b < ntr; ++b, ++p)
            mypar[(size_t)nq * p + s] += mult * (re[a] * re[b] + im[a] * im[b]);
      }
    }
  }
  for (int t = 0; t < nthreads; ++t) {
    for (int s = 0; s < nq; ++s) num[s] += lnum[(size_t)nq * t + s];
    if (partial)
      for (int k = 0; k < nq * npair; ++k) partial[k] += lpar[(size_t)nq * npair * t + k];
  }
  free(lnum);
  free(lpar);
}

/*
 * Direct type-1 sum, the check of the library's cuFINUFFT-shaped entry points:
 *   fk[t][k] = sum_j c[t][j] exp(iflag i (k1 x_j + k2 y_j + k3 z_j))
 * for k_d in [-N_d/2, (N_d-1)/2], written in CMCL order (modeord 0, k1 fastest
 * from -N1/2) or FFT order (modeord 1, k = 0 first), as the direct transform
 * FINUFFT's own tests compare against (external/finufft/test/utils/
 * dirft3d.hpp:13-20).  c and fk hold interleaved (re, im) pairs; FP64.
 */
void sqo_dirft3d1(int64_t M, const double *x, const double *y, const double *z,
                  const double *c, int32_t ntr, int32_t iflag, int64_t N1, int64_t N2,
                  int64_t N3, int32_t modeord, double *fk) {
  const int64_t nm = N1 * N2 * N3;
  const double sg = iflag >= 0 ? 1.0 : -1.0;
#pragma omp parallel for schedule(static)
  for (int64_t m = 0; m < nm; ++m) {
    int64_t r = m;
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
    for (int32_t t = 0; t < ntr; ++t) {
      double sre = 0.0, sim = 0.0;
      for (int64_t j = 0; j < M; ++j) {
        const double ph = sg * ((double)k1 * x[j] + (double)k2 * y[j] + (double)k3 * z[j]);
        const double cr = cos(ph), si = sin(ph);
        const double are = c[2 * (t * M + j)], aim = c[2 * (t * M + j) + 1];
        sre += are * cr - aim * si;
        sim += are * si + aim * cr;
      }
      fk[2 * (t * nm + m)] = sre;
      fk[2 * (t * nm + m) + 1] = sim;
    }
  }
}
