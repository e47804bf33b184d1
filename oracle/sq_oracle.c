/*
 * CPU oracle for the static S(q) hot path of sqcalc.  TEST INFRASTRUCTURE ONLY:
 * the tests, the smoke check and the CPU-baseline leg of the benchmark load this
 * library as the checker; the product path (libsqnufft.so) never links or calls it.
 *
 * It is a plain FP64 restatement of the reference's direct method and of the
 * bookkeeping every static method shares (file:line refer to thatstar/sqcalc):
 *
 *   cell set up and fractional coordinates   src/sqc_cell.f90:131-141, :143-152, :225-241
 *   grid extent and mode enumeration         src/sqc_structure_factor.f90:329-381
 *   shell assignment, den, shell_count       src/sqc_structure_factor.f90:389-416
 *   mode_denominator                          src/sqc_structure_factor.f90:425-451
 *   amplitudes (unit, neutron, IT92 x-ray)   src/sqc_weights.f90:136-154, src/sqc_elements.f90:226-239
 *   direct_accumulate (total + partials)     src/sqc_structure_factor.f90:1398-1515
 *   accumulate_values (shell + grid sums)    src/sqc_structure_factor.f90:595-643
 *
 * Arithmetic follows the reference's operation order and is compiled without
 * floating-point contraction, so shell indices and |q| agree bit for bit with a
 * non-FMA build of the reference.  Parity of this restatement is pinned by the
 * golden vectors under tests/golden (produced by the reference's own numpy
 * reference test/ref_sq.py and by the known-answer cases of test/test_sqcalc.py).
 *
 * Layouts follow the Fortran arrays the reference uses:
 *   cell[9]      a(3,3) column major: cell[3*i + r] = component r of lattice vector i
 *   recip[9]     b(3,3) column major: recip[3*j + r] = component r of b_j
 *   pos[3*N]     frame%pos(3, N)
 *   partial[T*T*nq]  partial_num(ia, ib, shell), ia fastest
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SQO_WEIGHT_UNIT 0
#define SQO_WEIGHT_NEUTRON 1
#define SQO_WEIGHT_XRAY 2
#define SQO_NORM_MEAN 1
#define SQO_NORM_SELF 2
#define SQO_NORM_NATOM 3


int sqo_abi_version(void) { return 1; }

/* determinant3 / inverse3 of src/sqc_cell.f90:131-152 (m(r,c) = cell[3*c + r]). */
static double det3(const double *a) {
#define M(r, c) a[3 * ((c)-1) + ((r)-1)]
  return M(1, 1) * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)) -
         M(1, 2) * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1)) +
         M(1, 3) * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
}

/* inv(r,c) stored as inv[3*(c-1) + (r-1)], same column-major layout. */
static void inv3(const double *a, double *inv) {
  double det = det3(a);
#define I(r, c) inv[3 * ((c)-1) + ((r)-1)]
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
#undef I
}

/* cell_setup (src/sqc_cell.f90:131-141): b_j = 2 pi * row j of A^-1. */
void sqo_cell_setup(const double *cell, double *inv, double *recip) {
  const double two_pi = 2.0 * acos(-1.0);
  inv3(cell, inv);
  for (int j = 0; j < 3; ++j)
    for (int r = 0; r < 3; ++r) recip[3 * j + r] = two_pi * inv[3 * r + j];
}

/* Grid extent (src/sqc_structure_factor.f90:329-337). Returns 0, or 1 for a
 * degenerate cell. */
int sqo_modes(const double *cell, double qmax, int32_t *modes) {
  const double two_pi = 2.0 * acos(-1.0);
  for (int i = 0; i < 3; ++i) {
    const double *v = cell + 3 * i;
    double len = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (len <= 0.0) return 1;
    int32_t m = 2 * (int32_t)ceil(qmax * len / two_pi) + 1;
    modes[i] = m < 3 ? 3 : m;
  }
  return 0;
}

/* |q| of mode h in the reference's operation order (:366-368). */
static inline double qlen_of(const double *b, int h1, int h2, int h3, double *q) {
  for (int r = 0; r < 3; ++r)
    q[r] = b[r] * (double)h1 + b[3 + r] * (double)h2 + b[6 + r] * (double)h3;
  return sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
}

/* Two-pass enumeration of the kept modes (:352-381) plus the shell map (:389-399).
 * With hkl == NULL only the count is returned. */
int64_t sqo_enumerate(const double *recip, const int32_t *modes, double qmin, double qmax,
                      int32_t nq, int32_t *hkl, double *qvec, double *qlen, int64_t *gidx,
                      int32_t *shell) {
  int64_t n = 0;
  const double dq = (qmax - qmin) / (double)nq;
  for (int p3 = 1; p3 <= modes[2]; ++p3) {
    int h3 = p3 - (modes[2] + 1) / 2;
    for (int p2 = 1; p2 <= modes[1]; ++p2) {
      int h2 = p2 - (modes[1] + 1) / 2;
      for (int p1 = 1; p1 <= modes[0]; ++p1) {
        int h1 = p1 - (modes[0] + 1) / 2;
        if (h1 == 0 && h2 == 0 && h3 == 0) continue;
        double q[3];
        double ql = qlen_of(recip, h1, h2, h3, q);
        if (ql > qmax || ql < qmin) continue;
        if (hkl) {
          hkl[3 * n] = h1;
          hkl[3 * n + 1] = h2;
          hkl[3 * n + 2] = h3;
          qvec[3 * n] = q[0];
          qvec[3 * n + 1] = q[1];
          qvec[3 * n + 2] = q[2];
          qlen[n] = ql;
          gidx[n] = (int64_t)p1 + (int64_t)modes[0] * ((int64_t)p2 - 1 + (int64_t)modes[1] * ((int64_t)p3 - 1));
          int s = (int)((ql - qmin) / dq) + 1;
          if (s < 1) s = 1;
          if (s > nq) s = nq;
          shell[n] = s;
        }
        ++n;
      }
    }
  }
  return n;
}

/* scheme_amplitude (src/sqc_weights.f90:136-154) for a type id t (1-based).
 * amp_const[t-1] holds b for neutron weights; xray[9*(t-1) ..] holds a1..a4,
 * b1..b4, c of the IT92 row (src/sqc_elements.f90:226-239). */
static inline double amplitude(int kind, const double *amp_const, const double *xray, int t,
                               double q) {
  if (kind == SQO_WEIGHT_NEUTRON) return amp_const[t - 1];
  if (kind == SQO_WEIGHT_XRAY) {
    const double *c = xray + 9 * (t - 1);
    double stol2 = q / (4.0 * acos(-1.0));
    stol2 = stol2 * stol2;
    double f = c[8];
    for (int i = 0; i < 4; ++i) f = f + c[i] * exp(-c[4 + i] * stol2);
    return f;
  }
  return 1.0;
}

double sqo_amplitude(int kind, const double *amp_const, const double *xray, int t, double q) {
  return amplitude(kind, amp_const, xray, t, q);
}

/* mode_denominator (:425-451). */
double sqo_mode_denominator(int norm, int kind, const double *amp_const, const double *xray,
                            int32_t natoms, int32_t ntypes, const int32_t *type_counts, double q) {
  if (norm == SQO_NORM_NATOM) return (double)natoms;
  double sum_w = 0.0, sum_w2 = 0.0;
  for (int t = 1; t <= ntypes; ++t) {
    if (type_counts[t - 1] <= 0) continue;
    double w = amplitude(kind, amp_const, xray, t, q);
    sum_w = sum_w + (double)type_counts[t - 1] * w;
    sum_w2 = sum_w2 + (double)type_counts[t - 1] * w * w;
  }
  if (norm == SQO_NORM_MEAN) return sum_w * sum_w / (double)natoms;
  return sum_w2;
}

/* den(shell) and shell_count(shell) over the kept modes (:405-416). */
void sqo_shell_norms(int norm, int kind, const double *amp_const, const double *xray,
                     int32_t natoms, int32_t ntypes, const int32_t *type_counts, int64_t nmodes,
                     const double *qlen, const int32_t *shell, int32_t nq, double *den,
                     int64_t *shell_count) {
  for (int s = 0; s < nq; ++s) {
    den[s] = 0.0;
    shell_count[s] = 0;
  }
  for (int64_t i = 0; i < nmodes; ++i) {
    double d = sqo_mode_denominator(norm, kind, amp_const, xray, natoms, ntypes, type_counts,
                                    qlen[i]);
    den[shell[i] - 1] += d;
    shell_count[shell[i] - 1] += 1;
  }
}

/* Wrapped fractional coordinates of every atom (cell_fractional + s - floor(s),
 * src/sqc_cell.f90:143-152 and src/sqc_structure_factor.f90:1431-1435). */
void sqo_wrap(int64_t natoms, const double *pos, const double *cell, const double *origin,
              double *frac) {
  double inv[9];
  inv3(cell, inv);
  for (int64_t i = 0; i < natoms; ++i) {
    double d[3] = {pos[3 * i] - origin[0], pos[3 * i + 1] - origin[1], pos[3 * i + 2] - origin[2]};
    for (int r = 0; r < 3; ++r) {
      double s = inv[r] * d[0] + inv[3 + r] * d[1] + inv[6 + r] * d[2];
      frac[3 * i + r] = s - floor(s);
    }
  }
}

/* One frame of direct_accumulate (:1398-1515): intensity(im) = |sum_a amp_a rho_a|^2
 * and, with partials, partial_num(ia, ib, shell) += Re(rho_a conj(rho_b)) for the
 * type ids with atoms.  Atoms are grouped by type id exactly as direct_setup does
 * (:1350-1366) so every per-type sum runs in the reference's order. */
void sqo_direct_frame(int64_t natoms, const double *pos, const double *cell,
                      const double *origin, const int32_t *type_id, int32_t ntypes, int kind,
                      const double *amp_const, const double *xray, int64_t nmodes,
                      const double *qvec, const double *qlen, const int32_t *shell, int32_t nq,
                      int partials, double *intensity, double *partial_num) {
  double *frac = (double *)malloc(sizeof(double) * 3 * (size_t)natoms);
  double *cart = (double *)malloc(sizeof(double) * 3 * (size_t)natoms);
  int64_t *first = (int64_t *)calloc((size_t)ntypes + 2, sizeof(int64_t));
  int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)natoms);
  sqo_wrap(natoms, pos, cell, origin, frac);
  for (int64_t i = 0; i < natoms; ++i) {
    for (int r = 0; r < 3; ++r)
      cart[3 * i + r] = cell[r] * frac[3 * i] + cell[3 + r] * frac[3 * i + 1] + cell[6 + r] * frac[3 * i + 2];
    first[type_id[i] + 1] += 1;
  }
  first[1] = 0;
  for (int t = 1; t <= ntypes; ++t) first[t + 1] += first[t];
  {
    int64_t *cursor = (int64_t *)malloc(sizeof(int64_t) * ((size_t)ntypes + 2));
    memcpy(cursor, first, sizeof(int64_t) * ((size_t)ntypes + 2));
    for (int64_t i = 0; i < natoms; ++i) order[cursor[type_id[i]]++] = i;
    free(cursor);
  }
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  size_t pair_size = partials ? (size_t)ntypes * ntypes * nq : 0;
  double *local = partials ? (double *)calloc(pair_size * nthreads, sizeof(double)) : NULL;

#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double *acc_re = (double *)malloc(sizeof(double) * ntypes);
    double *acc_im = (double *)malloc(sizeof(double) * ntypes);
#pragma omp for schedule(static)
    for (int64_t im = 0; im < nmodes; ++im) {
      double qx = qvec[3 * im], qy = qvec[3 * im + 1], qz = qvec[3 * im + 2];
      double tre = 0.0, tim = 0.0;
      for (int t = 1; t <= ntypes; ++t) {
        double amp = amplitude(kind, amp_const, xray, t, qlen[im]);
        double are = 0.0, aim = 0.0;
        for (int64_t k = first[t]; k < first[t + 1]; ++k) {
          int64_t i = order[k];
          double phase = qx * cart[3 * i] + qy * cart[3 * i + 1] + qz * cart[3 * i + 2];
          are += cos(phase);
          aim += sin(phase);
        }
        acc_re[t - 1] = are;
        acc_im[t - 1] = aim;
        tre += amp * are;
        tim += amp * aim;
      }
      intensity[im] = tre * tre + tim * tim;
      if (partials) {
        int sh = shell[im] - 1;
        double *lp = local + pair_size * tid;
        for (int ia = 1; ia <= ntypes; ++ia) {
          if (first[ia + 1] == first[ia]) continue;
          for (int ib = ia; ib <= ntypes; ++ib) {
            if (first[ib + 1] == first[ib]) continue;
            double v = acc_re[ia - 1] * acc_re[ib - 1] + acc_im[ia - 1] * acc_im[ib - 1];
            lp[(size_t)(ia - 1) + (size_t)ntypes * ((size_t)(ib - 1) + (size_t)ntypes * sh)] += v;
          }
        }
      }
    }
    free(acc_re);
    free(acc_im);
  }
  if (partials) {
    for (int t = 0; t < nthreads; ++t)
      for (size_t k = 0; k < pair_size; ++k) partial_num[k] += local[pair_size * t + k];
    free(local);
  }
  free(frac);
  free(cart);
  free(first);
  free(order);
}

/* accumulate_values (:595-643): num(shell) += values, gnum(gidx) += values. */
void sqo_accumulate_values(int64_t nmodes, const double *values, const int32_t *shell,
                           const int64_t *gidx, double *num, double *gnum) {
  for (int64_t im = 0; im < nmodes; ++im) {
    num[shell[im] - 1] += values[im];
    if (gnum) gnum[gidx[im] - 1] += values[im];
  }
}

/* Direct-sum gradient of L = sum_s wgt[s] * num_frame(s) with respect to the
 * Cartesian positions, for q-independent per-atom strengths c_j:
 *   dL/dr_j = sum_modes wgt[shell] * 2 c_j Re( conj(T(q)) * i q * exp(i q.r_j) ),
 *   T(q) = sum_k c_k exp(i q.r_k).
 * This is the FP64 reference for the adjoint (there is no counterpart in sqcalc;
 * it differentiates the direct sum of src/sqc_structure_factor.f90:1440-1456). */
void sqo_direct_grad(int64_t natoms, const double *pos, const double *cell, const double *origin,
                     const double *strength, int64_t nmodes, const double *qvec,
                     const int32_t *shell, const double *wgt, double *grad) {
  double *frac = (double *)malloc(sizeof(double) * 3 * (size_t)natoms);
  double *cart = (double *)malloc(sizeof(double) * 3 * (size_t)natoms);
  double *tre = (double *)malloc(sizeof(double) * (size_t)nmodes);
  double *tim = (double *)malloc(sizeof(double) * (size_t)nmodes);
  sqo_wrap(natoms, pos, cell, origin, frac);
  for (int64_t i = 0; i < natoms; ++i)
    for (int r = 0; r < 3; ++r)
      cart[3 * i + r] = cell[r] * frac[3 * i] + cell[3 + r] * frac[3 * i + 1] + cell[6 + r] * frac[3 * i + 2];
#pragma omp parallel for schedule(static)
  for (int64_t im = 0; im < nmodes; ++im) {
    double re = 0.0, imv = 0.0;
    for (int64_t i = 0; i < natoms; ++i) {
      double ph = qvec[3 * im] * cart[3 * i] + qvec[3 * im + 1] * cart[3 * i + 1] + qvec[3 * im + 2] * cart[3 * i + 2];
      re += strength[i] * cos(ph);
      imv += strength[i] * sin(ph);
    }
    tre[im] = re;
    tim[im] = imv;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < natoms; ++i) {
    double g[3] = {0.0, 0.0, 0.0};
    for (int64_t im = 0; im < nmodes; ++im) {
      double ph = qvec[3 * im] * cart[3 * i] + qvec[3 * im + 1] * cart[3 * i + 1] + qvec[3 * im + 2] * cart[3 * i + 2];
      double c = cos(ph), s = sin(ph);
      /* Re(conj(T) * i * e^{i ph}) = Re((tre - i tim) * (i c - s)) = tim*c - tre*s */
      double f = wgt[shell[im] - 1] * 2.0 * strength[i] * (tim[im] * c - tre[im] * s);
      g[0] += f * qvec[3 * im];
      g[1] += f * qvec[3 * im + 1];
      g[2] += f * qvec[3 * im + 2];
    }
    grad[3 * i] = g[0];
    grad[3 * i + 1] = g[1];
    grad[3 * i + 2] = g[2];
  }
  free(frac);
  free(cart);
  free(tre);
  free(tim);
}
