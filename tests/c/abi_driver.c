/* A plain C99 caller of libsqnufft.so through include/sqnufft.h only, in the
 * order sqcalc's GPU method would call it (src/sqc_gpu.f90: gpu_setup ->
 * gpu_accumulate per frame -> write_results): sqn_default_desc, sqn_plan_create,
 * sqn_accumulate_frames with host positions, sqn_finalize, sqn_plan_destroy.
 * The system is generated here from a fixed linear congruential sequence
 * (L = 16 A, N = 1500, types 1 and 2 alternating, 2 frames, q_max 5, nq 50,
 * partials, FP64, eps 1e-10); S(q) is printed one value per line, then the
 * partial S(1-2), so that a test can compare it with the same plan built from
 * Python.  Exit status: 0, or the first nonzero library status. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "sqnufft.h"

static uint64_t lcg_state = 88172645463325252ull;
static double lcg_uniform(void) {
  lcg_state = lcg_state * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(lcg_state >> 11) * (1.0 / 9007199254740992.0);
}

int main(void) {
  enum { N = 1500, NFRAMES = 2, NQ = 50, NTYPES = 2 };
  const double box = 16.0;
  static int32_t type_id[N];
  static double pos[NFRAMES * N * 3];
  double S[NQ], Sp[NTYPES * NTYPES * NQ];
  sqn_plan_desc d;
  sqn_plan *plan = NULL;
  int64_t nframes = 0;
  int i, st;

  if (sqn_abi_version() != SQN_ABI_VERSION) {
    fprintf(stderr, "ABI %d, header %d\n", sqn_abi_version(), SQN_ABI_VERSION);
    return 1;
  }
  for (i = 0; i < N; ++i) type_id[i] = 1 + (i & 1);
  for (i = 0; i < NFRAMES * N * 3; ++i) pos[i] = box * lcg_uniform();

  sqn_default_desc(&d);
  for (i = 0; i < 9; ++i) d.cell[i] = (i % 4 == 0) ? box : 0.0;
  d.natoms = N;
  d.type_id = type_id;
  d.ntypes = NTYPES;
  d.weight = SQN_WEIGHT_UNIT;
  d.qmin = 0.0;
  d.qmax = 5.0;
  d.nq = NQ;
  d.norm = SQN_NORM_MEAN;
  d.partials = 1;
  d.precision = SQN_PREC_DOUBLE;
  d.eps = 1e-10;

  st = sqn_plan_create(&d, &plan);
  if (st > SQN_WARN_EPS_TOO_SMALL) {
    fprintf(stderr, "sqn_plan_create: %s\n", sqn_error_string(st));
    return st;
  }
  st = sqn_accumulate_frames(plan, pos, NFRAMES, SQN_HOST);
  if (st == SQN_OK) st = sqn_finalize(plan, 0, S, Sp, NULL, &nframes);
  if (st != SQN_OK) {
    fprintf(stderr, "frame path: %s\n", sqn_error_string(st));
    sqn_plan_destroy(plan);
    return st;
  }
  for (i = 0; i < NQ; ++i) printf("%.17g\n", S[i]);
  /* S(1-2): partial index (a-1) + T (b-1) + T T s, a = 1, b = 2 */
  for (i = 0; i < NQ; ++i) printf("%.17g\n", Sp[0 + NTYPES * 1 + NTYPES * NTYPES * i]);
  st = sqn_plan_destroy(plan);
  return nframes == NFRAMES ? st : 1;
}
